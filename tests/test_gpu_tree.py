"""The octree built on the GPU (bbfmm_b200_set_particles_device) against the host build
(bbfmm_b200_set_particles): the same particle order and leaf ranges, so every solve is bitwise
the same (-m gpu)."""
import numpy as np
import pytest

from conftest import uniform_inputs

pytestmark = pytest.mark.gpu


def _inputs(kind, N, seed):
    rng = np.random.default_rng(seed)
    if kind == "uniform":
        x, q = uniform_inputs(N, seed=seed)
    elif kind == "clustered":
        c = rng.uniform(-0.4, 0.4, (3, 3))
        x = (c[rng.integers(0, 3, N)] + 0.01 * rng.standard_normal((N, 3))).clip(-0.5, 0.5)
        x[N // 2:N // 2 + 50] = x[:50]  # coincident particles keep their original order
        q = rng.uniform(-1, 1, N)
    else:  # points on leaf faces (depth 4: multiples of 1/16) and on the root boundary
        g = rng.integers(-8, 9, (N, 3)) / 16.0
        jitter = rng.random((N, 3)) < 0.5
        x = np.where(jitter, (rng.random((N, 3)) - 0.5), g)
        x[:6] = [[-0.5, -0.5, -0.5], [0.5, 0.5, 0.5], [0.5, -0.5, 0.0], [0.0, 0.0, 0.0],
                 [-0.5, 0.5, 0.25], [0.0625, -0.0625, 0.5]]
        q = rng.uniform(-1, 1, N)
    return np.ascontiguousarray(x, dtype=np.float64), q


@pytest.mark.parametrize("kind,N,mode,n,lev", [
    ("uniform", 40000, "d", 4, 4),
    ("uniform", 4097, "mixed", 8, 3),       # two radix blocks, the second with one particle
    ("clustered", 30011, "mixed", 8, 4),
    ("faces", 20000, "d", 4, 4),
    ("faces", 20000, "s", 4, 4),
    ("uniform", 1, "d", 4, 2),
])
def test_device_tree_solves_bitwise_like_host_tree(kind, N, mode, n, lev):
    import torch
    from bbfmm_b200 import Solver
    x, q = _inputs(kind, N, 21)
    dt = torch.float32 if mode == "s" else torch.float64
    qd = torch.as_tensor(q, dtype=dt, device="cuda")
    out = []
    for device_tree in (False, True):
        s = Solver(n, lev, 1.0, mode=mode)
        s.set_particles(torch.as_tensor(x, dtype=dt, device="cuda") if device_tree else x)
        out.append(s.solve(qd).cpu().numpy())
        s.close()
    assert np.isfinite(out[0]).all()
    assert np.array_equal(out[0], out[1])


def test_device_tree_rejects_particles_outside_the_root():
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200._lib import BBFMMError
    x, _ = uniform_inputs(1000, seed=3)
    x[17, 1] = 0.5000001
    s = Solver(4, 3, 1.0, mode="d")
    with pytest.raises(BBFMMError):
        s.set_particles(torch.as_tensor(x, device="cuda"))
    s.close()


def _batch_sets(seed):
    """Sets of four (n, depth) groups: several radix blocks in one group, an empty set, 20 small
    sets in one group (set slots above the leaf bits of the sort keys), clustered sets with
    coincident points, points on leaf faces and on the root boundary."""
    rng = np.random.default_rng(seed)
    spec = [("uniform", 5000, 8, 3), ("clustered", 7001, 4, 3), (None, 0, 8, 3), ("faces", 3000, 4, 3),
            ("uniform", 20000, 8, 4), ("clustered", 4097, 8, 3), ("uniform", 1, 4, 2)]
    spec += [("uniform", int(k), 4, 2) for k in rng.integers(50, 500, 20)]
    sets, qs = [], []
    for j, (kind, N, n, lev) in enumerate(spec):
        if kind is None:
            x, q = np.zeros((0, 3)), np.zeros(0)
        else:
            x, q = _inputs(kind, N, seed + j)
        sets.append((x, n, lev))
        qs.append(q)
    return sets, np.concatenate(qs)


@pytest.mark.parametrize("mode", ["d", "s", "mixed"])
def test_batch_device_trees_solve_bitwise_like_host_trees(mode):
    """bbfmm_b200_batch_create_device: each group's trees from one device sort over (set, leaf)
    keys give every set the host sort's particle order and leaf ranges, so the batch solves
    bitwise the same as a batch whose trees were sorted on the host."""
    import torch
    from bbfmm_b200 import Batch
    sets, q = _batch_sets(31)
    dt = torch.float32 if mode == "s" else torch.float64
    qd = torch.as_tensor(q, dtype=dt, device="cuda")
    out = []
    for on_device in (False, True):
        ss = [(torch.as_tensor(x, dtype=dt, device="cuda") if on_device else x, n, lev) for x, n, lev in sets]
        b = Batch(ss, mode=mode)
        assert len(b.groups()) == 4
        out.append(b.solve(qd, graph=False).cpu().numpy())
        b.close()
    assert np.isfinite(out[0]).all()
    assert np.array_equal(out[0], out[1])


def test_batch_device_trees_reject_particles_outside_the_root():
    import torch
    from bbfmm_b200 import Batch
    from bbfmm_b200._lib import BBFMMError
    sets, _ = _batch_sets(32)
    x = sets[3][0].copy()
    x[5, 2] = -0.5000001
    ss = [(torch.as_tensor(xx if k != 3 else x, device="cuda"), n, lev) for k, (xx, n, lev) in enumerate(sets)]
    with pytest.raises(BBFMMError):
        Batch(ss, mode="d")
