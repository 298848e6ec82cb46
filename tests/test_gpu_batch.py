"""Batched uneven particle sets (-m gpu): a batch must give every set the result of a
single-set solver of the same (n, depth), because stacking only renumbers cells.

Tolerances: FP64 batch vs single solvers relative L2 1e-13 per set (the autotuner may pick a
different split of the M2L offsets, which changes the FP64 summation order); graph replay vs
eager launch bitwise; mixed-precision sets within 1.2x the FP64 error against the FP64
direct sum (plus 1e-9 absolute slack for sets whose FMM error is tiny).
"""
import numpy as np
import pytest

from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def _sets(seed, spec):
    """spec: list of (N, n, maxlev, kind) with kind 'u' (uniform) or 'c' (4-cluster, sigma 0.04)."""
    rng = np.random.default_rng(seed)
    out = []
    for N, n, lev, kind in spec:
        if kind == "u":
            x = rng.random((N, 3))
        else:
            c = rng.uniform(0.1, 0.9, (4, 3))
            x = np.clip(c[rng.integers(0, 4, N)] + 0.04 * rng.standard_normal((N, 3)), 0.0, np.nextafter(1.0, 0.0))
        out.append((x - 0.5, n, lev))
    q = rng.uniform(-1, 1, sum(s[0].shape[0] for s in out))
    return out, q


SPEC = [(5000, 8, 3, "u"), (12000, 4, 3, "c"), (0, 8, 3, "u"), (7000, 8, 3, "c"), (30000, 8, 4, "u"),
        (3000, 4, 2, "u"), (20000, 4, 3, "u"), (9000, 8, 4, "c")]


def _single(sets, q, offsets, mode, kernel="laplacian"):
    import torch
    from bbfmm_b200 import Solver
    out = np.zeros(q.size)
    for k, (x, n, lev) in enumerate(sets):
        a, b = offsets[k], offsets[k + 1]
        if b == a:
            continue
        s = Solver(n, lev, 1.0, mode=mode, kernel=kernel)
        s.set_particles(x)
        out[a:b] = s.solve(torch.as_tensor(q[a:b], device="cuda")).double().cpu().numpy()
        s.close()
    return out


def test_batch_matches_single_solvers():
    import torch
    from bbfmm_b200 import Batch
    sets, q = _sets(1, SPEC)
    b = Batch(sets, mode="d")
    assert len(b.groups()) == 4  # (4, 2), (4, 3), (8, 3), (8, 4)
    qd = torch.as_tensor(q, device="cuda")
    eager = b.solve(qd, graph=False).cpu().numpy()
    g1 = b.solve(qd, graph=True).cpu().numpy()
    g2 = b.solve(qd, graph=True).cpu().numpy()
    assert b.graph_nodes > 0
    assert np.array_equal(eager, g1) and np.array_equal(g1, g2)
    want = _single(sets, q, b.offsets, "d")
    for k in range(len(sets)):
        a, e = b.offsets[k], b.offsets[k + 1]
        if e > a:
            assert rel_l2(eager[a:e], want[a:e]) < 1e-13, k
    b.close()


def test_graph_reads_the_current_charges():
    import torch
    from bbfmm_b200 import Batch
    sets, q = _sets(2, SPEC[:4])
    b = Batch(sets, mode="d")
    qd = torch.as_tensor(q, device="cuda")
    out = torch.empty_like(qd)
    b.solve(qd, out=out, graph=True)
    first = out.cpu().numpy()
    qd.mul_(-2.0)  # same buffer, new values: the replayed graph must see them
    b.solve(qd, out=out, graph=True)
    assert np.allclose(out.cpu().numpy(), 4.0 * first, rtol=1e-12, atol=0)
    b.close()


def test_autotune_keeps_results():
    import torch
    from bbfmm_b200 import Batch
    sets, q = _sets(3, SPEC)
    b = Batch(sets, mode="d")
    qd = torch.as_tensor(q, device="cuda")
    before = b.solve(qd).cpu().numpy()
    groups = b.autotune(qd)
    for g in groups:
        assert g["p2p_threads"] in (64, 128, 256)
        assert all(x in (0, 1, 3, 7, 21) for x in g["m2l_groups"][2:])
    after = b.solve(qd).cpu().numpy()
    assert rel_l2(after, before) < 1e-13
    b.close()


def test_mixed_batch_error_vs_direct():
    import torch
    from bbfmm_b200 import Batch
    from bbfmm_b200.fmm import direct
    sets, q = _sets(4, [(20000, 8, 3, "u"), (40000, 8, 4, "c"), (30000, 4, 3, "u"), (60000, 8, 4, "u")])
    qd = torch.as_tensor(q, device="cuda")
    res = {}
    for mode in ("d", "mixed"):
        b = Batch(sets, mode=mode)
        res[mode] = b.solve(qd).double().cpu().numpy()
        b.close()
    rng = np.random.default_rng(5)
    for k, (x, n, lev) in enumerate(sets):
        a, e = b.offsets[k], b.offsets[k + 1]
        t = rng.choice(e - a, 512, replace=False).astype(np.int32)
        ref = direct(torch.as_tensor(x, device="cuda"), qd[a:e], torch.as_tensor(t, device="cuda")).cpu().numpy()
        err = {m: rel_l2(res[m][a:e][t], ref) for m in res}
        assert err["mixed"] <= 1.2 * err["d"] + 1e-9, (k, err)


@pytest.mark.parametrize("kernel", ["oneoverr4", "laplacianforce"])
def test_batch_other_kernels(kernel):
    """The 1/r^4 and x / r^3 kernels in a batch (bbfmm_b200_batch_set_kernel): FP64 sets equal
    single-set FP64 solvers of that kernel (relative L2 1e-13, as for 1/r), graph replay equals
    eager launch bitwise, and the mixed batch is within 1e-5 relative L2 of the FP64 batch per
    set (the mixed single-solver bound of these kernels)."""
    import torch
    from bbfmm_b200 import Batch
    sets, q = _sets(6, SPEC[:6])
    qd = torch.as_tensor(q, device="cuda")
    b = Batch(sets, mode="d", kernel=kernel)
    eager = b.solve(qd, graph=False).cpu().numpy()
    got = b.solve(qd, graph=True).cpu().numpy()
    assert np.array_equal(eager, got)
    b.close()
    want = _single(sets, q, b.offsets, "d", kernel)
    bm = Batch(sets, mode="mixed", kernel=kernel)
    mixed = bm.solve(qd).cpu().numpy()
    bm.close()
    for k in range(len(sets)):
        a, e = b.offsets[k], b.offsets[k + 1]
        if e > a:
            assert rel_l2(got[a:e], want[a:e]) < 1e-13, k
            assert rel_l2(mixed[a:e], got[a:e]) < 1e-5, (k, rel_l2(mixed[a:e], got[a:e]))


def test_mixed_mode_order4_single_solver(oracle_d):
    """Mixed mode with n = 4 (r = 32): FP64 M2L on CUDA cores, FP32 compensated near field."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200 import operators as ops
    from conftest import uniform_inputs
    x, q = uniform_inputs(20000, seed=8)
    _, U, E = ops.load_operators(4, single=False)
    want = oracle_d.fmm(x, q, 4, 3, U, E)
    s = Solver(4, 3, 1.0, mode="mixed")
    s.set_particles(x)
    got = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    assert rel_l2(got, want) < 1e-6  # FP32 reciprocal distances in the near field
    s.close()



def test_set_tuning_round_trip_and_groups_keep_results():
    """Launch choices set by hand (offset groups of the FP64 M2L, near-field block size) are
    reported back and keep the FP64 result to summation order (1e-13)."""
    import torch
    from bbfmm_b200 import Solver
    sets, q = _sets(9, [(60000, 8, 3, "c")])
    s = Solver(8, 3, 1.0, mode="d")
    s.set_particles(sets[0][0])
    qd = torch.as_tensor(q, device="cuda")
    a = s.solve(qd).cpu().numpy()
    t = s.tuning()
    t2 = dict(t, p2p_threads=64, m2l_groups=[0, 0, 3, 7] + [0] * 7)
    s.set_tuning(t2)
    assert s.tuning() == t2
    b = s.solve(qd).cpu().numpy()
    assert rel_l2(b, a) < 1e-13
    s.close()
