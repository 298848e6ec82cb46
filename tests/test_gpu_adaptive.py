"""Two-level adaptive refinement (-m gpu): bbfmm_b200_set_first_m2l_level,
bbfmm_b200_set_target_region and AdaptiveSolver. The reference has uniform trees only, so the
oracle here is the FP64 direct sum.

* Local solves: with a target region below the first M2L level the passes run only over the
  region's cells and their neighbours; the region's results equal the unrestricted solve's.
* Partition: a solve whose local expansions start at level l + 1 returns, for every target,
  the sum over the sources in the 3 x 3 x 3 neighbourhood of its level-l ancestor -- checked
  against that restricted direct sum (FP64 solve, n = 8: relative L2 < 1e-6, the FMM's own
  approximation at these separations), with a target region that drops the near field of the
  inactive cells' targets.
* Composition: on a clustered set (four tight Gaussian clusters over a uniform background), the
  adaptive solve against the FP64 direct sum on 2,048 targets, half of them in heavy leaves:
  FP64 and mixed within 1.2x the error of the uniform FP64 solve at the fine depth; with no heavy
  leaf it is exactly the coarse solve.
* Batches (AdaptiveBatch): every set equal to its own AdaptiveSolver (FP64, 1e-12), graph replay
  bitwise equal to eager launches, mixed within 1.2x the error of the uniform solve at the fine
  depth per set (the larger of its FP64 and its mixed error).
"""
import numpy as np
import pytest

from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def _clustered(N, seed):
    rng = np.random.default_rng(seed)
    nb = N // 4
    c = rng.uniform(-0.3, 0.3, (4, 3))
    xc = c[rng.integers(0, 4, N - nb)] + 0.02 * rng.standard_normal((N - nb, 3))
    x = np.concatenate([rng.random((nb, 3)) - 0.5, np.clip(xc, -0.5, np.nextafter(0.5, 0))])
    return x, rng.uniform(-1.0, 1.0, N)


def test_first_m2l_level_gives_the_ancestor_neighbourhood():
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import leaf_of_particles, morton_to_grid
    rng = np.random.default_rng(3)
    N, lev, l = 30000, 4, 2
    x = rng.random((N, 3)) - 0.5
    q = rng.uniform(-1, 1, N)
    s = Solver(8, lev, 1.0, mode="d")
    s.set_particles(x)
    s.set_first_m2l_level(l + 1)
    # targets only in the level-l cells with an even Morton index
    active = (np.arange(8 ** l) % 2 == 0)
    s.set_target_region(l, active)
    got = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    s.close()
    anc, _ = leaf_of_particles(x, 1.0, l)
    g = np.stack(morton_to_grid(anc, l), 1)
    t = np.random.default_rng(4).choice(N, 600, replace=False)
    want = np.empty(t.size)
    for k, i in enumerate(t):
        near = np.all(np.abs(g - g[i]) <= 1, axis=1)
        near[i] = False
        r = np.linalg.norm(x[near] - x[i], axis=1)
        want[k] = q[i] * np.sum(q[near] / r)
    act = active[anc[t]]  # targets outside the region get no near field and are not checked
    assert rel_l2(got[t[act]], want[act]) < 1e-6, rel_l2(got[t[act]], want[act])
    assert np.all(np.isfinite(got))


@pytest.mark.parametrize("mode,n,slab", [("d", 8, 0), ("mixed", 8, 0), ("s", 4, 0), ("mixed", 8, 512),
                                         ("d", 4, 64)])
def test_local_solve_equals_the_unrestricted_solve(mode, n, slab):
    """A local solve (first M2L level above the region level) runs its passes only below the
    active cells and their neighbours, in compact row order, and skips the levels above: its
    results on the region's targets equal those of the same solve without the region (FP64 and
    mixed 1e-12, FP32 1e-5), and the other targets get 0. slab > 0 also cuts the compact leaf
    rows into slabs of that many cells."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200.fmm import leaf_of_particles
    x, q = _clustered(60000, 11)
    qd = torch.as_tensor(q, device="cuda")
    lev, R = 5, 3
    rng = np.random.default_rng(12)
    active = rng.random(8 ** R) < 0.1
    out = []
    for region in (False, True):
        s = Solver(n, lev, 1.0, mode=mode)
        if slab:
            s.set_leaf_slab(slab)
        s.set_particles(x)
        s.set_first_m2l_level(R + 1)
        if region:
            s.set_target_region(R, active)
        out.append(s.solve(qd).double().cpu().numpy())
        s.close()
    anc, _ = leaf_of_particles(x, 1.0, R, fp32=(mode == "s"))  # the solver's own cells
    act = active[anc]
    tol = 1e-5 if mode == "s" else 1e-12
    assert act.any() and rel_l2(out[1][act], out[0][act]) < tol, rel_l2(out[1][act], out[0][act])
    assert np.all(out[1][~act] == 0.0)


@pytest.mark.parametrize("mode", ["d", "mixed"])
def test_adaptive_solver_against_direct(mode):
    import torch
    from bbfmm_b200 import AdaptiveSolver, Solver
    from bbfmm_b200.fmm import direct, leaf_of_particles
    N = 400_000
    x, q = _clustered(N, 7)
    qd = torch.as_tensor(q, device="cuda")
    a = AdaptiveSolver(8, 4, 6, mode=mode, cap=256)
    a.set_particles(x)
    assert a.heavy_leaves > 0 and a.fine is not None
    got = a.solve(qd).double().cpu().numpy()
    u = Solver(8, 6, 1.0, mode="d")
    u.set_particles(x)
    uni = u.solve(qd).cpu().numpy()
    u.close()
    leaf, counts = leaf_of_particles(x, 1.0, 4)
    heavy = counts[leaf] > 256
    rng = np.random.default_rng(8)
    t = np.concatenate([rng.choice(np.nonzero(heavy)[0], 1024, replace=False),
                        rng.choice(np.nonzero(~heavy)[0], 1024, replace=False)]).astype(np.int32)
    ref = direct(torch.as_tensor(x, device="cuda"), qd, torch.as_tensor(t, device="cuda")).cpu().numpy()
    e_a, e_u = rel_l2(got[t], ref), rel_l2(uni[t], ref)
    print(f"adaptive ({mode}) {e_a:.3e}, uniform FP64 depth 6 {e_u:.3e}, heavy leaves {a.heavy_leaves}, "
          f"refined particles {a.fine_particles}")
    assert e_a <= 1.2 * e_u, (e_a, e_u)
    a.close()


def test_adaptive_without_heavy_leaves_is_the_coarse_solve():
    import torch
    from bbfmm_b200 import AdaptiveSolver, Solver
    rng = np.random.default_rng(9)
    x = rng.random((50000, 3)) - 0.5
    q = torch.as_tensor(rng.uniform(-1, 1, 50000), device="cuda")
    a = AdaptiveSolver(8, 4, 6, mode="mixed", cap=10_000)
    a.set_particles(x)
    assert a.fine is None
    s = Solver(8, 4, 1.0, mode="mixed")
    s.set_particles(x)
    assert torch.equal(a.solve(q), s.solve(q))
    a.close()
    s.close()


def _batch_sets(seed):
    rng = np.random.default_rng(seed)
    out = []
    for N, n, lev, clustered in [(60000, 8, 3, True), (50000, 8, 3, False), (80000, 4, 3, True),
                                 (30000, 8, 2, True), (40000, 8, 3, True)]:
        if clustered:
            x, _ = _clustered(N, int(rng.integers(1 << 30)))
        else:
            x = rng.random((N, 3)) - 0.5
        out.append((x, n, lev))
    q = rng.uniform(-1, 1, sum(len(x) for x, _, _ in out))
    return out, q


def test_adaptive_batch_matches_adaptive_solvers():
    """Every set of an adaptive batch (heavy leaves refined by two levels in a second, stacked
    batch) gets the result of an AdaptiveSolver of its own (FP64: 1e-12; the batch stacks sets,
    which changes no arithmetic but the autotuned offset split); graph replay equals eager
    launches bitwise."""
    import torch
    from bbfmm_b200 import AdaptiveBatch, AdaptiveSolver
    sets, q = _batch_sets(21)
    qd = torch.as_tensor(q, device="cuda")
    b = AdaptiveBatch(sets, mode="d", cap=256)
    assert b.refined is not None and b.heavy_leaves > 0
    eager = b.solve(qd, graph=False).cpu().numpy()
    g1 = b.solve(qd, graph=True).cpu().numpy()
    g2 = b.solve(qd, graph=True).cpu().numpy()
    assert np.array_equal(eager, g1) and np.array_equal(g1, g2)
    for k, (x, n, lev) in enumerate(sets):
        a0, a1 = b.offsets[k], b.offsets[k + 1]
        s = AdaptiveSolver(n, lev, lev + 2, mode="d", cap=256)
        s.set_particles(x)
        want = s.solve(qd[a0:a1]).cpu().numpy()
        s.close()
        assert rel_l2(eager[a0:a1], want) < 1e-12, (k, rel_l2(eager[a0:a1], want))
    b.close()


def test_adaptive_batch_mixed_against_direct():
    import torch
    from bbfmm_b200 import AdaptiveBatch, Solver
    from bbfmm_b200.fmm import direct
    sets, q = _batch_sets(22)
    qd = torch.as_tensor(q, device="cuda")
    b = AdaptiveBatch(sets, mode="mixed", cap=256)
    got = b.solve(qd).cpu().numpy()
    rng = np.random.default_rng(23)
    for k, (x, n, lev) in enumerate(sets):
        a0, a1 = b.offsets[k], b.offsets[k + 1]
        uni = {}
        for m in ("d", "mixed"):
            u = Solver(n, lev + 2, 1.0, mode=m)
            u.set_particles(x)
            uni[m] = u.solve(qd[a0:a1]).cpu().numpy()
            u.close()
        t = rng.choice(a1 - a0, 512, replace=False).astype(np.int32)
        ref = direct(torch.as_tensor(x, device="cuda"), qd[a0:a1], torch.as_tensor(t, device="cuda")).cpu().numpy()
        e_a, e_u, e_m = rel_l2(got[a0:a1][t], ref), rel_l2(uni["d"][t], ref), rel_l2(uni["mixed"][t], ref)
        print(f"set {k} (n={n}, depth {lev}): adaptive mixed {e_a:.3e}, uniform depth {lev + 2}: "
              f"FP64 {e_u:.3e}, mixed {e_m:.3e}")
        # the FMM's own error, or the mixed mode's rounding where that is larger (a set with few
        # particles per leaf, whose FP64 error falls below what FP32 near-field sums resolve)
        assert e_a <= 1.2 * max(e_u, e_m), (k, e_a, e_u, e_m)
    b.close()


@pytest.mark.parametrize("mode", ["d", "mixed"])
def test_adaptive_from_device_positions_equals_host_positions(mode):
    """AdaptiveBatch and AdaptiveSolver from positions already on the GPU -- trees and refinement
    plans built there (the plan's leaf assignment in the solver's own arithmetic) -- give the
    results of the host-built ones bit for bit."""
    import torch
    from bbfmm_b200 import AdaptiveBatch, AdaptiveSolver
    sets, q = _batch_sets(24)
    qd = torch.as_tensor(q, device="cuda")
    out = []
    for on_device in (False, True):
        ss = [(torch.as_tensor(x, device="cuda") if on_device else x, n, lev) for x, n, lev in sets]
        b = AdaptiveBatch(ss, mode=mode, cap=256)
        assert b.refined is not None and b.heavy_leaves > 0
        out.append(b.solve(qd, graph=False).cpu().numpy())
        b.close()
    assert np.isfinite(out[0]).all()
    assert np.array_equal(out[0], out[1])
    x, q1 = _clustered(100000, 7)
    q1d = torch.as_tensor(q1, device="cuda")
    res = []
    for on_device in (False, True):
        a = AdaptiveSolver(8, 3, 5, mode=mode, cap=256)
        a.set_particles(torch.as_tensor(x, device="cuda") if on_device else x)
        assert a.fine is not None
        res.append(a.solve(q1d).cpu().numpy())
        a.close()
    assert np.array_equal(res[0], res[1])
