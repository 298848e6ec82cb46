"""Parity at the depths the headline workload runs (-m gpu): levels 5-7, where the class-major
grid has P = 16..64 cells per axis and the tensor-core M2L runs hundreds to thousands of its
two-box tiles per sibling class.

* FP64, n = 8, depth 5 (N = 262,144, 8 per leaf): the whole solve against the oracle FMM (its
  M2L spread over the host cores, Oracle.fmm_staged), relative L2 < 1e-12, and the multipoles
  of every level < 1e-13.
* Sampled M2L at levels 6 and 7, FP64 and mixed: the solver's M2L output of the level
  (bbfmm_b200_copy_m2l) on 384 cells -- the domain's corners, cells on the faces of the
  8 x 8 x 4 tile boxes of every sibling class, random cells -- against the oracle's M2L of the
  same cells from the solver's own multipoles of that level (interaction lists enumerated from
  the grid, Oracle.m2l_sample). FP64: 1e-12; mixed: 1e-6 relative L2 over the sampled rows
  (split-BF16 products with FP32 accumulation outside the FP64 leading block).
* Levels 2 and 3 (mixed): every cell of a single set's level-2 and level-3 M2L against the
  oracle, where the tensor-core kernel tiles 32 or 4 stacked sets' class grids at once, and a
  batch with partial set groups against single solvers.
* Mixed, n = 8, depth 6 (N = 524,288): the whole solve against the FP64 solve < 3e-7, its
  error against the FP64 direct sum on 2,048 targets within 1.2x of the FP64 solve's, and the
  tolerance-rank form (SVD cut 1e-8 -> rank 160) mixed vs FP64 at the same rank < 3e-7.

Partial tiles: at every level l >= 4 the class grid has P = 2^(l-1) cells per axis, a multiple
of the 8 x 8 x 4 box, so no level of a uniform tree has a partial box; the boxes at the edge of
the grid, whose source boxes reach outside it (zero-filled by the tensor copies), are what the
corner and face cells exercise.
"""
import numpy as np
import pytest

from conftest import uniform_inputs
from oracle.oracle import grid_to_morton, levsta, rel_l2

pytestmark = pytest.mark.gpu


def _solver(mode, lev, x, **kw):
    from bbfmm_b200 import Solver
    s = Solver(8, lev, 1.0, mode=mode, **kw)
    s.set_particles(x)
    return s


def test_fp64_depth5_matches_oracle(oracle_d):
    import torch
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(8, single=False)
    x, q = uniform_inputs(262_144, seed=51)
    want = oracle_d.fmm_staged(x, q, 8, 5, U, E)
    s = _solver("d", 5, x)
    got = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    assert rel_l2(got, want) < 1e-12, rel_l2(got, want)
    tree = oracle_d.build_tree(x, 5)
    _, P = oracle_d.upward(tree, x, q, 8, U)
    for lev in range(2, 6):
        lo = levsta(lev)
        assert rel_l2(s.multipoles(lev), P[lo * 256:(lo + 8 ** lev) * 256]) < 1e-13, lev
    s.close()


def _sample_cells(lev, seed):
    """Morton indices of level `lev`: the 8 corners, cells on the faces of the 8 x 8 x 4 tile
    boxes (parent coordinates 0, 7, 8 ... mod the box) of every sibling class, random cells."""
    rng = np.random.default_rng(seed)
    m, P = 2 ** lev, 2 ** (lev - 1)
    c = np.array([0, m - 1])
    pts = [np.stack(np.meshgrid(c, c, c, indexing="ij"), -1).reshape(-1, 3)]
    fx = np.unique(np.concatenate([np.arange(0, P, 8), np.arange(7, P, 8)]))
    fz = np.unique(np.concatenate([np.arange(0, P, 4), np.arange(3, P, 4)]))
    for cls in range(8):
        b = ((cls >> 2) & 1, (cls >> 1) & 1, cls & 1)
        px, py, pz = rng.choice(fx, 16), rng.choice(fx, 16), rng.choice(fz, 16)
        pts.append(np.stack([2 * px + b[0], 2 * py + b[1], 2 * pz + b[2]], -1))
    pts.append(rng.integers(0, m, (384 - 8 - 128, 3)))
    g = np.concatenate(pts)
    return grid_to_morton(g[:, 0], g[:, 1], g[:, 2], lev)


@pytest.mark.parametrize("mode,tol", [("d", 1e-12), ("mixed", 1e-6)])
@pytest.mark.parametrize("lev,N", [(6, 524_288), (7, 2_097_152)])
def test_m2l_level_matches_oracle_on_sampled_cells(oracle_d, mode, tol, lev, N):
    import torch
    from bbfmm_b200 import operators as ops
    _, _, E = ops.load_operators(8, single=False)
    x, q = uniform_inputs(N, seed=60 + lev)
    s = _solver(mode, lev, x)
    s.solve(torch.as_tensor(q, device="cuda"))
    torch.cuda.synchronize()
    M = s.multipoles(lev)
    got = s.m2l_output(lev)
    cells = _sample_cells(lev, lev)
    want = oracle_d.m2l_sample(lev, 256, E, M, cells)
    err = rel_l2(got[cells], want)
    print(f"level {lev} {mode}: sampled-cell M2L relL2 {err:.3e}")
    assert err < tol, err
    # every row's own error, so that one wrong tile cannot hide in the sum
    row = np.linalg.norm(got[cells] - want, axis=1) / np.linalg.norm(want, axis=1)
    assert row.max() < 50 * tol, (row.max(), cells[row.argmax()])
    s.close()


def force_tc(solver, levels):
    """M2L kind 2 (the tensor cores wherever they tile the level) at the given levels."""
    t = solver.tuning()
    for lev in levels:
        t["m2l_kind"][lev] = 2
    solver.set_tuning(t)


def test_m2l_levels_2_3_stacked_set_tiles(oracle_d):
    """Levels 2 and 3 on the tensor cores, whose 2 x 2 x 2 and 4 x 4 x 4 class grids the two-box
    kernel tiles 32 and 4 stacked sets at a time. One set with those levels put on the tensor
    cores (kind 2; by default a single set keeps them in FP64; the other slots of each tile load
    it again and are not written): every cell of both levels against the oracle's M2L of the
    solver's own multipoles, mixed tolerance 1e-6. A batch of depth-2, depth-3 and depth-4 sets
    (a full and a partial group of four at level 3) gives each set the result of its own mixed
    solver."""
    import torch
    from bbfmm_b200 import Batch, Solver
    from bbfmm_b200 import operators as ops
    _, _, E = ops.load_operators(8, single=False)
    x, q = uniform_inputs(40_000, seed=33)
    s = _solver("mixed", 3, x)
    force_tc(s, (2, 3))  # a single set keeps levels 2-3 in FP64 by default
    s.solve(torch.as_tensor(q, device="cuda"))
    torch.cuda.synchronize()
    for lev in (2, 3):
        cells = np.arange(8 ** lev)
        want = oracle_d.m2l_sample(lev, 256, E, s.multipoles(lev), cells)
        got = s.m2l_output(lev)
        err = rel_l2(got, want)
        row = np.linalg.norm(got - want, axis=1) / np.linalg.norm(want, axis=1)
        print(f"level {lev} mixed: M2L relL2 {err:.3e}, worst row {row.max():.3e}")
        assert err < 1e-6 and row.max() < 5e-5, (lev, err, row.max())
    s.close()
    rng = np.random.default_rng(34)
    sets = [(rng.random((int(rng.integers(5000, 30000)), 3)) - 0.5, 8, 3) for _ in range(6)]
    sets += [(rng.random((40000, 3)) - 0.5, 8, 4), (rng.random((3000, 3)) - 0.5, 8, 2),
             (rng.random((2500, 3)) - 0.5, 8, 2)]
    qs = rng.uniform(-1, 1, sum(len(a) for a, _, _ in sets))
    qd = torch.as_tensor(qs, device="cuda")
    b = Batch(sets, mode="mixed")
    got = b.solve(qd).cpu().numpy()
    stacked = {lev: sum(1 for _, _, lv in sets if lv == lev) > 1 for _, _, lev in sets}
    for k, (xs, n, lev) in enumerate(sets):
        a0, a1 = b.offsets[k], b.offsets[k + 1]
        one = Solver(n, lev, 1.0, mode="mixed")
        one.set_particles(xs)
        if stacked[lev]:  # the batch runs this group's levels 2-3 on the tensor cores
            force_tc(one, (2, 3))
        want = one.solve(qd[a0:a1]).cpu().numpy()
        one.close()
        assert rel_l2(got[a0:a1], want) < 1e-12, (k, rel_l2(got[a0:a1], want))
    b.close()


def test_mixed_depth6_against_fp64_and_direct():
    import torch
    from bbfmm_b200.fmm import direct
    x, q = uniform_inputs(524_288, seed=66)
    qd = torch.as_tensor(q, device="cuda")
    out = {}
    for mode in ("mixed", "d"):
        s = _solver(mode, 6, x)
        out[mode] = s.solve(qd).cpu().numpy()
        s.close()
    assert rel_l2(out["mixed"], out["d"]) < 3e-7, rel_l2(out["mixed"], out["d"])
    t = np.random.default_rng(6).choice(x.shape[0], 2048, replace=False).astype(np.int32)
    ref = direct(torch.as_tensor(x, device="cuda"), qd, torch.as_tensor(t, device="cuda")).cpu().numpy()
    e_mixed, e_d = rel_l2(out["mixed"][t], ref), rel_l2(out["d"][t], ref)
    assert e_mixed <= 1.2 * e_d, (e_mixed, e_d)
    # tolerance rank at the same depth
    res = {}
    for mode in ("mixed", "d"):
        s = _solver(mode, 6, x, tol=1e-8)
        assert s.rank == 160
        res[mode] = s.solve(qd).cpu().numpy()
        s.close()
    assert rel_l2(res["mixed"], res["d"]) < 3e-7, rel_l2(res["mixed"], res["d"])
