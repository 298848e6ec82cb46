"""CUDA path vs the CPU oracle on identical seeded inputs and operators (-m gpu).

Tolerances (relative L2 over all particles):
  mode d (FP64): 1e-12 against the FP64 oracle (summation order only).
  mode s (FP32): 2e-5 against the FP32 oracle (FP32 order/FMA differences; the FP32
                 oracle itself differs from the reference SINGLE build by ~2e-7).
"""
import numpy as np
import pytest

from conftest import uniform_inputs
from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def _solve(mode, n, maxlev, x, q, U, E):
    import torch
    from bbfmm_b200 import Solver
    s = Solver(n, maxlev, 1.0, mode=mode, operators=(U, E))
    s.set_particles(x)
    dt = torch.float32 if mode == "s" else torch.float64
    phi = s.solve(torch.as_tensor(q, dtype=dt, device="cuda"))
    torch.cuda.synchronize()
    out = phi.cpu().numpy()
    return s, out


@pytest.mark.parametrize("n,maxlev,N", [(4, 2, 4096), (4, 3, 32768), (4, 4, 32768), (8, 3, 32768)])
def test_fp64_matches_oracle(oracle_d, n, maxlev, N):
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(n, single=False)
    x, q = uniform_inputs(N, seed=n * 10 + maxlev)
    ref = oracle_d.fmm(x, q, n, maxlev, U, E)
    s, got = _solve("d", n, maxlev, x, q, U, E)
    assert rel_l2(got, ref) < 1e-12
    # multipoles of every level in the reference's cell order
    tree = oracle_d.build_tree(x, maxlev)
    _, P = oracle_d.upward(tree, x, q, n, U)
    r = n ** 3 // 2
    for lev in range(2, maxlev + 1):
        lo = (8 ** lev - 1) // 7
        want = P[lo * r:(lo + 8 ** lev) * r]
        assert rel_l2(s.multipoles(lev), want) < 1e-13
    s.close()


@pytest.mark.parametrize("n,maxlev,N", [(4, 3, 32768), (8, 3, 32768)])
def test_fp32_matches_oracle(oracle_s, n, maxlev, N):
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(n, single=True)
    x, q = uniform_inputs(N, seed=7, dtype="float32")
    ref = oracle_s.fmm(x, q, n, maxlev, U, E)
    s, got = _solve("s", n, maxlev, x, q, U, E)
    assert rel_l2(got, ref) < 2e-5
    s.close()


def test_fp64_against_direct(oracle_d):
    """Absolute accuracy: FP64 FMM vs the FP64 direct sum on sampled targets matches the
    oracle FMM's own error (n=8 truncation error ~1e-7)."""
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(8, single=False)
    x, q = uniform_inputs(32768, seed=3)
    targets = np.random.default_rng(0).choice(32768, 1024, replace=False).astype(np.int32)
    dref = oracle_d.direct_fp64(x, q, targets)
    s, got = _solve("d", 8, 3, x, q, U, E)
    err = rel_l2(got[targets], dref)
    assert err < 5e-7
    s.close()


@pytest.mark.parametrize("case", ["one_leaf", "boundary", "sparse", "single"])
def test_edge_cases_fp64(oracle_d, case):
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(4, single=False)
    rng = np.random.default_rng(5)
    if case == "one_leaf":          # every particle in one leaf, all others empty
        x = rng.random((500, 3)) * 0.1 - 0.45
    elif case == "boundary":        # particles exactly on the faces and corners of the root
        x = rng.random((600, 3)) - 0.5
        x[:100, 0] = 0.5; x[100:200, 1] = -0.5; x[200:220] = 0.5; x[220:240] = -0.5
    elif case == "sparse":          # far fewer particles than leaves
        x = rng.random((37, 3)) - 0.5
    else:
        x = np.array([[0.1, -0.2, 0.3]])
    q = rng.uniform(-1, 1, x.shape[0])
    ref = oracle_d.fmm(x, q, 4, 3, U, E)
    s, got = _solve("d", 4, 3, x, q, U, E)
    assert np.all(np.isfinite(got))
    if np.linalg.norm(ref) == 0:
        assert np.linalg.norm(got) == 0
    else:
        assert rel_l2(got, ref) < 1e-12
    s.close()


def test_host_entry_matches_device_entry():
    from bbfmm_b200 import operators as ops
    import torch
    from bbfmm_b200 import Solver
    _, U, E = ops.load_operators(4, single=False)
    x, q = uniform_inputs(20000, seed=11)
    s = Solver(4, 3, 1.0, mode="d", operators=(U, E))
    s.set_particles(x)
    a = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    b = s.solve_host(q)
    assert np.array_equal(a, b)
    s.close()


def _clustered(N, seed, k=4, sigma=0.02):
    rng = np.random.default_rng(seed)
    c = rng.uniform(-0.4, 0.4, (k, 3))
    x = np.clip(c[rng.integers(0, k, N)] + sigma * rng.standard_normal((N, 3)), -0.5, np.nextafter(0.5, 0))
    return x, rng.uniform(-1.0, 1.0, N)


@pytest.mark.parametrize("mode,tol", [(0, 1e-13), (2, 1e-6)])
@pytest.mark.parametrize("layout", ["dense", "sparse", "clustered"])
def test_near_field_entry_matches_oracle(oracle_d, mode, tol, layout):
    """bbfmm_b200_near_field on caller-owned device arrays vs the oracle's P2P
    (anotherNearField semantics). FP64 mode: 1e-13; mixed mode (FP32 reciprocal distances): 1e-6.
    Layouts: ~12 particles per leaf (every 4 x 4 x 4 block is split into per-leaf chunks),
    ~1.5 per leaf (whole blocks staged at once), and 4 tight clusters at depth 5 (both kinds,
    empty blocks, and leaves of several hundred particles whose neighbourhoods stream through
    shared memory in many tiles)."""
    import ctypes as C
    import torch
    from bbfmm_b200 import _lib
    N, lev = 50000, {"dense": 4, "sparse": 5, "clustered": 5}[layout]
    x, q = _clustered(N, 32) if layout == "clustered" else uniform_inputs(N, seed=31)
    tree = oracle_d.build_tree(x, lev)
    want = oracle_d.nearfield(tree, x, q, np.zeros(N))
    perm = np.zeros(N, dtype=np.int32)
    ls = np.zeros(8 ** lev + 1, dtype=np.int32)
    xc = np.ascontiguousarray(x)
    _lib.check(_lib.lib().bbfmm_b200_sort_particles(N, 0, C.c_void_p(xc.ctypes.data), 1.0, lev,
                                                    perm.ctypes.data_as(C.POINTER(C.c_int)),
                                                    ls.ctypes.data_as(C.POINTER(C.c_int))))
    assert np.array_equal(perm, tree.fieldlist)          # same leaf order as the reference
    xyzq = np.concatenate([x[perm], q[perm, None]], axis=1)
    dx = torch.as_tensor(xyzq, device="cuda")
    dl = torch.as_tensor(ls, device="cuda")
    phi = torch.zeros(N, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    _lib.check(_lib.lib().bbfmm_b200_near_field(N, lev, 1.0, C.c_void_p(dx.data_ptr()), C.c_void_p(dl.data_ptr()),
                                                C.c_void_p(phi.data_ptr()), mode, None))
    got = np.empty(N)
    got[perm] = phi.cpu().numpy()
    assert rel_l2(got, want) < tol


@pytest.mark.parametrize("mode,n", [("d", 8), ("mixed", 8), ("s", 4)])
def test_leaf_slabs_are_bitwise_identical(mode, n):
    """The leaf level processed in slabs of 64 / 512 leaves (P2M -> projection -> M2M and
    projection -> L2L -> L2P per slab) gives exactly the whole-level result."""
    import torch
    from bbfmm_b200 import Solver
    x, q = uniform_inputs(40000, seed=12)
    s = Solver(n, 4, 1.0, mode=mode)
    s.set_particles(x)
    qd = torch.as_tensor(q, device="cuda")
    whole = s.solve(qd).cpu().numpy()
    p0, f0 = s.solve_fields(qd)
    for cells in (64, 512):
        s.set_leaf_slab(cells)
        assert np.array_equal(s.solve(qd).cpu().numpy(), whole), cells
        p, f = s.solve_fields(qd)
        assert torch.equal(p, p0) and torch.equal(f, f0), cells
    s.close()


def _compact(U, E, n, rank):
    """Rank-`rank` operators in the compact reference layout (U: n^3 x rank, E: rank x rank blocks)."""
    n3, r = n ** 3, n ** 3 // 2
    Uc = np.ascontiguousarray(np.asarray(U).reshape(r, n3)[:rank]).reshape(-1)
    Ec = np.ascontiguousarray(np.asarray(E).reshape(316, r, r)[:, :rank, :rank]).reshape(-1)
    return Uc, Ec


def test_tolerance_rank_matches_truncated_oracle(oracle_d):
    """An SVD cut at relative singular value 1e-8 (rank 147 -> 160): the solver's zero-padded
    rank-160 operators with the zero blocks skipped equal the oracle FMM run with the compact
    rank-160 operators (FP64, 1e-12)."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200 import operators as ops
    rank = ops.tolerance_rank(8, 1e-8)
    assert rank == 160
    x, q = uniform_inputs(20000, seed=14)
    _, U, E = ops.load_operators(8, single=False)
    want = oracle_d.fmm(x, q, 8, 3, *_compact(U, E, 8, rank))
    s = Solver(8, 3, 1.0, mode="d", tol=1e-8)
    assert s.rank == rank
    s.set_particles(x)
    got = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    assert rel_l2(got, want) < 1e-12
    s.close()


def test_tolerance_rank_mixed_matches_fp64_rank():
    """Mixed precision at rank 160 (tensor-core M2L with N = 160, K-chunks up to 160; down
    projection K = 160) against the FP64 solve at the same rank: 3e-7."""
    import torch
    from bbfmm_b200 import Solver
    x, q = uniform_inputs(40000, seed=15)
    qd = torch.as_tensor(q, device="cuda")
    out = {}
    for mode in ("mixed", "d"):
        s = Solver(8, 4, 1.0, mode=mode, rank=160)
        s.set_particles(x)
        out[mode] = s.solve(qd).cpu().numpy()
        s.close()
    assert rel_l2(out["mixed"], out["d"]) < 3e-7


def test_tolerance_rank_fp32_matches_fp64_rank():
    """FP32 mode with an SVD cut at 1e-5 (the FP32 tolerance of the 4M-particle workload): the
    CUDA-core M2L contracts over the rank and writes zeros above it; against the FP64 solve at
    the same rank: 2e-5 (FP32 arithmetic throughout)."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200 import operators as ops
    rank = ops.tolerance_rank(8, 1e-5)
    assert rank < 256
    x, q = uniform_inputs(20000, seed=16)
    out = {}
    for mode in ("s", "d"):
        s = Solver(8, 3, 1.0, mode=mode, tol=1e-5)
        assert s.rank == rank
        s.set_particles(x)
        dt = torch.float32 if mode == "s" else torch.float64
        out[mode] = s.solve(torch.as_tensor(q, dtype=dt, device="cuda")).double().cpu().numpy()
        s.close()
    assert rel_l2(out["s"], out["d"]) < 2e-5


@pytest.mark.parametrize("kernel,mode,tol", [("oneoverr4", "d", 1e-12), ("oneoverr4", "s", 2e-5),
                                             ("laplacianforce", "d", 1e-12), ("laplacianforce", "s", 1e-4)])
def test_other_kernels_match_oracle(oracle_d, oracle_s, kernel, mode, tol):
    """The reference's other kernels against the oracle with the same operators: 1/r^4
    (ONEOVERR4; homogeneity 4: near field q / r^4 and the per-level scale (1/L_l)^4) and
    x / r^3 (LAPLACIANFORCE; homogeneity 2: near field q dx / r^3 with dx = x_source -
    x_target, scale (1/L_l)^2). FP32 tolerance for x / r^3: the FP32 oracle itself is 1.8e-5
    from the FP64 oracle on this input (odd kernel, cancelling near-field sums), so two FP32
    summation orders may differ by about that much."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200 import operators as ops
    single = mode == "s"
    _, U, E = ops.load_operators(4, single=single, kernel=kernel)
    x, q = uniform_inputs(30000, seed=17)
    O = oracle_s if single else oracle_d
    want = O.fmm(x, q, 4, 3, U, E, homogen=ops.homogeneity(kernel))
    s = Solver(4, 3, 1.0, mode=mode, kernel=kernel)
    s.set_particles(x)
    dt = torch.float32 if single else torch.float64
    got = s.solve(torch.as_tensor(q, dtype=dt, device="cuda")).double().cpu().numpy()
    assert rel_l2(got, want) < tol
    s.close()


@pytest.mark.parametrize("kernel", ["oneoverr4", "laplacianforce"])
def test_other_kernels_mixed_mode(oracle_d, kernel):
    """The mixed mode for 1/r^4 and x / r^3 (n = 8, depth 4): the same product map and leading
    FP64 block as for 1/r on that kernel's operators; the near-field pair value dx rinv^3 in FP32
    from the FP64 separation with the compensated sum, rinv^4 in FP64 (its FP64 FMM error, 3e-11,
    is below what FP32 pair terms resolve). Against the FP64 direct sum of the kernel on 2,048
    targets: within 1.2x the error of the FP64 solve; against the FP64 solve: relative L2 below
    1e-5. Field solves stay refused for these kernels."""
    import torch
    from bbfmm_b200 import Solver
    from bbfmm_b200 import operators as ops
    from bbfmm_b200._lib import BBFMMError
    x, q = uniform_inputs(65536, seed=19)
    qd = torch.as_tensor(q, device="cuda")
    out = {}
    for mode in ("mixed", "d"):
        s = Solver(8, 4, 1.0, mode=mode, kernel=kernel)
        s.set_particles(x)
        out[mode] = s.solve(qd).cpu().numpy()
        if mode == "mixed":
            with pytest.raises(BBFMMError):
                s.solve_fields(qd)
        s.close()
    t = np.random.default_rng(19).choice(65536, 2048, replace=False).astype(np.int32)
    ref = oracle_d.direct_fp64(x, q, t, homogen=ops.homogeneity(kernel))
    e_mixed, e_d = rel_l2(out["mixed"][t], ref), rel_l2(out["d"][t], ref)
    print(f"{kernel}: mixed vs direct {e_mixed:.3e}, FP64 vs direct {e_d:.3e}, "
          f"mixed vs FP64 {rel_l2(out['mixed'], out['d']):.3e}")
    assert e_mixed <= 1.2 * e_d, (e_mixed, e_d)
    assert rel_l2(out["mixed"], out["d"]) < 1e-5
