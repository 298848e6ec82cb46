"""Host-side logic: depth formula, interaction counts, operator precompute properties."""
import numpy as np
import pytest

from bbfmm_b200 import operators as ops
from bbfmm_b200.fmm import reference_depth


def test_reference_depth_formula():
    # (int)log(N)/log(8) binds the cast to log(N) only (bbfmm.c:151-160)
    assert reference_depth(32768) == 3 and reference_depth(32768, 1) == 4
    assert reference_depth(4194304) == 6 and reference_depth(4194304, 1) == 7
    assert reference_depth(10) == 2 and reference_depth(1) == 2


def test_interaction_counts_full_tree():
    import bench
    tot = sum(bench.interactions_per_level(l) for l in range(2, 8))
    assert tot == 435_570_912
    assert sum(bench.interactions_per_level(l) for l in range(2, 5)) == 640_584


def test_ktable_and_offsets():
    t = ops.ktable()
    assert (t >= 0).sum() == 316 and t.max() == 315
    off = ops.offsets()
    for k, (vx, vy, vz) in enumerate(off):
        assert t[49 * (vx + 3) + 7 * (vy + 3) + (vz + 3)] == k


def test_operator_precompute_properties():
    U, E, s = ops.kernel_svd(4)
    n3, r = 64, 32
    Um = U.reshape(r, n3).T
    assert np.allclose(Um.T @ Um, np.eye(r), atol=1e-12)
    Ek = E.reshape(316, r, r).transpose(0, 2, 1)
    off = ops.offsets()
    idx = {tuple(v): k for k, v in enumerate(off)}
    for k, v in enumerate(off):  # symmetric kernel: E_{-v} = E_v^T
        assert np.allclose(Ek[idx[tuple(-v)]], Ek[k].T, rtol=1e-10, atol=1e-12 * np.abs(Ek[k]).max())
    assert np.all(np.diff(s) <= 1e-12 * s[0])


def test_operator_files_roundtrip(tmp_path):
    U, E, _ = ops.kernel_svd(4)
    ops.write_operator_files(str(tmp_path), 4, U, E, False)
    r, U2, E2 = ops.read_operator_files(str(tmp_path), 4, False)
    assert r == 32 and np.array_equal(U, U2) and np.array_equal(E, E2)


def test_kernel_operator_files_round_trip(tmp_path):
    """The 1/r^4 operators (the reference's ONEOVERR4 build) use the reference's file names
    and layout, stay apart from the 1/r files in one directory, and differ from them."""
    import numpy as np
    import pytest
    from bbfmm_b200 import operators as ops
    assert ops.operator_file_names(4, False, "oneoverr4") == ("oneoverr4K4.bin", "oneoverr4U4.bin")
    assert ops.operator_file_names(8, True, "oneoverr4") == ("soneoverr4K8.bin", "soneoverr4U8.bin")
    assert ops.operator_file_names(4, False) == ("laplacianK4.bin", "laplacianU4.bin")
    assert ops.operator_file_names(4, False, "laplacianforce") == ("laplacianforceK4.bin",
                                                                   "laplacianforceU4.bin")
    assert ops.homogeneity("laplacian") == 1 and ops.homogeneity("oneoverr4") == 4
    assert ops.homogeneity("laplacianforce") == 2
    # kernel ids of bbfmm_b200_set_kernel (include/bbfmm_b200.h)
    assert [ops.KERNELS[k][1] for k in ("laplacian", "laplacianforce", "oneoverr4")] == [0, 1, 2]
    with pytest.raises(ValueError):
        ops.operator_file_names(4, False, "yukawa")
    r4, U4, E4 = ops.load_operators(4, cache_dir=str(tmp_path), kernel="oneoverr4")
    r1, U1, E1 = ops.load_operators(4, cache_dir=str(tmp_path))
    assert r4 == r1 == 32
    assert (tmp_path / "oneoverr4K4.bin").exists() and (tmp_path / "laplacianK4.bin").exists()
    r, U, E = ops.read_operator_files(str(tmp_path), 4, False, "oneoverr4")
    assert np.array_equal(U, U4) and np.array_equal(E, E4)
    assert not np.allclose(np.abs(E4), np.abs(E1))
    _, Us, _ = ops.load_operators(4, single=True, cache_dir=str(tmp_path), kernel="oneoverr4")
    assert Us.dtype == np.float32 and np.allclose(Us, U4, rtol=1e-6, atol=1e-7)


def test_force_kernel_matrix_is_odd_and_compressed_by_one_basis():
    """x / r^3 (LAPLACIANFORCE) is odd in the separation, so over the symmetric offset set
    K_{-k} = -K_k^T (to rounding of the node coordinates), and the field-side singular
    vectors U of [K_0 ... K_315] also capture each K_k's source side: U U^T K_k U U^T keeps
    K_k to the size of the first dropped singular value, as it does for 1/r."""
    import numpy as np
    from bbfmm_b200 import operators as ops
    n, n3, r = 4, 64, 32
    offs = [tuple(o) for o in ops.offsets()]
    for kern in ("laplacianforce", "laplacian"):
        K0 = ops.kernel_matrix(n, kern)
        blk = lambda k: K0[:, k * n3:(k + 1) * n3]
        sign = -1.0 if kern == "laplacianforce" else 1.0
        for k in (0, 100, 200, 315):
            mk = offs.index(tuple(-v for v in offs[k]))
            assert np.allclose(blk(mk), sign * blk(k).T, rtol=1e-12, atol=1e-14 * np.abs(blk(k)).max())
        U = np.fromiter(ops.kernel_svd(n, kernel=kern)[0], float).reshape(r, n3).T  # (n3, r)
        _, sv, _ = np.linalg.svd(K0, full_matrices=False)
        P = U @ U.T
        worst = max(np.linalg.norm(blk(k) - P @ blk(k) @ P, 2) for k in range(316))
        assert worst < 2 * sv[r], (kern, worst / sv[r])  # ~0.3; a random basis gives ~300


def test_python_api_checks_buffer_sizes_before_the_c_abi():
    """The C-ABI takes bare pointers sized by the particle count the solver holds: the Python
    layer refuses shorter or longer charge arrays before any copy or launch (a bare solver
    object stands in for one on a GPU; nothing reaches the library)."""
    import torch
    from bbfmm_b200 import Batch, Solver
    from bbfmm_b200.fmm import direct
    s = Solver.__new__(Solver)
    s.torch, s.N, s.device, s.dtype, s.np_dtype, s.h = torch, 100, 0, torch.float64, np.float64, None
    for bad in (99, 101):
        with pytest.raises(ValueError, match="q has"):
            s.solve(torch.zeros(bad, dtype=torch.float64))
        with pytest.raises(ValueError, match="q has"):
            s.solve_fields(torch.zeros(bad, dtype=torch.float64))
        with pytest.raises(ValueError, match="q has"):
            s.solve_host(np.zeros(bad))
        with pytest.raises(ValueError, match="q has"):
            s.autotune(torch.zeros(bad, dtype=torch.float64))
    b = Batch.__new__(Batch)
    b.torch, b.N, b.device, b.dtype, b.h = torch, 50, 0, torch.float64, None
    with pytest.raises(ValueError, match="q has"):
        b.solve(torch.zeros(49, dtype=torch.float64))
    x, q, t = torch.zeros(10, 3, dtype=torch.float64), torch.zeros(10, dtype=torch.float64), torch.zeros(2)
    with pytest.raises(ValueError, match="xyz has"):
        direct(x[:9], q, t)
    with pytest.raises(ValueError, match="CUDA tensors"):
        direct(x, q, t)


def test_operator_cache_is_written_atomically(tmp_path):
    """Files appear complete or not at all (rename into place), and no temporaries remain."""
    from bbfmm_b200 import operators as ops
    r, U, E = ops.load_operators(4, single=True, cache_dir=str(tmp_path))
    sv = ops.singular_values(4, cache_dir=str(tmp_path))
    names = sorted(p.name for p in tmp_path.iterdir())
    assert names == ["laplacianK4.bin", "laplacianU4.bin", "sigma4.npy", "slaplacianK4.bin", "slaplacianU4.bin"]
    assert np.array_equal(ops.singular_values(4, cache_dir=str(tmp_path)), sv) and sv[0] == 1.0
    r2, U2, E2 = ops.read_operator_files(str(tmp_path), 4, True)
    assert r2 == r == 32 and np.array_equal(U2, U) and np.array_equal(E2, E)


def test_operator_text_files(tmp_path):
    """The text form of the operator files (the reference's ENABLE_ASCII_IO builds, .out):
    the cutoff on the first line of the U file, one %18.12e value per line, read back to
    13 significant digits."""
    from bbfmm_b200 import operators as ops
    assert ops.operator_file_names(8, True, "oneoverr4", ascii=True) == ("soneoverr4K8.out", "soneoverr4U8.out")
    U, E, _ = ops.kernel_svd(4)
    ops.write_operator_files(str(tmp_path), 4, U, E, False, ascii=True)
    lines = (tmp_path / "laplacianU4.out").read_text().splitlines()
    assert lines[0] == "32" and len(lines) == 1 + 64 * 32 and lines[1] == "%18.12e" % U[0]
    assert len((tmp_path / "laplacianK4.out").read_text().splitlines()) == 316 * 32 * 32
    r, U2, E2 = ops.read_operator_files(str(tmp_path), 4, False, ascii=True)
    assert r == 32 and np.allclose(U2, U, rtol=1e-12, atol=1e-15) and np.allclose(E2, E, rtol=1e-12, atol=1e-15)
    ops.write_operator_files(str(tmp_path), 4, U2, E2, True, ascii=True)
    _, Us, _ = ops.read_operator_files(str(tmp_path), 4, True, ascii=True)
    assert Us.dtype == np.float32 and np.array_equal(Us, U2.astype(np.float32))


def test_ascii_single_operator_text_rounds_once():
    """The FP32 reader of the reference's ENABLE_ASCII_IO operator text rounds each decimal once,
    as strtof does (fscanf "%f"), also where FP64 would land exactly between two FP32 values."""
    import ctypes
    from bbfmm_b200.operators import _parse_text
    libc = ctypes.CDLL(None)
    libc.strtof.restype = ctypes.c_float
    libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    a = np.float32(1.0)
    mid = (float(a) + float(np.nextafter(a, np.float32(2)))) / 2
    tokens = [repr(mid) + "0000000001", "0.1", "-3.25e-7", repr(mid)]
    assert float(tokens[0]) == mid  # FP64 alone loses the digits above the midpoint
    want = np.array([libc.strtof(t.encode(), None) for t in tokens], dtype=np.float32)
    got = _parse_text(tokens, True)
    assert got.dtype == np.float32 and np.array_equal(got, want)
    assert got[0] != np.float32(float(tokens[0]))  # the double rounding it avoids
    assert np.array_equal(_parse_text(tokens, False), np.array([float(t) for t in tokens]))


def _plan_brute(xyz, L, depth, cap, dtype):
    """Refinement plan by direct enumeration: each particle's leaf grid cell from truncated
    (x + L/2) / leaf length in `dtype` (the leaf sort's arithmetic), heavy leaves by count, and
    a particle selected when a heavy leaf lies within one cell of its own along every axis."""
    x = np.asarray(xyz, dtype)
    m = 2 ** depth
    inv = dtype(1) / (dtype(L) * dtype(0.5) ** depth)
    g = np.minimum(((x + dtype(L) / dtype(2)) * inv).astype(np.int64), m - 1)
    key = (g[:, 0] * m + g[:, 1]) * m + g[:, 2]
    cnt = np.bincount(key, minlength=m ** 3)
    hv = np.nonzero(cnt > cap)[0]
    hg = np.stack([hv // (m * m), (hv // m) % m, hv % m], 1)
    near = (np.abs(g[:, None, :] - hg[None, :, :]).max(2) <= 1).any(1)
    return cnt > cap, key, near


@pytest.mark.parametrize("fp32", [False, True])
def test_refinement_plan_equals_enumeration(fp32):
    """fmm.refinement_plan (heavy leaves, their neighbourhoods' particles, the heavy ones among
    them) against a direct enumeration in the leaf sort's own precision, on clustered points
    that include particles within FP32 rounding of leaf faces."""
    from bbfmm_b200.fmm import morton_to_grid, refinement_plan
    rng = np.random.default_rng(3)
    L, depth, cap = 1.0, 3, 40
    x = np.clip(rng.uniform(0.2, 0.8, (3, 3))[rng.integers(0, 3, 4000)] + 0.03 * rng.standard_normal((4000, 3)),
                0.0, np.nextafter(1.0, 0.0)) - 0.5
    # particles just below a leaf face in FP64 that round onto it in FP32
    face = -0.5 + np.arange(1, 8) / 8.0
    x[:7, 0] = face - 1e-12
    x[7:14, 1] = face - 1e-12
    heavy, sel, keep = refinement_plan(x, L, depth, cap, fp32=fp32)
    h_b, key, near = _plan_brute(x, L, depth, cap, np.float32 if fp32 else np.float64)
    gx, gy, gz = morton_to_grid(np.arange(8 ** depth), depth)
    m = 2 ** depth
    assert np.array_equal(heavy, h_b[(gx * m + gy) * m + gz])
    assert heavy.any() and not heavy.all()
    assert np.array_equal(sel, np.nonzero(near)[0])
    assert np.array_equal(keep, h_b[key[sel]])
    if fp32:  # the face particles change leaf between the two precisions
        assert not np.array_equal(_plan_brute(x, L, depth, cap, np.float64)[1], key)


@pytest.mark.parametrize("fp32", [False, True])
@pytest.mark.parametrize("L,depth", [(1.0, 3), (1.3, 4)])
def test_refinement_plan_on_tensors_equals_host_plan(fp32, L, depth):
    """The tensor form of the refinement plan (used for positions already on the GPU; run here on
    CPU tensors) gives the host plan bit for bit: heavy leaves, selected particles and the kept
    ones, with particles on and within rounding of leaf faces, and an L whose leaf length is not
    a power of two."""
    import torch
    from bbfmm_b200.fmm import refinement_plan
    rng = np.random.default_rng(5)
    N = 6000
    x = np.clip(rng.uniform(0.2, 0.8, (3, 3))[rng.integers(0, 3, N)] + 0.03 * rng.standard_normal((N, 3)),
                0.0, np.nextafter(1.0, 0.0)) * L - L / 2
    k = np.arange(1, 2 ** depth)
    face = -L / 2 + k * (L / 2 ** depth)
    x[:k.size, 0] = face
    x[k.size:2 * k.size, 1] = np.nextafter(face, -1.0)
    x[2 * k.size:2 * k.size + 2] = [[-L / 2] * 3, [L / 2] * 3]
    cap = 30
    want = refinement_plan(x, L, depth, cap, fp32=fp32)
    got = refinement_plan(torch.as_tensor(x), L, depth, cap, fp32=fp32)
    assert want[0].any() and want[1].size > 0
    for w, g in zip(want, got):
        assert np.array_equal(w, g.numpy())


def test_refinement_plan_of_an_empty_set_and_unknown_batch_kernel():
    """Host logic that runs before any device work: an empty set has no heavy leaves in either
    form of the plan, and a batch with an unknown kernel name is refused with ValueError."""
    import torch
    from bbfmm_b200 import Batch
    from bbfmm_b200.fmm import refinement_plan
    for x in (np.zeros((0, 3)), torch.zeros((0, 3), dtype=torch.float64)):
        heavy, sel, keep = refinement_plan(x, 1.0, 2, 4)
        assert len(heavy) == 64 and not np.asarray(heavy).any()
        assert len(sel) == 0 and len(keep) == 0
    with pytest.raises(ValueError):
        Batch([(np.zeros((1, 3)), 4, 2)], kernel="oneoverr3")
