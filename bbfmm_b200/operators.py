"""Chebyshev tables and SVD-compressed M2L operators (host, FP64) for the reference's
homogeneous kernels: 1/r (LAPLACIAN, the default), x/r^3 (LAPLACIANFORCE) and 1/r^4
(ONEOVERR4).

This is set-up work, not the solve: it runs once per interpolation order ``n`` and
its output is cached in the reference's operator-file format so that the same
operators can be fed to the reference code, to the CPU oracle and to the CUDA path.

What is computed, and the reference function each piece restates:

* ``chebyshev_tables(n)`` -> nodes, ``Tkz`` (n x n), ``Kweights`` (n^3),
  ``Cweights`` (2 n^2), ``Ktable`` (343)  -- ``ComputeWeights`` (bbfmm.c:922-1028),
  ``ComputeTk`` (bbfmm.c:1626-1633), ``ComputeSn`` (bbfmm.c:1641-1679).
* ``kernel_svd(n)`` -> ``U`` (n^3 x r, column-major) and ``E`` (316 r x r,
  column-major per offset)  -- ``ComputeKernelSVD`` (bbfmm.c:1209-1421).
  The rank is the reference's fixed cutoff r = n^3/2 (bbfmm.c:1340-1343).
* ``write_operator_files`` / ``read_operator_files`` -- the binary layout of
  ``[s]laplacian{K,U}{n}.bin``: U file = int32 cutoff + n^3 r reals, K file = 316 r^2
  reals (bbfmm.c:1361-1405 writer, bbfmm.c:216-254 reader).

The SVD itself goes through LAPACK (numpy), as the reference's ``?gesvd`` call does;
the left singular vectors are taken from an R factor of the transposed kernel matrix
(``K0^T = Q R`` so ``K0 = R^T Q^T`` and the left singular vectors of ``K0`` are those of
``R^T``), which never forms the 316 n^3-wide right singular vectors.
"""
from __future__ import annotations

import io
import os
import struct
from dataclasses import dataclass

import numpy as np

NUM_OFFSETS = 316  # |[-3,3]^3 \ [-1,1]^3|

# The reference's compile-time kernels (bbfmm.c:109-144, 798-849): name -> (degree of
# homogeneity, kernel id of the C-ABI). "laplacianforce" is x / r^3 with x the first component
# of source - field (LAPLACIANFORCE). It is odd in the separation, so K_{-k} = -K_k^T over the
# symmetric set of 316 offsets: the field-side singular vectors of [K_0 ... K_315] also span
# every K_k's source side, and E_k = U^T K_k U compresses it as it does the even kernels.
KERNELS = {"laplacian": (1, 0), "laplacianforce": (2, 1), "oneoverr4": (4, 2)}


def homogeneity(kernel: str) -> int:
    return KERNELS[kernel][0]


def _kernel_values(kernel: str, d: np.ndarray) -> np.ndarray:
    """K at separations d = source - field (..., 3), as the reference's EvaluateKernel
    (bbfmm.c:798-849)."""
    r = np.sqrt(np.einsum("...x,...x->...", d, d))
    rinv = 1.0 / r
    if kernel == "laplacian":
        return rinv
    if kernel == "laplacianforce":
        return d[..., 0] * rinv * rinv * rinv
    if kernel == "oneoverr4":
        return rinv * rinv * rinv * rinv
    raise ValueError(f"unknown kernel {kernel!r} ({', '.join(KERNELS)})")


def ktable() -> np.ndarray:
    """Offset (vx,vy,vz) in [-3,3]^3 -> operator index k in [0,316), -1 for near cells.

    Index layout ``49*(vx+3) + 7*(vy+3) + (vz+3)`` (m2l_aux.c:3-26, bbfmm.c:937-950)."""
    t = np.full(343, -1, dtype=np.int32)
    k = 0
    c = 0
    for vx in range(-3, 4):
        for vy in range(-3, 4):
            for vz in range(-3, 4):
                if abs(vx) > 1 or abs(vy) > 1 or abs(vz) > 1:
                    t[c] = k
                    k += 1
                c += 1
    return t


def offsets() -> np.ndarray:
    """(316, 3) int array: the offset (vx, vy, vz) of each operator index k."""
    out = []
    for vx in range(-3, 4):
        for vy in range(-3, 4):
            for vz in range(-3, 4):
                if abs(vx) > 1 or abs(vy) > 1 or abs(vz) > 1:
                    out.append((vx, vy, vz))
    return np.asarray(out, dtype=np.int32)


def _tk(x: float, n: int) -> np.ndarray:
    """T_0..T_{n-1}(x) by the three-term recurrence (bbfmm.c:1626-1633)."""
    v = np.zeros(n)
    v[0] = 1.0
    if n > 1:
        v[1] = x
    for k in range(2, n):
        v[k] = 2 * x * v[k - 1] - v[k - 2]
    return v


def sn_clenshaw(tk_row: np.ndarray, x: np.ndarray) -> np.ndarray:
    """S(x_m, x) = 1/2 + sum_{k>=1} T_k(x_m) T_k(x) by Clenshaw (bbfmm.c:1682-1690).

    ``tk_row`` holds T_k(x_m) for k < n; ``x`` is any array of points in [-1, 1]."""
    n = tk_row.shape[0]
    x = np.asarray(x, dtype=np.float64)
    d1 = np.zeros_like(x)  # d[j+1]
    d2 = np.zeros_like(x)  # d[j+2]
    for j in range(n - 1, 0, -1):
        d0 = 2 * x * d1 - d2 + tk_row[j]
        d2 = d1
        d1 = d0
    return x * d1 - d2 + 0.5 * tk_row[0]


@dataclass
class ChebTables:
    n: int
    nodes: np.ndarray     # (n,)
    Tkz: np.ndarray       # (n*n,)  Tkz[m*n+k] = T_k(x_m)
    Kweights: np.ndarray  # (n^3,)  prod_axis 1/sqrt(1-x^2), index l1*n^2+l2*n+l3
    Cweights: np.ndarray  # (2*n^2,) Cweights[side*n^2 + p*n + c] = S(x_p, (x_c -/+ 1)/2)
    Ktable: np.ndarray    # (343,) int32


def chebyshev_tables(n: int) -> ChebTables:
    """Restates ``ComputeWeights`` (bbfmm.c:922-1028) in FP64."""
    nodes = np.cos(np.pi * (2 * np.arange(n) + 1) / (2 * n))
    Tkz = np.stack([_tk(nodes[m], n) for m in range(n)]).reshape(-1)
    w = 1.0 / np.sqrt(1.0 - nodes * nodes)
    Kweights = (w[:, None, None] * w[None, :, None] * w[None, None, :]).reshape(-1)
    C = np.zeros((2, n, n))
    for side, shift in ((0, -1.0), (1, 1.0)):
        xc = 0.5 * (nodes + shift)
        for p in range(n):
            C[side, p, :] = sn_clenshaw(Tkz[p * n:(p + 1) * n], xc)
    return ChebTables(n, nodes, Tkz, Kweights, C.reshape(-1), ktable())


def kernel_matrix(n: int, kernel: str = "laplacian") -> np.ndarray:
    """K0 (n^3 x 316 n^3): the weighted kernel between unit-cell field nodes and the nodes of
    the 316 well-separated unit cells, block k = columns [k n^3, (k+1) n^3).

    Entry (i, k n^3 + j) = K(s_j - f_i) / (w_i w_j) with f at 0.5*nodes and s at
    offset_k + 0.5*nodes (bbfmm.c:1247-1324), K = 1/r, x/r^3 or 1/r^4."""
    tab = chebyshev_tables(n)
    h = 0.5 * tab.nodes
    g = np.stack(np.meshgrid(h, h, h, indexing="ij"), axis=-1).reshape(-1, 3)  # (n3, 3)
    offs = offsets().astype(np.float64)
    n3 = n ** 3
    w = tab.Kweights
    ww = w[:, None] * w[None, :]
    K = np.empty((n3, NUM_OFFSETS * n3))
    for k in range(NUM_OFFSETS):
        src = offs[k][None, :] + g                      # (n3, 3)
        d = src[None, :, :] - g[:, None, :]             # (n3 field, n3 source, 3)
        K[:, k * n3:(k + 1) * n3] = _kernel_values(kernel, d) / ww
    return K


def kernel_svd(n: int, rank: int | None = None, kernel: str = "laplacian"):
    """Returns (U, E, sigma): U column-major (n^3, r) flattened, E (316, r, r) as
    column-major blocks flattened, sigma all n^3 singular values.

    Restates ``ComputeKernelSVD`` (bbfmm.c:1209-1421): SVD of K0, keep r = n^3/2
    leading left singular vectors, E_k = U^T K_k U (the right factor reuses U,
    bbfmm.c:1384-1405; for the odd x / r^3 kernel too, see KERNELS)."""
    n3 = n ** 3
    r = n3 // 2 if rank is None else rank
    K0 = kernel_matrix(n, kernel)
    R = np.linalg.qr(K0.T, mode="r")          # (n3, n3), K0 = R^T Q^T
    Ul, s, _ = np.linalg.svd(R.T)
    U = np.ascontiguousarray(Ul[:, :r])       # (n3, r)
    E = np.empty((NUM_OFFSETS, r, r))
    for k in range(NUM_OFFSETS):
        Kk = K0[:, k * n3:(k + 1) * n3]
        E[k] = U.T @ Kk @ U
    # column-major storage: element (i, j) of block k at k r^2 + j r + i
    Ucol = U.T.reshape(-1).copy()             # U(i, j) at j*n3 + i
    Ecol = np.ascontiguousarray(E.transpose(0, 2, 1)).reshape(-1)
    return Ucol, Ecol, s


def operator_file_names(n: int, single: bool, kernel: str = "laplacian", ascii: bool = False) -> tuple[str, str]:
    """The reference's file names (bbfmm.c:96-144): [s]laplacian{K,U}{n}.bin,
    [s]laplacianforce{K,U}{n}.bin, [s]oneoverr4{K,U}{n}.bin; extension .out for the text
    form of its ENABLE_ASCII_IO builds."""
    if kernel not in KERNELS:
        raise ValueError(f"unknown kernel {kernel!r} ({', '.join(KERNELS)})")
    p = "s" if single else ""
    ext = "out" if ascii else "bin"
    return f"{p}{kernel}K{n}.{ext}", f"{p}{kernel}U{n}.{ext}"


def _ascii_lines(values) -> bytes:
    # one "%18.12e" line per value, as the reference's fprintf (bbfmm.c:1366-1370, 1398-1400)
    return "".join("%18.12e\n" % v for v in np.asarray(values, np.float64).tolist()).encode()


def _write_atomic(path: str, *chunks: bytes):
    """Write a file under a private name, then rename it into place: processes that share the
    cache (one per GPU) see either no file or a complete one."""
    tmp = f"{path}.{os.getpid()}.tmp"
    with open(tmp, "wb") as f:
        for c in chunks:
            f.write(c)
    os.replace(tmp, path)


def write_operator_files(dirpath: str, n: int, Ucol: np.ndarray, Ecol: np.ndarray, single: bool,
                         kernel: str = "laplacian", ascii: bool = False):
    """Write ``[s]<kernel>{K,U}{n}.bin`` in the reference layout (bbfmm.c:1361-1405); with
    ``ascii`` the text form ``.out`` of its ENABLE_ASCII_IO builds (the cutoff, then one value
    per line; values rounded to 13 significant digits, as that form holds them)."""
    os.makedirs(dirpath, exist_ok=True)
    kname, uname = operator_file_names(n, single, kernel, ascii)
    dt = np.float32 if single else np.float64
    r = Ucol.size // n ** 3
    U = np.asarray(Ucol, dtype=dt)
    E = np.asarray(Ecol, dtype=dt)
    if ascii:
        _write_atomic(os.path.join(dirpath, uname), b"%d\n" % r, _ascii_lines(U))
        _write_atomic(os.path.join(dirpath, kname), _ascii_lines(E))
        return
    _write_atomic(os.path.join(dirpath, uname), struct.pack("i", r), U.tobytes())
    _write_atomic(os.path.join(dirpath, kname), E.tobytes())


def _parse_text(tokens, single: bool):
    """Decimal tokens -> FP64, or FP32 correctly rounded from the decimal as strtof gives it.
    Going through FP64 rounds twice, which differs from one rounding only where the FP64 value
    lies exactly halfway between two FP32 values; those tokens are parsed again by strtof."""
    d = np.array(tokens, dtype=np.float64)
    if not single:
        return d
    f = d.astype(np.float32)
    bits = d.view(np.int64)
    tie = (bits & ((1 << 29) - 1)) == (1 << 28)  # low 29 of the 52 mantissa bits: a float32 midpoint
    if tie.any():
        import ctypes
        libc = ctypes.CDLL(None)
        libc.strtof.restype = ctypes.c_float
        libc.strtof.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
        for i in np.nonzero(tie)[0]:
            f[i] = libc.strtof(tokens[i].encode(), None)
    return f


def read_operator_files(dirpath: str, n: int, single: bool, kernel: str = "laplacian", ascii: bool = False):
    """Read ``[s]<kernel>{K,U}{n}.bin`` (bbfmm.c:216-254), or with ``ascii`` the ``.out`` text
    form of the reference's ENABLE_ASCII_IO builds. Returns (r, Ucol, Ecol)."""
    kname, uname = operator_file_names(n, single, kernel, ascii)
    dt = np.float32 if single else np.float64
    if ascii:
        u = open(os.path.join(dirpath, uname)).read().split()
        r = int(u[0])
        # as fscanf "%f" / "%lf" read the text: correctly rounded to the file's precision
        Ucol = _parse_text(u[1:1 + n ** 3 * r], single)
        e = open(os.path.join(dirpath, kname)).read().split()
        Ecol = _parse_text(e[:NUM_OFFSETS * r * r], single)
        if Ucol.size != n ** 3 * r or Ecol.size != NUM_OFFSETS * r * r:
            raise ValueError("operator text files are shorter than their cutoff implies")
        return r, Ucol, Ecol
    with open(os.path.join(dirpath, uname), "rb") as f:
        r = struct.unpack("i", f.read(4))[0]
        Ucol = np.frombuffer(f.read(), dtype=dt, count=n ** 3 * r).copy()
    with open(os.path.join(dirpath, kname), "rb") as f:
        Ecol = np.frombuffer(f.read(), dtype=dt, count=NUM_OFFSETS * r * r).copy()
    return r, Ucol, Ecol


def default_cache_dir() -> str:
    return os.environ.get(
        "BBFMM_B200_OPERATOR_DIR",
        os.path.join(os.path.expanduser("~"), ".cache", "bbfmm_b200", "operators"))


def singular_values(n: int, cache_dir: str | None = None, kernel: str = "laplacian") -> np.ndarray:
    """Singular values of the FP64 kernel matrix K0 of order n, relative to the largest
    (cached as sigma{n}.npy, sigma_<kernel>{n}.npy for other kernels, beside the operator
    files)."""
    cache_dir = cache_dir or default_cache_dir()
    tag = "" if kernel == "laplacian" else f"_{kernel}"
    path = os.path.join(cache_dir, f"sigma{tag}{n}.npy")
    if os.path.exists(path):
        return np.load(path)
    K0 = kernel_matrix(n, kernel)
    R = np.linalg.qr(K0.T, mode="r")
    sv = np.linalg.svd(R.T, compute_uv=False)
    sv = sv / sv[0]
    os.makedirs(cache_dir, exist_ok=True)
    buf = io.BytesIO()
    np.save(buf, sv)
    _write_atomic(path, buf.getvalue())
    return sv


def tolerance_rank(n: int, tol: float, multiple: int = 32, cache_dir: str | None = None,
                   kernel: str = "laplacian") -> int:
    """Rank of an SVD cut at relative singular value `tol` (the number of sigma_j / sigma_0 >= tol),
    rounded up to `multiple` (the kernels' component granularity) and capped at n^3 / 2."""
    sv = singular_values(n, cache_dir, kernel)
    r = int((sv >= tol).sum())
    r = -(-r // multiple) * multiple
    return max(multiple, min(r, n ** 3 // 2))


def truncate_operators(n: int, Ucol: np.ndarray, Ecol: np.ndarray, rank: int):
    """The rank-`rank` bbFMM operators inside the rank-r arrays: U keeps its leading `rank`
    singular vectors (the rest zero) and E_k = U^T K_k U keeps its leading rank x rank block,
    which is exactly U'^T K_k U' for the truncated basis U'. Zero padding keeps every array
    layout (and kernel) of rank r = n^3 / 2."""
    n3 = n ** 3
    r = n3 // 2
    U = np.array(Ucol, copy=True).reshape(r, n3)        # row j = column j of U
    U[rank:] = 0
    E = np.array(Ecol, copy=True).reshape(NUM_OFFSETS, r, r)  # [k][j][i]
    E[:, rank:, :] = 0
    E[:, :, rank:] = 0
    return U.reshape(-1), E.reshape(-1)


def load_operators(n: int, single: bool = False, cache_dir: str | None = None, kernel: str = "laplacian"):
    """Cached operators for order n and a kernel: returns (r, Ucol, Ecol) in the requested
    precision.

    The FP64 SVD is always the source; single-precision files hold its rounding
    (operators are FP64-derived in every mode)."""
    cache_dir = cache_dir or default_cache_dir()
    kname, uname = operator_file_names(n, single, kernel)
    if not (os.path.exists(os.path.join(cache_dir, kname))
            and os.path.exists(os.path.join(cache_dir, uname))):
        dk, du = operator_file_names(n, False, kernel)
        if os.path.exists(os.path.join(cache_dir, dk)) and os.path.exists(os.path.join(cache_dir, du)):
            _, Ucol, Ecol = read_operator_files(cache_dir, n, False, kernel)
        else:
            Ucol, Ecol, _ = kernel_svd(n, kernel=kernel)
            write_operator_files(cache_dir, n, Ucol, Ecol, False, kernel)
        if single:
            write_operator_files(cache_dir, n, Ucol, Ecol, True, kernel)
    return read_operator_files(cache_dir, n, single, kernel)
