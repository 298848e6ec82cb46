"""ctypes access to the CPU ORACLE (bbfmm_oracle.c) and to the reference harness.

TEST INFRASTRUCTURE ONLY. Tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module as the checker; the product package never imports it.

* ``Oracle(prec)``      -- our CPU restatement, ``prec`` in {"d", "s"}.
* ``Reference(prec, variant)`` -- the reference's own CPU code built from its sources by
  ``oracle/build_ref.sh`` into ``oracle/_ref/`` (variant "cpu8a" = default sibling-blocking
  M2L, "cpu9a" = ij-blocking CPU M2L, "cpu8a_ascii" = its operator files as text, "dropin" =
  the same code with its pass objects taken from the B200 library; ``kernel`` "oneoverr4" / "laplacianforce" for the -DONEOVERR4 /
  -DLAPLACIANFORCE builds). Present only where that build ran.
"""
from __future__ import annotations

import ctypes as C
import os
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PITCH_NEIGHBORS = 64
PITCH_INTERACTION = 192


def ncell(maxlev: int) -> int:
    return (8 ** (maxlev + 1) - 1) // 7


def levsta(level: int) -> int:
    return (8 ** level - 1) // 7


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Tree:
    """Flat arrays of the full uniform octree (same meaning as the reference's)."""

    def __init__(self, N, maxlev, dt):
        nc = ncell(maxlev)
        self.maxlev = maxlev
        self.center = np.zeros(3 * nc, dtype=dt)
        self.fieldlist = np.zeros(max(N, 1), dtype=np.int32)
        self.sta = np.zeros(nc, dtype=np.int32)
        self.end = np.zeros(nc, dtype=np.int32)
        self.ineigh = np.zeros(nc, dtype=np.int32)
        self.neighbors = np.zeros(nc * PITCH_NEIGHBORS, dtype=np.int32)
        self.iinter = np.zeros(nc, dtype=np.int32)
        self.interaction = np.zeros(nc * PITCH_INTERACTION, dtype=np.int32)

    def args(self):
        return [_p(self.center), _p(self.fieldlist), _p(self.sta), _p(self.end), _p(self.ineigh),
                _p(self.neighbors), _p(self.iinter), _p(self.interaction)]


class Oracle:
    def __init__(self, prec: str = "d"):
        assert prec in ("d", "s")
        self.prec = prec
        self.dt = np.float64 if prec == "d" else np.float32
        path = os.path.join(HERE, "_build", f"liboracle_{prec}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_oracle.sh")
        self.lib = C.CDLL(path)
        self.R = C.c_double if prec == "d" else C.c_float
        self.sfx = "_" + prec

    def _f(self, name):
        return getattr(self.lib, name + self.sfx)

    def _arr(self, a):
        return np.ascontiguousarray(a, dtype=self.dt)

    def weights(self, n):
        Tkz = np.zeros(n * n, self.dt)
        Kt = np.zeros(343, np.int32)
        Kw = np.zeros(n ** 3, self.dt)
        Cw = np.zeros(2 * n * n, self.dt)
        self._f("orc_weights")(n, _p(Tkz), _p(Kt), _p(Kw), _p(Cw))
        return Tkz, Kt, Kw, Cw

    def build_tree(self, xyz, maxlev, L=1.0):
        xyz = self._arr(xyz).reshape(-1)
        N = xyz.size // 3
        t = Tree(N, maxlev, self.dt)
        self._f("orc_build_tree")(N, _p(xyz), self.R(L), maxlev, *t.args())
        return t

    def upward(self, tree, xyz, q, n, U, L=1.0):
        nc = ncell(tree.maxlev)
        r = U.size // n ** 3
        Tkz, _, Kw, Cw = self.weights(n)
        S = np.zeros(nc * n ** 3, self.dt)
        P = np.zeros(nc * r, self.dt)
        self._f("orc_upward")(tree.maxlev, n, r, _p(self._arr(xyz).reshape(-1)), _p(self._arr(q)),
                              _p(tree.center), _p(tree.fieldlist), _p(tree.sta), _p(tree.end),
                              _p(Tkz), _p(Kw), _p(Cw), _p(self._arr(U)), self.R(L), _p(S), _p(P))
        return S, P

    def m2l(self, tree, r, E, M, L=1.0):
        _, Kt, _, _ = self.weights(4)
        PF = np.zeros(ncell(tree.maxlev) * r, self.dt)
        self._f("orc_m2l")(tree.maxlev, r, _p(self._arr(E)), _p(self._arr(M)), _p(tree.center),
                           _p(tree.iinter), _p(tree.interaction), _p(Kt), self.R(L), _p(PF))
        return PF

    def m2l_pairs(self, r, E, M, cell, src, k, acc):
        """acc[cell[p]] += E_{k[p]} M[src[p]] for the pairs in order (orc_m2l_pairs)."""
        cell = np.ascontiguousarray(cell, np.int32)
        src = np.ascontiguousarray(src, np.int64)
        k = np.ascontiguousarray(k, np.int32)
        self._f("orc_m2l_pairs")(r, _p(E), _p(M), C.c_longlong(cell.size), _p(cell), _p(src), _p(k), _p(acc))

    def _pairs_threaded(self, r, E, M, cell, src, k, acc, threads):
        """Runs the pairs in `threads` chunks of whole target cells (disjoint rows of acc),
        each chunk sorted by operator so that every E_k block is read once per chunk. ctypes
        releases the GIL during the C call, so the chunks run in parallel."""
        from concurrent.futures import ThreadPoolExecutor
        E = self._arr(E)
        M = self._arr(M)
        order = np.argsort(cell, kind="stable")
        cell, src, k = cell[order], src[order], k[order]
        cuts = np.linspace(0, cell.size, threads + 1).astype(np.int64)
        # move each cut to a cell boundary so that no cell is split between chunks
        cuts = np.unique(np.searchsorted(cell, cell[np.minimum(cuts, cell.size - 1)], side="left").tolist()
                         + [0, cell.size])
        jobs = []
        for a, b in zip(cuts[:-1], cuts[1:]):
            o = np.argsort(k[a:b], kind="stable")
            jobs.append((cell[a:b][o], src[a:b][o], k[a:b][o]))
        with ThreadPoolExecutor(max_workers=threads) as ex:
            list(ex.map(lambda j: self.m2l_pairs(r, E, M, *j, acc), jobs))

    def m2l_parallel(self, tree, r, E, M, L=1.0, threads=None):
        """PF of orc_m2l (every level's M2L over the tree's interaction lists), computed with
        orc_m2l_pairs on all host cores: the same products, summed in operator order per cell
        instead of list order (agrees with orc_m2l to rounding)."""
        threads = threads or os.cpu_count() or 1
        _, Kt, _, _ = self.weights(4)
        PF = np.zeros(ncell(tree.maxlev) * r, self.dt)
        for level in range(2, tree.maxlev + 1):
            lo, hi = levsta(level), levsta(level + 1)
            cnt = tree.iinter[lo:hi].astype(np.int64)
            F = np.repeat(np.arange(lo, hi, dtype=np.int64), cnt)
            slot = np.arange(F.size) - np.repeat(np.cumsum(cnt) - cnt, cnt)
            S = tree.interaction[F * PITCH_INTERACTION + slot].astype(np.int64)
            cen = tree.center.reshape(-1, 3).astype(np.float64)
            Lc = L * 0.5 ** level
            v = np.rint((cen[S] - cen[F]) / Lc).astype(np.int64)
            k = Kt[49 * (v[:, 0] + 3) + 7 * (v[:, 1] + 3) + (v[:, 2] + 3)]
            self._pairs_threaded(r, E, M, F.astype(np.int32), S, k, PF, threads)
        return PF

    def fmm_staged(self, xyz, q, n, maxlev, U, E, L=1.0, threads=None):
        """The oracle FMM (orc_fmm's stages: tree, upward, M2L, post-M2L, downward, near field)
        with the M2L of m2l_parallel, for depths where the single-threaded M2L is too slow."""
        r = U.size // n ** 3
        tree = self.build_tree(xyz, maxlev, L)
        _, P = self.upward(tree, xyz, q, n, U, L)
        PF = self.m2l_parallel(tree, r, E, P, L, threads)
        F = self.postm2l(tree, n, U, PF, L)
        phi, _ = self.downward(tree, xyz, q, n, F, L)
        return self.nearfield(tree, xyz, q, phi)

    def m2l_sample(self, level, r, E, M_level, cells, threads=None):
        """M2L output rows of the given cells of `level` (Morton indices within the level) from
        that level's multipoles M_level (Morton order, r per cell): each cell's interaction list
        (the children of its parent's neighbours that are not its own neighbours, as
        anotherInteractionList.c:11-111 forms it) is enumerated from the grid, so no tree arrays
        are needed at any depth. Rows in the order of `cells`."""
        threads = threads or os.cpu_count() or 1
        _, Kt, _, _ = self.weights(4)
        cells = np.asarray(cells, np.int64)
        ix, iy, iz = morton_to_grid(cells, level)
        m = 2 ** level
        d = np.arange(-2, 4)
        dx, dy, dz = [a.reshape(-1) for a in np.meshgrid(d, d, d, indexing="ij")]
        # source grid coordinates: children of the parent's 3 x 3 x 3 neighbourhood
        jx = (ix[:, None] // 2) * 2 + dx[None, :]
        jy = (iy[:, None] // 2) * 2 + dy[None, :]
        jz = (iz[:, None] // 2) * 2 + dz[None, :]
        vx, vy, vz = jx - ix[:, None], jy - iy[:, None], jz - iz[:, None]
        ok = ((jx >= 0) & (jx < m) & (jy >= 0) & (jy < m) & (jz >= 0) & (jz < m)
              & (np.maximum(np.maximum(abs(vx), abs(vy)), abs(vz)) > 1))
        row = np.broadcast_to(np.arange(cells.size)[:, None], ok.shape)[ok]
        src = grid_to_morton(jx[ok], jy[ok], jz[ok], level)
        k = Kt[49 * (vx[ok] + 3) + 7 * (vy[ok] + 3) + (vz[ok] + 3)]
        acc = np.zeros(cells.size * r, self.dt)
        self._pairs_threaded(r, E, M_level, row.astype(np.int32), src, k, acc, threads)
        return acc.reshape(cells.size, r)

    def postm2l(self, tree, n, U, PF, L=1.0):
        r = U.size // n ** 3
        _, _, Kw, _ = self.weights(n)
        F = np.zeros(ncell(tree.maxlev) * n ** 3, self.dt)
        self._f("orc_postm2l")(tree.maxlev, n, r, _p(self._arr(U)), _p(Kw), _p(self._arr(PF)),
                               self.R(L), _p(F))
        return F

    def downward(self, tree, xyz, q, n, F, L=1.0):
        Tkz, _, _, Cw = self.weights(n)
        F = self._arr(F).copy()
        phi = np.zeros(np.asarray(q).size, self.dt)
        self._f("orc_downward")(tree.maxlev, n, _p(self._arr(xyz).reshape(-1)), _p(self._arr(q)),
                                _p(tree.center), _p(tree.fieldlist), _p(tree.sta), _p(tree.end),
                                _p(Tkz), _p(Cw), self.R(L), _p(F), _p(phi))
        return phi, F

    def nearfield(self, tree, xyz, q, phi):
        phi = self._arr(phi).copy()
        N = phi.size
        self._f("orc_nearfield")(tree.maxlev, N, _p(self._arr(xyz).reshape(-1)), _p(self._arr(q)),
                                 _p(tree.fieldlist), _p(tree.sta), _p(tree.end), _p(tree.ineigh),
                                 _p(tree.neighbors), _p(phi))
        return phi

    def fmm(self, xyz, q, n, maxlev, U, E, L=1.0, homogen=1):
        """homogen: the kernel's degree of homogeneity, 1 (1/r), 2 (x/r^3) or 4 (1/r^4); U, E
        must be that kernel's operators."""
        xyz = self._arr(xyz).reshape(-1)
        q = self._arr(q)
        N = q.size
        r = U.size // n ** 3
        phi = np.zeros(N, self.dt)
        self._f("orc_set_kernel")(int(homogen))
        try:
            self._f("orc_fmm")(N, _p(xyz), _p(q), self.R(L), n, r, maxlev, _p(self._arr(E)),
                               _p(self._arr(U)), _p(phi))
        finally:
            self._f("orc_set_kernel")(1)
        return phi

    def ref_sources(self, N, L=1.0):
        """The reference's own particle generator (glibc rand(), alternating charges)."""
        xyz = np.zeros(3 * N, self.dt)
        q = np.zeros(N, self.dt)
        self._f("orc_ref_sources")(N, self.R(L), _p(xyz), _p(q))
        return xyz.reshape(N, 3), q

    def direct_field_fp64(self, xyz, q, targets):
        """FP64 potential (no target factor) and its gradient at the targets."""
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(q, dtype=np.float64)
        targets = np.ascontiguousarray(targets, dtype=np.int32)
        pot = np.zeros(targets.size)
        fld = np.zeros(3 * targets.size)
        self._f("orc_direct_field_fp64")(q.size, _p(xyz), _p(q), targets.size, _p(targets), _p(pot), _p(fld))
        return pot, fld.reshape(-1, 3)

    def direct_fp64(self, xyz, q, targets, homogen=1):
        xyz = np.ascontiguousarray(xyz, dtype=np.float64).reshape(-1)
        q = np.ascontiguousarray(q, dtype=np.float64)
        targets = np.ascontiguousarray(targets, dtype=np.int32)
        out = np.zeros(targets.size)
        self._f("orc_set_kernel")(int(homogen))
        try:
            self._f("orc_direct_fp64")(q.size, _p(xyz), _p(q), targets.size, _p(targets), _p(out))
        finally:
            self._f("orc_set_kernel")(1)
        return out


# File tag of the reference's build for each kernel (oracle/build_ref.sh).
_KERNEL_TAG = {"laplacian": "", "oneoverr4": "_r4", "laplacianforce": "_force"}


def reference_available(prec="d", variant="cpu8a", kernel="laplacian") -> bool:
    return os.path.exists(os.path.join(HERE, "_ref", f"libref_{variant}_{prec}{_KERNEL_TAG[kernel]}.so"))


class Reference:
    """The reference's own CPU implementation (oracle/_ref, built by build_ref.sh); kernel
    "oneoverr4" is its -DONEOVERR4 build, "laplacianforce" its -DLAPLACIANFORCE build."""

    def __init__(self, prec="d", variant="cpu8a", kernel="laplacian"):
        self.prec = prec
        self.dt = np.float64 if prec == "d" else np.float32
        self.R = C.c_double if prec == "d" else C.c_float
        self.kernel, self.variant = kernel, variant
        path = os.path.join(HERE, "_ref", f"libref_{variant}_{prec}{_KERNEL_TAG[kernel]}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"{path} missing: run oracle/build_ref.sh")
        self.lib = C.CDLL(path)
        assert self.lib.ref_real_size() == np.dtype(self.dt).itemsize

    def _arr(self, a):
        return np.ascontiguousarray(a, dtype=self.dt)

    def compute_operators(self, n, dirpath):
        """The reference's own SVD (ComputeKernelSVD) into [s]<kernel>{K,U}{n}.bin (.out, as
        text, for the ENABLE_ASCII_IO build)."""
        pre = ("s" if self.prec == "s" else "") + self.kernel
        ext = "out" if self.variant.endswith("ascii") else "bin"
        kp = os.path.join(dirpath, f"{pre}K{n}.{ext}").encode()
        up = os.path.join(dirpath, f"{pre}U{n}.{ext}").encode()
        os.makedirs(dirpath, exist_ok=True)
        self.lib.ref_compute_operators(n, C.c_char_p(kp), C.c_char_p(up))
        return kp.decode(), up.decode()

    def weights(self, n):
        Tkz = np.zeros(n * n, self.dt)
        Kt = np.zeros(343, np.int32)
        Kw = np.zeros(n ** 3, self.dt)
        Cw = np.zeros(2 * n * n, self.dt)
        self.lib.ref_weights(n, _p(Tkz), _p(Kt), _p(Kw), _p(Cw))
        return Tkz, Kt, Kw, Cw

    def set_sources(self, N, L=1.0):
        xyz = np.zeros(3 * N, self.dt)
        q = np.zeros(N, self.dt)
        self.lib.ref_set_sources(N, self.R(L), _p(xyz), _p(q))
        return xyz.reshape(N, 3), q

    def build_tree(self, xyz, n, maxlev, L=1.0):
        xyz = self._arr(xyz).reshape(-1).copy()
        N = xyz.size // 3
        t = Tree(N, maxlev, self.dt)
        self.lib.ref_build_tree(N, _p(xyz), self.R(L), n, maxlev, *t.args())
        return t

    def fmm(self, xyz, q, n, maxlev, Kpath, Upath, L=1.0, want_intermediates=False):
        xyz = self._arr(xyz).reshape(-1).copy()
        q = self._arr(q).copy()
        N = q.size
        phi = np.zeros(N, self.dt)
        nc = ncell(maxlev)
        r = n ** 3 // 2
        P = np.zeros(nc * r, self.dt) if want_intermediates else None
        F = np.zeros(nc * n ** 3, self.dt) if want_intermediates else None
        rc = self.lib.ref_fmm(N, _p(xyz), _p(q), self.R(L), n, maxlev, C.c_char_p(Kpath.encode()),
                              C.c_char_p(Upath.encode()), _p(phi), _p(P), _p(F))
        if rc != 0:
            raise RuntimeError("reference fmm failed")
        return (phi, P, F) if want_intermediates else phi

    def direct(self, xyz, q, L=1.0):
        xyz = self._arr(xyz).reshape(-1).copy()
        q = self._arr(q).copy()
        phi = np.zeros(q.size, self.dt)
        self.lib.ref_direct(q.size, _p(xyz), _p(q), self.R(L), _p(phi))
        return phi


def morton_to_grid(m, level):
    """Grid coordinates of Morton cell indices (anotherFMMDistribute.c:239-253 bit order)."""
    m = np.asarray(m, np.int64)
    ix = np.zeros_like(m); iy = np.zeros_like(m); iz = np.zeros_like(m)
    for b in range(level):
        t = (m >> (3 * b)) & 7
        ix |= ((t >> 2) & 1) << b
        iy |= ((t >> 1) & 1) << b
        iz |= (t & 1) << b
    return ix, iy, iz


def grid_to_morton(ix, iy, iz, level):
    ix, iy, iz = (np.asarray(a, np.int64) for a in (ix, iy, iz))
    m = np.zeros_like(ix)
    for b in range(level):
        m |= (((ix >> b) & 1) << (3 * b + 2)) | (((iy >> b) & 1) << (3 * b + 1)) | (((iz >> b) & 1) << (3 * b))
    return m


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| in FP64 (tools/comperr4.c:61-93 with SUM_IN_DOUBLE)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
