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


def rel_l2(a, b) -> float:
    """||a - b|| / ||b|| in FP64 (tools/comperr4.c:61-93 with SUM_IN_DOUBLE)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(((a - b) ** 2).sum() / (b ** 2).sum()))
