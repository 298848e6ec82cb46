"""The reference's own entry points served by the B200 library (-m gpu).

1. Drop-in: the reference's own code (tree build, weights, operator files, pass order of
   its harness) built with its pass objects replaced by libbbfmm_b200_ref_{d,s}.so
   (oracle/build_ref.sh, "dropin") against the unmodified reference build ("cpu8a"):
   multipoles, field values after M2L + post-M2L, and the final potentials.
   Tolerances (relative L2): d 1e-12 (summation order); s 5e-5 (FP32).
2. The shim symbols called directly (m2l_drv, anotherNearField) against the oracle.
"""
import ctypes as C
import os
import tempfile

import numpy as np
import pytest

from conftest import uniform_inputs
from oracle.oracle import Reference, reference_available, rel_l2

pytestmark = pytest.mark.gpu
LIB = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "bbfmm_b200", "lib")


@pytest.fixture(scope="module")
def opdir():
    d = tempfile.mkdtemp()
    for prec in ("d", "s"):
        if reference_available(prec):
            Reference(prec).compute_operators(4, d)
    return d


@pytest.mark.skipif(not reference_available("d", "dropin"), reason="drop-in reference build absent")
@pytest.mark.parametrize("prec,lev,tol", [("d", 3, 1e-12), ("d", 4, 1e-12), ("s", 3, 5e-5)])
def test_reference_pipeline_with_b200_passes(prec, lev, tol, opdir):
    ref, drop = Reference(prec, "cpu8a"), Reference(prec, "dropin")
    kp = os.path.join(opdir, ("laplacianK4.bin" if prec == "d" else "slaplacianK4.bin"))
    up = kp.replace("K4", "U4")
    x, q = uniform_inputs(30000, seed=41, dtype="float64" if prec == "d" else "float32")
    pr, Pr, Fr = ref.fmm(x, q, 4, lev, kp, up, want_intermediates=True)
    pd, Pd, Fd = drop.fmm(x, q, 4, lev, kp, up, want_intermediates=True)
    lo32, lo64 = 9 * 32, 9 * 64          # entries of levels >= 2
    assert rel_l2(Pd[lo32:], Pr[lo32:]) < tol
    assert rel_l2(Fd[lo64:], Fr[lo64:]) < tol
    assert rel_l2(pd, pr) < tol


@pytest.mark.parametrize("kernel", ["oneoverr4", "laplacianforce"])
def test_reference_pipeline_with_b200_passes_other_kernels(kernel):
    """The same drop-in check for the reference's -DONEOVERR4 and -DLAPLACIANFORCE builds
    (homogen 4 and 2 through the shims: the near field q / r^4 or q dx / r^3 and the per-level
    scale (1/L_l)^homogen), on the operators that build computes itself: 1e-12."""
    if not reference_available("d", "dropin", kernel=kernel):
        pytest.skip(f"{kernel} drop-in reference build absent")
    ref = Reference("d", "cpu8a", kernel=kernel)
    drop = Reference("d", "dropin", kernel=kernel)
    d = tempfile.mkdtemp()
    kp, up = os.path.join(d, f"{kernel}K4.bin"), os.path.join(d, f"{kernel}U4.bin")
    ref.lib.ref_compute_operators(4, C.c_char_p(kp.encode()), C.c_char_p(up.encode()))
    x, q = uniform_inputs(30000, seed=43)
    pr, Pr, Fr = ref.fmm(x, q, 4, 3, kp, up, want_intermediates=True)
    pd, Pd, Fd = drop.fmm(x, q, 4, 3, kp, up, want_intermediates=True)
    lo32, lo64 = 9 * 32, 9 * 64
    assert rel_l2(Pd[lo32:], Pr[lo32:]) < 1e-12
    assert rel_l2(Fd[lo64:], Fr[lo64:]) < 1e-12
    assert rel_l2(pd, pr) < 1e-12


class Cell(C.Structure):
    _fields_ = [("neighbors", C.c_void_p), ("interaction", C.c_void_p), ("center", C.c_void_p),
                ("fieldsta", C.c_void_p), ("fieldend", C.c_void_p), ("sourcesta", C.c_void_p),
                ("sourceend", C.c_void_p), ("ineigh", C.c_void_p), ("iinter", C.c_void_p),
                ("pitch_neighbors", C.c_int), ("pitch_interaction", C.c_int)]


class Tree(C.Structure):
    _fields_ = [("ncell", C.c_int), ("minlev", C.c_int), ("maxlev", C.c_int), ("levsta", C.c_void_p),
                ("levend", C.c_void_p), ("celeng", C.c_void_p), ("c", C.POINTER(Cell)), ("fieldval", C.c_void_p),
                ("sourceval", C.c_void_p), ("proxysval", C.c_void_p), ("ncell0", C.c_int), ("Nf", C.c_int),
                ("Ns", C.c_int), ("fieldlist", C.c_void_p), ("sourcelist", C.c_void_p)]


def _tree(t, N, maxlev, keep):
    """A reference anotherTree over the oracle's tree arrays (arrays kept alive in keep)."""
    p = lambda a: C.c_void_p(a.ctypes.data)
    levsta = np.array([(8 ** l - 1) // 7 for l in range(maxlev + 1)], np.int32)
    levend = np.array([(8 ** (l + 1) - 1) // 7 - 1 for l in range(maxlev + 1)], np.int32)
    celeng = np.array([0.5 ** l for l in range(maxlev + 1)])
    keep += [levsta, levend, celeng]
    c = Cell(p(t.neighbors), p(t.interaction), p(t.center), p(t.sta), p(t.end), p(t.sta), p(t.end), p(t.ineigh),
             p(t.iinter), 64, 192)
    keep.append(c)
    return Tree(t.center.size // 3, 2, maxlev, p(levsta), p(levend), p(celeng), C.pointer(c), None, None, None, 0,
                N, N, p(t.fieldlist), p(t.fieldlist))


def test_m2l_drv_and_near_field_symbols(oracle_d):
    from bbfmm_b200 import operators as ops
    shim = C.CDLL(os.path.join(LIB, "libbbfmm_b200_ref_d.so"))
    lev, N = 4, 30000
    x, q = uniform_inputs(N, seed=42)
    t = oracle_d.build_tree(x, lev)
    _, U, E = ops.load_operators(4, single=False)
    _, P = oracle_d.upward(t, x, q, 4, U)
    want = oracle_d.m2l(t, 32, E, P)
    L = np.zeros_like(want)
    dp = C.POINTER(C.c_double)
    vp, i = C.c_void_p, C.c_int
    # r, L, K, M, minlev, maxlev, L0, center, ineigh, pitch_neighbors, neighbors, iinter,
    # pitch_interaction, interaction, scheme (m2l_drv.cu:14-19); the lists are implied, not read
    shim.m2l_drv.argtypes = [i, dp, dp, dp, i, i, C.c_double, vp, vp, i, vp, vp, i, vp, i]
    args = [32, L.ctypes.data_as(dp), E.ctypes.data_as(dp), P.ctypes.data_as(dp), 2, lev, 1.0,
            None, None, 0, None, None, 0, None]
    assert shim.m2l_drv(*args, 3) == 0
    lo = 9 * 32
    assert rel_l2(L[lo:], want[lo:]) < 1e-12
    assert C.c_double.in_dll(shim, "kernel_exec_time").value > 0
    assert shim.m2l_drv(*args, 4) == 1                        # unknown scheme -> M2L_EXIT_FAIL
    keep = []
    tree = _tree(t, N, lev, keep)
    ptree = C.pointer(tree)
    phi0 = np.random.default_rng(0).standard_normal(N)
    phi = phi0.copy()
    xs = np.ascontiguousarray(x)
    shim.anotherNearField.argtypes = [C.c_void_p, C.c_int, C.c_double, C.c_void_p, C.c_void_p, dp, dp]
    shim.anotherNearField(C.byref(ptree), 1, 1.0, C.c_void_p(xs.ctypes.data), C.c_void_p(xs.ctypes.data),
                          phi.ctypes.data_as(dp), q.ctypes.data_as(dp))
    want_nf = oracle_d.nearfield(t, x, q, phi0)
    assert rel_l2(phi, want_nf) < 1e-13
