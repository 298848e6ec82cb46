"""The C-ABI library without a GPU: it loads, exports every symbol that include/*.h
declares, and its host-side entry points (Chebyshev tables, leaf sort, argument checks)
match the oracle bit for bit."""
import ctypes as C
import subprocess

import numpy as np
import pytest

from bbfmm_b200 import _lib


def test_library_exports_every_declared_symbol():
    names = _lib.exported_symbols()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    L = _lib.lib()
    for n in names:
        getattr(L, n)


def _c_kind(decl):
    """Kind of one C parameter or return type of include/bbfmm_b200.h."""
    import re
    d = decl.strip()
    if d in ("", "void"):
        return None
    if "*" in d:
        return "ptr"
    for pat, k in ((r"long long", "i64"), (r"\bdouble\b", "f64"), (r"\bfloat\b", "f32"), (r"\bunsigned\b", "u32"),
                   (r"\bint\b", "i32")):
        if re.search(pat, d):
            return k
    return "?" + d


def _py_kind(t):
    if t is None:
        return None
    if t in (C.c_void_p, C.c_char_p) or (isinstance(t, type) and issubclass(t, C._Pointer)):
        return "ptr"
    return {C.c_int: "i32", C.c_double: "f64", C.c_float: "f32", C.c_uint: "u32", C.c_longlong: "i64"}.get(t, "?")


def test_ctypes_declarations_match_the_header():
    """Every function of include/bbfmm_b200.h has ctypes argument and result types in _lib.py of
    the same kinds (int, unsigned, long long, float, double, pointer) in the same order."""
    import os
    import re
    src = open(os.path.join(os.path.dirname(_lib.HERE), "include", "bbfmm_b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    decls = re.findall(r"BBFMM_B200_API\s+([\w\s\*]+?)\s*\b(bbfmm_b200_\w+)\s*\(([^)]*)\)\s*;", src)
    assert len(decls) >= 40
    L = _lib.lib()
    for ret, name, params in decls:
        f = getattr(L, name)
        want = [k for k in (_c_kind(p) for p in params.split(",")) if k is not None]
        got = [_py_kind(t) for t in (f.argtypes or [])]
        assert got == want, (name, got, want)
        assert _py_kind(f.restype) == _c_kind(ret), (name, f.restype, ret)


@pytest.mark.parametrize("shim", ["libbbfmm_b200_ref_d.so", "libbbfmm_b200_ref_s.so"])
def test_reference_name_shims_export_the_reference_symbols(shim):
    import os
    names = _lib.exported_symbols("BBFMM_B200_REF_API")
    assert {"m2l_drv", "anotherFMMCompute", "anotherUpwardPass", "anotherFMMInteraction", "anotherDownwardPass",
            "anotherNearField", "m2l_host_basic", "m2l_host_ij_blocking"} <= set(names)
    path = os.path.join(os.path.dirname(_lib.LIB_PATH), shim)
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines()}
    assert not [n for n in names + ["kernel_exec_time"] if n not in exported]
    C.CDLL(path)  # loads, resolving libbbfmm_b200.so through its run path


@pytest.mark.parametrize("fp32", [0, 1])
@pytest.mark.parametrize("n", [4, 8])
def test_weights_equal_oracle(fp32, n, oracle_d, oracle_s):
    o = oracle_s if fp32 else oracle_d
    dt = o.dt
    Tkz, Kw, Cw = np.zeros(n * n, dt), np.zeros(n ** 3, dt), np.zeros(2 * n * n, dt)
    Kt = np.zeros(343, np.int32)
    _lib.check(_lib.lib().bbfmm_b200_weights(n, fp32, C.c_void_p(Tkz.ctypes.data),
                                             Kt.ctypes.data_as(C.POINTER(C.c_int)),
                                             C.c_void_p(Kw.ctypes.data), C.c_void_p(Cw.ctypes.data)))
    a = o.weights(n)
    for x, y in zip((Tkz, Kt, Kw, Cw), a):
        assert np.array_equal(x, y)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("lev", [2, 3, 4])
def test_leaf_sort_equals_reference_order(prec, lev, oracle_d, oracle_s):
    o = oracle_d if prec == "d" else oracle_s
    xyz, _ = o.ref_sources(32768)
    t = o.build_tree(xyz, lev)
    N = xyz.shape[0]
    perm = np.zeros(N, np.int32)
    ls = np.zeros(8 ** lev + 1, np.int32)
    xyz = np.ascontiguousarray(xyz)
    _lib.check(_lib.lib().bbfmm_b200_sort_particles(N, int(prec == "s"), C.c_void_p(xyz.ctypes.data), 1.0, lev,
                                                    perm.ctypes.data_as(C.POINTER(C.c_int)),
                                                    ls.ctypes.data_as(C.POINTER(C.c_int))))
    assert np.array_equal(perm, t.fieldlist)
    lo = (8 ** lev - 1) // 7
    assert np.array_equal(ls[:-1], t.sta[lo:lo + 8 ** lev])
    assert np.array_equal(ls[1:] - 1, t.end[lo:lo + 8 ** lev])


def test_sort_rejects_particles_outside_root_cell():
    xyz = np.array([[0.1, 0.2, 0.7]])
    perm = np.zeros(1, np.int32)
    ls = np.zeros(8 ** 2 + 1, np.int32)
    rc = _lib.lib().bbfmm_b200_sort_particles(1, 0, C.c_void_p(xyz.ctypes.data), 1.0, 2,
                                              perm.ctypes.data_as(C.POINTER(C.c_int)),
                                              ls.ctypes.data_as(C.POINTER(C.c_int)))
    assert rc == 1 and b"outside" in _lib.lib().bbfmm_b200_last_error()


def test_create_rejects_unsupported_order_before_touching_a_device():
    cfg = _lib.Config(n=5, maxlev=3, L=1.0, mode=0, lead=0, lead_rows=0, device=0, stream=None)
    U = np.zeros(10)
    h = C.c_void_p()
    rc = _lib.lib().bbfmm_b200_create(C.byref(cfg), C.c_void_p(U.ctypes.data), C.c_void_p(U.ctypes.data), 0,
                                      C.byref(h))
    assert rc == 4 and not h.value


def test_near_field_argument_checks():
    L = _lib.lib()
    assert L.bbfmm_b200_near_field(10, 1, 1.0, None, None, None, 0, None) == 1
    assert L.bbfmm_b200_near_field(10, 3, 1.0, None, None, None, 0, None) == 1
    assert L.bbfmm_b200_near_field_noalloc(262145, 3, 1.0, C.c_void_p(16), C.c_void_p(16), C.c_void_p(16), 0,
                                           None) == 1
    assert L.bbfmm_b200_near_field(0, 3, 1.0, None, None, None, 0, None) == 0


def test_handle_setters_reject_null_handles_and_bad_values():
    """Argument checks of the handle setters that run before any device work."""
    L = _lib.lib()  # argument types as declared by bbfmm_b200._lib
    for k in (0, 1, 2):  # LAPLACIAN, LAPLACIAN_FORCE, ONEOVERR4
        assert L.bbfmm_b200_set_kernel(None, k) == 1
        assert L.bbfmm_b200_batch_set_kernel(None, k) == 1
    assert L.bbfmm_b200_set_rank(None, 64) == 1
    assert L.bbfmm_b200_set_tc_products(None, 0) == 1
    assert L.bbfmm_b200_set_leaf_slab(None, 64) == 1
    assert L.bbfmm_b200_solve(None, None, None) == 1
    assert L.bbfmm_b200_set_particles(None, 10, None) == 1
    assert L.bbfmm_b200_set_particles_device(None, 10, None) == 1
    assert b"null" in L.bbfmm_b200_last_error() or b"bad" in L.bbfmm_b200_last_error()
