"""ctypes binding of the bbfmm_b200 C-ABI (include/bbfmm_b200.h).

The compiled library must exist in-tree (bbfmm_b200/lib/libbbfmm_b200.so, built by
``python -m bbfmm_b200.build``); there is no fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libbbfmm_b200.so")

MODE_D, MODE_S, MODE_MIXED = 0, 1, 2
MODES = {"d": MODE_D, "s": MODE_S, "mixed": MODE_MIXED}
STAGES = ["gather", "p2m", "m2m", "proj_up", "m2l", "proj_down", "l2l", "l2p", "p2p", "scatter"]

ERRORS = {1: "argument", 2: "cuda", 3: "out of memory", 4: "unsupported", 5: "state"}


class BBFMMError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bbfmm_b200 error {code} ({ERRORS.get(code, '?')}): {msg}")
        self.code = code


class Config(C.Structure):
    _fields_ = [("n", C.c_int), ("maxlev", C.c_int), ("L", C.c_double), ("mode", C.c_int),
                ("lead", C.c_int), ("lead_rows", C.c_int), ("device", C.c_int), ("stream", C.c_void_p)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: build it with `python -m bbfmm_b200.build`")
        L = C.CDLL(LIB_PATH)
        vp, ip, i, d = C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_double
        L.bbfmm_b200_last_error.restype = C.c_char_p
        L.bbfmm_b200_create.argtypes = [C.POINTER(Config), vp, vp, i, C.POINTER(vp)]
        L.bbfmm_b200_set_particles.argtypes = [vp, i, vp]
        L.bbfmm_b200_set_particles_device.argtypes = [vp, i, vp]
        L.bbfmm_b200_set_kernel.argtypes = [vp, i]
        L.bbfmm_b200_solve.argtypes = [vp, vp, vp]
        L.bbfmm_b200_solve_host.argtypes = [vp, vp, vp]
        L.bbfmm_b200_solve_fields.argtypes = [vp, vp, vp, vp]
        L.bbfmm_b200_solve_fields2.argtypes = [vp, vp, vp, vp, vp, vp, vp]
        L.bbfmm_b200_set_timing.argtypes = [vp, i]
        L.bbfmm_b200_stage_times.argtypes = [vp, C.POINTER(C.c_float), i]
        L.bbfmm_b200_copy_multipoles.argtypes = [vp, i, vp]
        L.bbfmm_b200_copy_m2l.argtypes = [vp, i, vp]
        L.bbfmm_b200_set_target_region.argtypes = [vp, i, vp]
        L.bbfmm_b200_set_first_m2l_level.argtypes = [vp, i]
        L.bbfmm_b200_time_m2l.argtypes = [vp, i, i, C.POINTER(C.c_float)]
        L.bbfmm_b200_direct.argtypes = [i, vp, vp, i, vp, vp, vp]
        L.bbfmm_b200_direct_field.argtypes = [i, vp, vp, i, vp, vp, vp, vp]
        L.bbfmm_b200_autotune.argtypes = [vp, vp]
        L.bbfmm_b200_set_tc_products.argtypes = [vp, i]
        L.bbfmm_b200_set_rank.argtypes = [vp, i]
        L.bbfmm_b200_set_leaf_slab.argtypes = [vp, C.c_longlong]
        L.bbfmm_b200_tuning.argtypes = [vp, ip]
        L.bbfmm_b200_set_tuning.argtypes = [vp, ip]
        L.bbfmm_b200_batch_create.argtypes = [C.POINTER(Config), i, ip, ip, ip, vp, vp, vp, vp, vp, i, C.POINTER(vp)]
        L.bbfmm_b200_batch_create_device.argtypes = [C.POINTER(Config), i, ip, ip, ip, vp, vp, vp, vp, vp, i,
                                                     C.POINTER(vp)]
        L.bbfmm_b200_batch_solve.argtypes = [vp, vp, vp, i]
        L.bbfmm_b200_batch_autotune.argtypes = [vp, vp]
        L.bbfmm_b200_batch_set_target_regions.argtypes = [vp, i, vp, i]
        L.bbfmm_b200_batch_set_kernel.argtypes = [vp, i]
        L.bbfmm_b200_batch_groups.argtypes = [vp]
        L.bbfmm_b200_batch_graph_nodes.argtypes = [vp]
        L.bbfmm_b200_batch_graph_nodes.restype = C.c_longlong
        L.bbfmm_b200_batch_group_info.argtypes = [vp, i, ip]
        L.bbfmm_b200_batch_group_stage_times.argtypes = [vp, i, vp, vp, C.POINTER(C.c_float), i]
        L.bbfmm_b200_batch_stream.argtypes = [vp]
        L.bbfmm_b200_batch_stream.restype = vp
        L.bbfmm_b200_batch_destroy.argtypes = [vp]
        L.bbfmm_b200_batch_destroy.restype = None
        L.bbfmm_b200_device_status.argtypes = [i]
        L.bbfmm_b200_wait_selftest.argtypes = [C.c_uint]
        L.bbfmm_b200_near_field.argtypes = [i, i, d, vp, vp, vp, i, vp]
        L.bbfmm_b200_near_field_noalloc.argtypes = [i, i, d, vp, vp, vp, i, vp]
        L.bbfmm_b200_stream.argtypes = [vp]
        L.bbfmm_b200_stream.restype = vp
        L.bbfmm_b200_destroy.argtypes = [vp]
        L.bbfmm_b200_destroy.restype = None
        L.bbfmm_b200_weights.argtypes = [i, i, vp, ip, vp, vp]
        L.bbfmm_b200_sort_particles.argtypes = [i, i, vp, d, i, ip, ip]
        _lib = L
    return _lib


def check(rc: int):
    if rc != 0:
        raise BBFMMError(rc, lib().bbfmm_b200_last_error().decode(errors="replace"))
    return rc


def exported_symbols(macro: str = "BBFMM_B200_API") -> list[str]:
    """Function names declared in include/*.h with the given export macro
    (BBFMM_B200_API: libbbfmm_b200.so; BBFMM_B200_REF_API: the reference-name shims)."""
    import glob
    import re
    names = []
    for h in sorted(glob.glob(os.path.join(os.path.dirname(HERE), "include", "*.h"))):
        txt = open(h).read()
        names += re.findall(r"^" + macro + r"\s+[^;(]*?\b(\w+)\s*\(", txt, flags=re.M)
    return names
