"""Build recipe for the CUDA library (sm_100a) -- in-tree, no JIT cache.

Produces bbfmm_b200/lib/libbbfmm_b200.so: the kernels, the solver, the handle C-ABI
(include/bbfmm_b200.h) and the reference-compatible entry points in both precisions.
Invoked by ``__graft_entry__.build()`` and ``python -m bbfmm_b200.build``.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "_build")
LIBNAME = "libbbfmm_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ["-O3", "-std=c++17", "-lineinfo", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC,-fvisibility=hidden",
           "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]

# (source, extra flags, object name)
UNITS = [
    ("host_setup.cpp", [], "host_setup"),
    ("passes.cu", [], "passes"),
    ("passes_dmma.cu", [], "passes_dmma"),
    ("p2p.cu", [], "p2p"),
    ("m2l_simt.cu", [], "m2l_simt"),
    ("m2l_tc.cu", [], "m2l_tc"),
    ("m2l_dmma.cu", [], "m2l_dmma"),
    ("proj_dmma.cu", [], "proj_dmma"),
    ("direct.cu", [], "direct"),
    ("solver.cu", [], "solver"),
    ("reference_abi.cu", [], "reference_abi"),
    ("batch.cu", [], "batch"),
    ("tree.cu", [], "tree"),
]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", "nvcc"):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return "nvcc"


def _compile(unit):
    src, extra, name = unit
    out = os.path.join(OBJDIR, name + ".o")
    srcp = os.path.join(CSRC, src)
    lang = ["-x", "cu"] if src.endswith(".cu") else []
    cmd = [nvcc(), *ARCH, *NVFLAGS, *extra, *lang, "-c", srcp, "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    return out, r.stderr


def build(verbose: bool = False) -> str:
    os.makedirs(LIBDIR, exist_ok=True)
    os.makedirs(OBJDIR, exist_ok=True)
    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(_compile, UNITS))
    objs = [o for o, _ in results]
    if verbose:
        for _, err in results:
            if err.strip():
                print(err)
    lib = os.path.join(LIBDIR, LIBNAME)
    tmp = lib + ".tmp"
    cmd = [nvcc(), *ARCH, "-shared", "-o", tmp, *objs, "-lcudart", "-lcuda"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, lib)
    build_shims()
    return lib


SHIMS = {"libbbfmm_b200_ref_d.so": [], "libbbfmm_b200_ref_s.so": ["-DBBFMM_B200_SINGLE"]}


def build_shims() -> None:
    """The reference's own entry-point names, one library per precision, forwarding to
    libbbfmm_b200.so (found next to them through the $ORIGIN run path)."""
    for name, defs in SHIMS.items():
        out = os.path.join(LIBDIR, name)
        cmd = ["gcc", "-std=gnu99", "-O2", "-fPIC", "-shared", *defs, "-I" + os.path.join(ROOT, "include"),
               os.path.join(CSRC, "reference_shim.c"), "-o", out + ".tmp", "-L" + LIBDIR, "-l:" + LIBNAME,
               "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"shim build failed:\n{' '.join(cmd)}\n{r.stdout}\n{r.stderr}")
        os.replace(out + ".tmp", out)


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
