"""Generates the golden fixtures in tests/golden/ from the REFERENCE CPU code built from its
own sources by oracle/build_ref.sh (oracle/_ref). Run once where the reference is present:

    oracle/build_ref.sh && python tests/golden/make_golden.py            # everything
    oracle/build_ref.sh && python tests/golden/make_golden.py kernels    # add the kernel
                                                                         # fixtures only

Fixtures (all produced by the reference itself):
  refU4_d.bin, refU4_s.bin, refU8_d.bin  U files of the reference's own SVD
                                          (ComputeKernelSVD, bbfmm.c:1209-1421)
  golden.json  known answers:
    * Chebyshev tables of ComputeWeights (bbfmm.c:922-1028), n = 4 and 8, s and d (hex)
    * tree / list digests for the reference's own particles (SetSources, bbfmm.c:401-463)
    * relL2 of the reference FMM against the reference direct code (tools/comperr4.c
      arithmetic with FP64 sums), reference inputs, N = 32768, and the first 32 values
      of the reference FMM output for n = 4, depth 3, d
    * the reference direct code's output at 64 fixed targets (N = 32768, d)
  For the reference's -DONEOVERR4 and -DLAPLACIANFORCE builds (d, n = 4, N = 32768, depth 3):
  refU4_d_<kernel>.bin (its U file), and in golden.json kat_d_n4_l3_<kernel>,
  fmm_d_n4_l3_<kernel>_first32 and direct_d_N32768_<kernel>_first64.
"""
import hashlib
import json
import os
import shutil
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")

from oracle.oracle import Reference, rel_l2  # noqa: E402


def digest(a) -> str:
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def tree_digest(t) -> dict:
    return {k: digest(getattr(t, k)) for k in
            ("center", "fieldlist", "sta", "end", "ineigh", "neighbors", "iinter", "interaction")}


def main():
    out = {}
    tmp = tempfile.mkdtemp()
    try:
        for prec in ("d", "s"):
            R = Reference(prec)
            for n in ((4, 8) if prec == "d" else (4,)):
                kp, up = R.compute_operators(n, tmp)
                shutil.copy(up, os.path.join(HERE, f"refU{n}_{prec}.bin"))
            for n in (4, 8):
                Tkz, Kt, Kw, Cw = R.weights(n)
                out[f"weights_{prec}_n{n}"] = {
                    "Tkz": [float(v).hex() for v in np.asarray(Tkz, np.float64)],
                    "Ktable": [int(v) for v in Kt],
                    "Kweights": [float(v).hex() for v in np.asarray(Kw, np.float64)],
                    "Cweights": [float(v).hex() for v in np.asarray(Cw, np.float64)]}
            xyz, q = R.set_sources(32768)
            out[f"sources_{prec}_N32768"] = {"xyz": digest(xyz), "q": digest(q)}
            for lev in (3, 4):
                out[f"tree_{prec}_N32768_l{lev}"] = tree_digest(R.build_tree(xyz, 4, lev))
            pd = R.direct(xyz, q)
            if prec == "d":
                out["direct_d_N32768_first64"] = [float(v).hex() for v in pd[:64]]
            kp4 = os.path.join(tmp, ("laplacianK4.bin" if prec == "d" else "slaplacianK4.bin"))
            up4 = kp4.replace("K4", "U4")
            for n, lev in ([(4, 3), (4, 4), (8, 3)] if prec == "d" else [(4, 3)]):
                kp = kp4.replace("K4", f"K{n}")
                up = up4.replace("U4", f"U{n}")
                if n == 8 and not os.path.exists(kp):
                    R.compute_operators(8, tmp)
                phi = R.fmm(xyz, q, n, lev, kp, up)
                out[f"kat_{prec}_n{n}_l{lev}"] = rel_l2(phi, pd)
                if (prec, n, lev) == ("d", 4, 3):
                    out["fmm_d_n4_l3_first32"] = [float(v).hex() for v in phi[:32]]
                print(prec, n, lev, out[f"kat_{prec}_n{n}_l{lev}"], flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    kernel_fixtures(out)
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=1)


def kernel_fixtures(out):
    """Known answers of the reference's other kernels (1/r^4, x/r^3), FP64, n = 4, depth 3."""
    tmp = tempfile.mkdtemp()
    try:
        for kernel in ("oneoverr4", "laplacianforce"):
            R = Reference("d", kernel=kernel)
            kp, up = R.compute_operators(4, tmp)
            shutil.copy(up, os.path.join(HERE, f"refU4_d_{kernel}.bin"))
            xyz, q = R.set_sources(32768)
            pd = R.direct(xyz, q)
            phi = R.fmm(xyz, q, 4, 3, kp, up)
            out[f"kat_d_n4_l3_{kernel}"] = rel_l2(phi, pd)
            out[f"fmm_d_n4_l3_{kernel}_first32"] = [float(v).hex() for v in phi[:32]]
            out[f"direct_d_N32768_{kernel}_first64"] = [float(v).hex() for v in pd[:64]]
            print(kernel, out[f"kat_d_n4_l3_{kernel}"], flush=True)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def add_kernel_fixtures():
    path = os.path.join(HERE, "golden.json")
    out = json.load(open(path))
    kernel_fixtures(out)
    with open(path, "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    if sys.argv[1:] == ["kernels"]:
        add_kernel_fixtures()
    else:
        main()
