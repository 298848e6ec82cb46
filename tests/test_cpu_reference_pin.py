"""CPU oracle against the reference implementation itself (oracle/_ref, built from the
reference's own sources by oracle/build_ref.sh). Skipped where that build is absent.

Bitwise: tree, lists and the upward-pass multipoles. Final potentials: relative L2
< 1e-14 (d) / 1e-6 (s) against the default CPU path (sibling-blocking M2L) and against
the ij-blocking CPU M2L (CPU9A); the residual is M2L summation order.
"""
import os
import tempfile

import numpy as np
import pytest

from oracle.oracle import Reference, reference_available, rel_l2

pytestmark = pytest.mark.skipif(not reference_available("d"), reason="oracle/_ref not built")


@pytest.fixture(scope="module")
def opdir():
    d = tempfile.mkdtemp()
    for prec in ("d", "s"):
        Reference(prec).compute_operators(4, d)
    return d


@pytest.mark.parametrize("prec,variant,tol", [("d", "cpu8a", 1e-14), ("d", "cpu9a", 1e-14),
                                              ("s", "cpu8a", 1e-6), ("s", "cpu9a", 1e-6)])
def test_oracle_equals_reference(prec, variant, tol, opdir, oracle_d, oracle_s):
    if not reference_available(prec, variant):
        pytest.skip("variant not built")
    R = Reference(prec, variant)
    O = oracle_d if prec == "d" else oracle_s
    kp = os.path.join(opdir, ("laplacianK4.bin" if prec == "d" else "slaplacianK4.bin"))
    up = kp.replace("K4", "U4")
    U = np.fromfile(up, dtype=O.dt, offset=4)
    E = np.fromfile(kp, dtype=O.dt)
    rng = np.random.default_rng(4)
    x = (rng.random((20000, 3)) - 0.5).astype(O.dt)
    q = rng.uniform(-1, 1, 20000).astype(O.dt)
    lev = 3
    tr, to = R.build_tree(x, 4, lev), O.build_tree(x, lev)
    for k in ("center", "fieldlist", "sta", "end", "ineigh", "neighbors", "iinter", "interaction"):
        assert np.array_equal(getattr(tr, k), getattr(to, k)), k
    phir, Pr, _ = R.fmm(x, q, 4, lev, kp, up, want_intermediates=True)
    _, Po = O.upward(to, x, q, 4, U)
    lo = 9 * 32  # levels >= 2
    assert np.array_equal(Pr[lo:], Po[lo:])
    phio = O.fmm(x, q, 4, lev, U, E)
    assert rel_l2(phio, phir) < tol
