"""CPU oracle against the reference's golden fixtures (tests/golden, made by
tests/golden/make_golden.py from the reference's own code).

Bitwise: Chebyshev tables, the reference's particle generator, tree and lists.
Known answers: relL2 of the FMM against the direct sum with the reference's own U files
(operators E = U^T K U rebuilt here in FP64, so agreement is to ~1e-10 relative in d).
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

from oracle.oracle import rel_l2

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
G = json.load(open(os.path.join(GOLD, "golden.json")))


def _digest(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _hexarr(v, dt):
    return np.array([float.fromhex(x) for x in v]).astype(dt)


def ref_operators(n, prec, kernel="laplacian"):
    """U from the reference's own SVD file; E = U^T K_k U in FP64 (bbfmm.c:1384-1405)."""
    from bbfmm_b200 import operators as ops
    dt = np.float64 if prec == "d" else np.float32
    tag = "" if kernel == "laplacian" else f"_{kernel}"
    raw = open(os.path.join(GOLD, f"refU{n}_{prec}{tag}.bin"), "rb").read()
    r = struct.unpack("i", raw[:4])[0]
    Ucol = np.frombuffer(raw[4:], dtype=dt).astype(np.float64)
    n3 = n ** 3
    U = Ucol.reshape(r, n3).T
    K0 = ops.kernel_matrix(n, kernel)
    E = np.stack([U.T @ K0[:, k * n3:(k + 1) * n3] @ U for k in range(316)])
    Ecol = np.ascontiguousarray(E.transpose(0, 2, 1)).reshape(-1)
    return Ucol.astype(dt), Ecol.astype(dt)


@pytest.mark.parametrize("prec", ["d", "s"])
@pytest.mark.parametrize("n", [4, 8])
def test_weights_bitwise(prec, n, oracle_d, oracle_s):
    o = oracle_d if prec == "d" else oracle_s
    Tkz, Kt, Kw, Cw = o.weights(n)
    g = G[f"weights_{prec}_n{n}"]
    assert np.array_equal(Tkz, _hexarr(g["Tkz"], o.dt))
    assert np.array_equal(Kt, np.array(g["Ktable"]))
    assert np.array_equal(Kw, _hexarr(g["Kweights"], o.dt))
    assert np.array_equal(Cw, _hexarr(g["Cweights"], o.dt))


@pytest.mark.parametrize("prec", ["d", "s"])
def test_reference_generator_and_tree_bitwise(prec, oracle_d, oracle_s):
    o = oracle_d if prec == "d" else oracle_s
    xyz, q = o.ref_sources(32768)
    g = G[f"sources_{prec}_N32768"]
    assert _digest(xyz) == g["xyz"] and _digest(q) == g["q"]
    for lev in (3, 4):
        t = o.build_tree(xyz, lev)
        want = G[f"tree_{prec}_N32768_l{lev}"]
        for k, v in want.items():
            assert _digest(getattr(t, k)) == v, (lev, k)


def test_direct_fp64_matches_reference_direct(oracle_d):
    xyz, q = oracle_d.ref_sources(32768)
    got = oracle_d.direct_fp64(xyz, q, np.arange(64))
    want = _hexarr(G["direct_d_N32768_first64"], np.float64)
    assert rel_l2(got, want) < 1e-13


@pytest.mark.parametrize("n,lev,prec,rtol", [(4, 3, "d", 1e-9), (4, 4, "d", 1e-9), (4, 3, "s", 2e-3),
                                            (8, 3, "d", 1e-7)])
def test_known_answers(n, lev, prec, rtol, oracle_d, oracle_s):
    o = oracle_d if prec == "d" else oracle_s
    U, E = ref_operators(n, prec)
    xyz, q = o.ref_sources(32768)
    phi = o.fmm(xyz, q, n, lev, U, E)
    dref = oracle_d.direct_fp64(xyz.astype(np.float64), q.astype(np.float64), np.arange(32768))
    err = rel_l2(phi, dref)
    want = G[f"kat_{prec}_n{n}_l{lev}"]
    assert abs(err - want) <= rtol * want, (err, want)
    if (n, lev, prec) == (4, 3, "d"):
        first = _hexarr(G["fmm_d_n4_l3_first32"], np.float64)
        assert rel_l2(phi[:32], first) < 1e-10


@pytest.mark.parametrize("kernel", ["oneoverr4", "laplacianforce"])
def test_known_answers_other_kernels(kernel, oracle_d):
    """The reference's -DONEOVERR4 and -DLAPLACIANFORCE builds on their own particles (N =
    32768, n = 4, depth 3, their own U files): the oracle's direct sum and FMM reproduce the
    reference's direct values, FMM values and FMM-vs-direct error. Measured: FMM values equal
    to 1e-16, direct values to 1e-15, the error to 2e-9 relative (1/r^4, whose error of 2e-9
    is itself near rounding: the near field dominates the norm) and 1e-14 (x/r^3)."""
    from bbfmm_b200 import operators as ops
    U, E = ref_operators(4, "d", kernel)
    h = ops.homogeneity(kernel)
    xyz, q = oracle_d.ref_sources(32768)
    phi = oracle_d.fmm(xyz, q, 4, 3, U, E, homogen=h)
    assert rel_l2(phi[:32], _hexarr(G[f"fmm_d_n4_l3_{kernel}_first32"], np.float64)) < 1e-13
    dref = oracle_d.direct_fp64(xyz, q, np.arange(32768), homogen=h)
    assert rel_l2(dref[:64], _hexarr(G[f"direct_d_N32768_{kernel}_first64"], np.float64)) < 1e-13
    want = G[f"kat_d_n4_l3_{kernel}"]
    assert abs(rel_l2(phi, dref) - want) <= 1e-7 * want


@pytest.mark.parametrize("n,lev", [(4, 3), (4, 4), (8, 3)])
def test_staged_oracle_and_sampled_m2l(oracle_d, n, lev):
    """The oracle's threaded, operator-sorted M2L (fmm_staged) agrees with orc_fmm to rounding,
    and the M2L of sampled cells with interaction lists enumerated from the grid
    (m2l_sample, used at depths whose explicit lists are too large) agrees with the M2L over
    the tree's explicit lists, which equal the reference's bitwise."""
    from bbfmm_b200 import operators as ops
    from oracle.oracle import levsta, rel_l2
    _, U, E = ops.load_operators(n, single=False)
    rng = np.random.default_rng(n + lev)
    N = 8000 * lev
    x = rng.random((N, 3)) - 0.5
    q = rng.uniform(-1, 1, N)
    assert rel_l2(oracle_d.fmm_staged(x, q, n, lev, U, E), oracle_d.fmm(x, q, n, lev, U, E)) < 1e-14
    r = n ** 3 // 2
    tree = oracle_d.build_tree(x, lev)
    _, P = oracle_d.upward(tree, x, q, n, U)
    PF = oracle_d.m2l(tree, r, E, P)
    lo = levsta(lev)
    cells = rng.choice(8 ** lev, 40, replace=False)
    got = oracle_d.m2l_sample(lev, r, E, P[lo * r:(lo + 8 ** lev) * r], cells)
    assert rel_l2(got, PF[lo * r:(lo + 8 ** lev) * r].reshape(-1, r)[cells]) < 1e-14
