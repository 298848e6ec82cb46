"""Mixed-precision solver (split-bf16 tcgen05 M2L + FP64 leading components + FP32
compensated P2P) against the FP64 oracle and the FP64 direct sum (-m gpu).

Bar: error against the FP64 direct sum at most 1.2x that of the FP64 FMM on the same
inputs. Tolerance to the FP64 oracle FMM: relative L2 < 3e-7 (n = 8; the split products
and FP32 accumulation leave a ~5e-8 to 1.3e-7 difference on these inputs, against an FMM
truncation error of ~1e-7 to 2e-7).
"""
import numpy as np
import pytest

from conftest import uniform_inputs
from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def _run(mode, n, maxlev, x, q, **kw):
    import torch
    from bbfmm_b200 import Solver
    s = Solver(n, maxlev, 1.0, mode=mode, **kw)
    s.set_particles(x)
    phi = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    return s, phi


def _status():
    from bbfmm_b200 import _lib
    return _lib.lib().bbfmm_b200_device_status(1)


def test_mixed_level4_matches_fp64(oracle_d):
    x, q = uniform_inputs(32768, seed=21)
    from bbfmm_b200 import operators as ops
    _, U, E = ops.load_operators(8, single=False)
    ref = oracle_d.fmm(x, q, 8, 4, U, E)
    s, got = _run("mixed", 8, 4, x, q)
    assert _status() == 0
    assert rel_l2(got, ref) < 3e-7
    s.close()


@pytest.mark.parametrize("lead,lead_rows", [(16, 32), (16, 256), (32, 64)])
def test_mixed_error_ratio_vs_direct(oracle_d, lead, lead_rows):
    x, q = uniform_inputs(32768, seed=22)
    t = np.random.default_rng(9).choice(32768, 2048, replace=False).astype(np.int32)
    dref = oracle_d.direct_fp64(x, q, t)
    s64, p64 = _run("d", 8, 4, x, q)
    sm, pm = _run("mixed", 8, 4, x, q, lead=lead, lead_rows=lead_rows)
    e64, em = rel_l2(p64[t], dref), rel_l2(pm[t], dref)
    assert _status() == 0
    assert em <= 1.2 * e64, (em, e64)
    s64.close(); sm.close()


def test_mixed_repeatable():
    x, q = uniform_inputs(40000, seed=23)
    s, a = _run("mixed", 8, 4, x, q)
    import torch
    b = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
    assert np.array_equal(a, b)
    s.close()
