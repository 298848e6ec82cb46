"""Failure detection on the GPU without a fault (-m gpu): a kernel waits on an mbarrier that
nothing arrives at, with the bounded wait of the tensor-core kernels; the wait must give up,
leave its code in the status word the host reads, and the context must stay usable (a
mixed-precision solve right after it, which runs the tensor-core kernels, still matches the
FP64 solve to the mixed-mode tolerance 3e-7)."""
import pytest

from conftest import uniform_inputs
from oracle.oracle import rel_l2

pytestmark = pytest.mark.gpu


def test_bounded_wait_gives_up_and_reports():
    import torch
    from bbfmm_b200 import Solver, _lib
    L = _lib.lib()
    assert L.bbfmm_b200_device_status(1) == 0
    assert L.bbfmm_b200_wait_selftest(4096) == 99      # BBFMM_B200_WAIT_SELFTEST_CODE
    assert L.bbfmm_b200_device_status(0) == 0          # read and cleared by the self test
    assert L.bbfmm_b200_wait_selftest(0) < 0           # bad limit: refused on the host
    x, q = uniform_inputs(8192, seed=31)
    out = {}
    for mode in ("mixed", "d"):
        s = Solver(8, 4, 1.0, mode=mode)
        s.set_particles(x)
        out[mode] = s.solve(torch.as_tensor(q, device="cuda")).cpu().numpy()
        s.close()
    assert rel_l2(out["mixed"], out["d"]) < 3e-7
    assert L.bbfmm_b200_device_status(1) == 0
