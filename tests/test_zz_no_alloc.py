"""The allocation-free near-field entry point (-m gpu).

bbfmm_b200_near_field_noalloc exists for callers that must not call cudaMalloc -- code
whose device memory belongs to another framework's allocator, or time-critical loops that
cannot take the device-wide synchronisation of cudaMalloc/cudaFree. It keeps its scratch in
a fixed array inside the library instead. This test calls it through the C-ABI twice in a
row, on different inputs, and checks each result against the allocating entry point
bbfmm_b200_near_field (relative L2 < 1e-12; both run the same kernels), in both precision
modes; and that sizes beyond the array's capacity are refused.

The file name sorts last so that a run stopping at the first failure has already run every
other test; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MAXLEV = 5
L = 1.0


def _sorted_inputs(N, seed):
    """Leaf-sorted (x, y, z, q) rows and leaf offsets, from the library's own host sort."""
    from bbfmm_b200 import _lib
    rng = np.random.default_rng(seed)
    x = np.ascontiguousarray(rng.random((N, 3)) - 0.5)
    q = rng.uniform(-1.0, 1.0, N)
    perm = np.zeros(N, dtype=np.int32)
    leaf_start = np.zeros(8 ** MAXLEV + 1, dtype=np.int32)
    _lib.check(_lib.lib().bbfmm_b200_sort_particles(
        N, 0, C.c_void_p(x.ctypes.data), L, MAXLEV,
        perm.ctypes.data_as(C.POINTER(C.c_int)), leaf_start.ctypes.data_as(C.POINTER(C.c_int))))
    xyzq = np.empty((N, 4))
    xyzq[:, :3] = x[perm]
    xyzq[:, 3] = q[perm]
    return xyzq, leaf_start


def _near(entry, xyzq, leaf_start, mode):
    import torch
    from bbfmm_b200 import _lib
    N = xyzq.shape[0]
    dx = torch.as_tensor(xyzq, device="cuda")
    dl = torch.as_tensor(leaf_start, device="cuda")
    phi = torch.zeros(N, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    rc = getattr(_lib.lib(), entry)(N, MAXLEV, L, C.c_void_p(dx.data_ptr()), C.c_void_p(dl.data_ptr()),
                                    C.c_void_p(phi.data_ptr()), mode, C.c_void_p(stream))
    _lib.check(rc)
    torch.cuda.synchronize()
    return phi.cpu().numpy()


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


@pytest.mark.parametrize("mode", [0, 2])  # BBFMM_B200_MODE_D, BBFMM_B200_MODE_MIXED
def test_noalloc_matches_allocating_entry_twice(mode):
    # the last call fills the static scratch to its stated capacity
    for call, (N, seed) in enumerate([(200_000, 1), (150_000, 2), (262_144, 3)]):
        xyzq, ls = _sorted_inputs(N, seed)
        want = _near("bbfmm_b200_near_field", xyzq, ls, mode)
        got = _near("bbfmm_b200_near_field_noalloc", xyzq, ls, mode)
        assert np.all(np.isfinite(got)), call
        assert _rel(got, want) < 1e-12, (call, _rel(got, want))


def test_noalloc_rejects_oversize():
    from bbfmm_b200 import _lib
    import torch
    N = 262_144 + 1
    buf = torch.zeros(4 * N, dtype=torch.float64, device="cuda")
    ls = torch.zeros(8 ** MAXLEV + 1, dtype=torch.int32, device="cuda")
    rc = _lib.lib().bbfmm_b200_near_field_noalloc(N, MAXLEV, L, C.c_void_p(buf.data_ptr()),
                                                  C.c_void_p(ls.data_ptr()), C.c_void_p(buf.data_ptr()), 0, None)
    assert rc == 1
    assert b"262144" in _lib.lib().bbfmm_b200_last_error()


@pytest.mark.parametrize("entry", ["bbfmm_b200_near_field", "bbfmm_b200_near_field_noalloc"])
@pytest.mark.parametrize("fault", ["past_n", "decreasing"])
def test_malformed_leaf_offsets_are_refused(entry, fault):
    """Leaf offsets that end past N or decrease are refused with BBFMM_B200_ERR_ARG and the
    leaf-range code in the status word. The arrays are sized for N + 16 particles, so even an
    access the clamps failed to stop would stay inside memory the test owns."""
    import torch
    from bbfmm_b200 import _lib
    N = 5000
    xyzq, ls = _sorted_inputs(N + 16, 4)
    ls = ls.copy()
    if fault == "past_n":
        pass                                   # offsets end at N + 16 but the call says N
    else:
        k = int(np.searchsorted(ls, N // 2))
        ls[k] = ls[k + 1] + 3                  # one offset above its successor
        ls[-1] = N
        ls = np.minimum(ls, N)
    dx = torch.as_tensor(xyzq, device="cuda")
    dl = torch.as_tensor(ls, device="cuda")
    phi = torch.zeros(N + 16, dtype=torch.float64, device="cuda")
    lib = _lib.lib()
    lib.bbfmm_b200_device_status(1)
    rc = getattr(lib, entry)(N, MAXLEV, L, C.c_void_p(dx.data_ptr()), C.c_void_p(dl.data_ptr()),
                             C.c_void_p(phi.data_ptr()), 0, None)
    torch.cuda.synchronize()
    assert rc == 1, rc
    assert b"leaf_start" in lib.bbfmm_b200_last_error()
    assert lib.bbfmm_b200_device_status(1) == 98       # BBFMM_B200_LEAF_RANGE_CODE
    assert float(phi[N:].abs().max()) == 0.0           # nothing written past N
    # the context stays usable: a well-formed call right after succeeds
    xyzq2, ls2 = _sorted_inputs(N, 5)
    got = _near(entry, xyzq2, ls2, 0)
    assert np.all(np.isfinite(got))
    assert lib.bbfmm_b200_device_status(1) == 0
