"""Host-side logic: depth formula, interaction counts, operator precompute properties."""
import numpy as np
import pytest

from bbfmm_b200 import operators as ops
from bbfmm_b200.fmm import reference_depth


def test_reference_depth_formula():
    # (int)log(N)/log(8) binds the cast to log(N) only (bbfmm.c:151-160)
    assert reference_depth(32768) == 3 and reference_depth(32768, 1) == 4
    assert reference_depth(4194304) == 6 and reference_depth(4194304, 1) == 7
    assert reference_depth(10) == 2 and reference_depth(1) == 2


def test_interaction_counts_full_tree():
    import bench
    tot = sum(bench.interactions_per_level(l) for l in range(2, 8))
    assert tot == 435_570_912
    assert sum(bench.interactions_per_level(l) for l in range(2, 5)) == 640_584


def test_ktable_and_offsets():
    t = ops.ktable()
    assert (t >= 0).sum() == 316 and t.max() == 315
    off = ops.offsets()
    for k, (vx, vy, vz) in enumerate(off):
        assert t[49 * (vx + 3) + 7 * (vy + 3) + (vz + 3)] == k


def test_operator_precompute_properties():
    U, E, s = ops.kernel_svd(4)
    n3, r = 64, 32
    Um = U.reshape(r, n3).T
    assert np.allclose(Um.T @ Um, np.eye(r), atol=1e-12)
    Ek = E.reshape(316, r, r).transpose(0, 2, 1)
    off = ops.offsets()
    idx = {tuple(v): k for k, v in enumerate(off)}
    for k, v in enumerate(off):  # symmetric kernel: E_{-v} = E_v^T
        assert np.allclose(Ek[idx[tuple(-v)]], Ek[k].T, rtol=1e-10, atol=1e-12 * np.abs(Ek[k]).max())
    assert np.all(np.diff(s) <= 1e-12 * s[0])


def test_operator_files_roundtrip(tmp_path):
    U, E, _ = ops.kernel_svd(4)
    ops.write_operator_files(str(tmp_path), 4, U, E, False)
    r, U2, E2 = ops.read_operator_files(str(tmp_path), 4, False)
    assert r == 32 and np.array_equal(U, U2) and np.array_equal(E, E2)
