import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
os.environ.setdefault("BBFMM_B200_OPERATOR_DIR", os.path.join(ROOT, "tests", ".opcache"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200 / sm_100a)")
    config.addinivalue_line("markers", "slow: long CPU test")
    # build outputs are not versioned: build what a fresh checkout lacks
    import subprocess
    if not os.path.exists(os.path.join(ROOT, "oracle", "_build", "liboracle_d.so")):
        subprocess.run(["bash", os.path.join(ROOT, "oracle", "build_oracle.sh")], check=True)
    if not os.path.exists(os.path.join(ROOT, "bbfmm_b200", "lib", "libbbfmm_b200.so")):
        subprocess.run([sys.executable, "-m", "bbfmm_b200.build"], check=True, cwd=ROOT)


@pytest.fixture(scope="session")
def oracle_d():
    from oracle.oracle import Oracle
    return Oracle("d")


@pytest.fixture(scope="session")
def oracle_s():
    from oracle.oracle import Oracle
    return Oracle("s")


def uniform_inputs(N, seed=1, dtype="float64"):
    """Seeded uniform positions in [-0.5, 0.5)^3 and charges U[-1, 1] (the unit-cube
    configurations shifted to the reference's origin-centred root cell)."""
    import numpy as np
    rng = np.random.default_rng(seed)
    x = rng.random((N, 3)) - 0.5
    q = rng.uniform(-1.0, 1.0, N)
    return x.astype(dtype), q.astype(dtype)
