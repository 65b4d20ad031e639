import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 (B200) GPU; parity tests through the C ABI")


def golden(name):
    return dict(np.load(os.path.join(GOLDEN, name), allow_pickle=False))


@pytest.fixture(scope="session")
def hlib():
    """The built libha_b200.so (built here with nvcc if it is missing or stale)."""
    from hyperalignment_b200 import build as B
    from hyperalignment_b200 import _lib as L
    if B.needs_build():
        B.build()
    return L.lib()


@pytest.fixture(scope="session")
def gpu(hlib):
    """Initialised B200 backend; a GPU test FAILS (never skips) when the device or kernels are unusable."""
    rc = hlib.ha_b200_init()
    assert rc == 0, "ha_b200_init failed: no sm_100 GPU or the CUDA library did not load"
    return hlib
