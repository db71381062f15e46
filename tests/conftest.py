import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product kernels")


@pytest.fixture(scope="session")
def cuda_device():
    """Index of the CUDA device the GPU tests use; skips when none is visible."""
    from wacommplusplus_b200 import _native
    if _native.device_count() == 0:
        pytest.skip("no CUDA device visible")
    return 0
