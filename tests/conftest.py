import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: larger CPU cases")


@pytest.fixture(scope="session")
def ref():
    """The reference's own CPU path (oracle/_ref/libv2m_ref.so)."""
    from oracle.ref import RefLib, available
    if not available():
        pytest.skip("oracle/_ref/libv2m_ref.so not built")
    return RefLib()


@pytest.fixture(scope="session")
def cuda_lib():
    """libv2m_cuda.so with a usable device; GPU tests fail (not skip) without one."""
    from trussnet_b200 import _lib
    L = _lib.load()
    assert L.v2m_cuda_device_count() > 0, "no CUDA device visible to libv2m_cuda.so"
    return L
