import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu():
    """The CUDA library on a visible device; GPU tests fail loudly if the library is missing."""
    from maille_b200 import build, _lib
    build.build()
    lib = _lib.load()
    if lib.maille_gpu_device_count() == 0:
        pytest.skip("no CUDA device visible")
    return lib
