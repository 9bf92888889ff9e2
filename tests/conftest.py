import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "softx-d-21-00014_b200")
for p in (os.path.join(ROOT, "tests"), PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.lib()
    return oracle_py


@pytest.fixture(scope="session")
def xamg():
    import xamg_b200
    xamg_b200.lib()
    return xamg_b200


@pytest.fixture(scope="session")
def gpu(xamg):
    """Initialise the library on the GPU once per session."""
    xamg.init()
    yield xamg
