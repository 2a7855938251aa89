import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs on a B200)")


@pytest.fixture(scope="session")
def oracle_built():
    from oracle import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, loaded; a GPU test fails (not skips) if it is missing."""
    from nexus_b200 import build, mpm
    build.build()
    return mpm.load()
