import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200); run with -m gpu")


@pytest.fixture(scope="session")
def g2lib():
    """The CUDA library, built in-tree if needed (nvcc cross-compiles without a GPU)."""
    from giem2g_b200 import build as b
    b.build()
    import giem2g_b200
    return giem2g_b200


@pytest.fixture(scope="session")
def orc():
    import oracle
    oracle.build()
    return oracle
