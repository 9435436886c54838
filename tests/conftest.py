import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def pond():
    """The CUDA library's Python front end (built in-tree)."""
    import lbmpond_b200
    from lbmpond_b200 import build as B
    if not os.path.exists(B.LIB):
        B.build()
    return lbmpond_b200
