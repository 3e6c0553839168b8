import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (runs the CUDA library)")


@pytest.fixture(scope="session")
def lib():
    """The in-tree CUDA library (built here if absent; nvcc cross-compiles without a GPU)."""
    from tarang_b200 import build as b
    b.build(verbose=False)
    from tarang_b200 import _lib
    return _lib.load()
