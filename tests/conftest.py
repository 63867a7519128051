import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def built():
    """Builds the native libraries in-tree (no-op when up to date)."""
    from segalign_b200 import _build
    import oracle

    _build.build()
    oracle.build()
    return True
