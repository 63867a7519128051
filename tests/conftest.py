import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# Small device workspaces for the test workloads (read at sa_initialize_processor).
os.environ.setdefault("SA_SURV_CAP", str(1 << 22))
os.environ.setdefault("SA_LONG_CAP", str(1 << 20))
os.environ.setdefault("SA_BATCH_SLOT_CAP", str(1 << 24))
os.environ.setdefault("SA_BATCH_SURV_CAP", str(1 << 22))
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
