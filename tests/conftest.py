import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the in-tree native libraries (no-op when up to date) and the oracle."""
    from poststackmig3d_b200 import build
    import oracle
    build.build()
    oracle.lib()
    yield
