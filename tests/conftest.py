import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and libct2g.so")


@pytest.fixture(scope="session")
def gpu():
    """The GPU tests run only where a CUDA device is present; the library must
    load (no fallback)."""
    from ct2_b200 import _lib
    lib = _lib.load()
    return lib
