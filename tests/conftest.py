import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (runs the CUDA solver)")


@pytest.fixture(scope="session")
def native():
    """The native library, built if needed; GPU tests fail loudly without it."""
    from briscola_b200 import _native
    from briscola_b200.build import build_native

    build_native()
    return _native.load()
