import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU (B200); runs through the CUDA library")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the oracle (test infrastructure) and the CUDA library if they are missing."""
    from oracle import pyoracle
    if not os.path.exists(pyoracle._SO):
        pyoracle.build()
    so = os.path.join(ROOT, "ariel_b200", "_lib", "libariel_b200.so")
    if not os.path.exists(so):
        from ariel_b200 import build
        build.build()
    yield
