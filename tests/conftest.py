"""pytest configuration: the ``gpu`` marker and shared fixtures."""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
HERE = os.path.dirname(os.path.abspath(__file__))
if HERE not in sys.path:
    sys.path.insert(0, HERE)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the product's GPU path")


@pytest.fixture(scope="session")
def built_library():
    """Builds the product libraries (and the oracle) once per session."""
    from libssa_b200 import build
    build.build()
    import oracle
    if not os.path.exists(oracle.LIB_PATH):
        oracle.build()
    import libssa_b200
    return libssa_b200.load()
