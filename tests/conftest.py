import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the engine on the GPU)")


@pytest.fixture(scope="session")
def ref_b2e():
    from reforacle import RefOracle
    return RefOracle("b2e")


@pytest.fixture(scope="session")
def ref_libm():
    from reforacle import RefOracle
    return RefOracle("libm")
