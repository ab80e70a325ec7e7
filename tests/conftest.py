import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the libzkb200.so kernels")


@pytest.fixture(scope="session")
def zk():
    """The product package (zikkurat-algebra_b200) with libzkb200.so loaded."""
    import zkutil
    mod = zkutil.load_package()
    mod.lib()
    return mod
