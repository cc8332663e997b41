import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 device (runs the sm_100a kernels)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o

    o.lib()
    return o


@pytest.fixture(scope="session")
def p2g():
    import par2rust_b200

    par2rust_b200._ffi.lib()
    return par2rust_b200


@pytest.fixture(scope="session")
def gpu(p2g):
    """A usable B200: fails (does not skip) when CUDA is unavailable."""
    info = p2g.device_info()
    return info
