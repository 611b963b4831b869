import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O
    O.build()
    return O


@pytest.fixture(scope="session")
def m3d_lib():
    """The package with its library loaded but no device initialised (host-side entries)."""
    import dispatch_b200 as m
    m.lib()
    return m


@pytest.fixture(scope="session")
def m3d():
    import dispatch_b200 as m
    m.init(0)
    return m
