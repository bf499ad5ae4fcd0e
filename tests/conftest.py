import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built sm_100a library")


def have_gpu():
    try:
        import galfast_b200 as G
        c = G.Context(0)
        c.close()
        return True
    except Exception:
        return False


@pytest.fixture(scope="session")
def lib():
    import galfast_b200 as G
    return G.lib()


@pytest.fixture(scope="session")
def multipliers(lib):
    import ctypes as C
    import numpy as np
    m = np.zeros(65536, dtype=np.uint32)
    assert lib.gf_multipliers(m.ctypes.data_as(C.POINTER(C.c_uint32)), 65536) == 0
    return m


@pytest.fixture(scope="session")
def ctx():
    if not have_gpu():
        pytest.skip("no CUDA device")
    import galfast_b200 as G
    c = G.Context(0)
    yield c
    c.close()
