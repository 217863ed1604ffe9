import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA library")
    config.addinivalue_line("markers", "slow: larger scenes")


@pytest.fixture(scope="session")
def oracle():
    from oracle import zoracle
    return zoracle.lib()


@pytest.fixture(scope="session")
def golden():
    import numpy as np
    return np.load(os.path.join(ROOT, "tests", "golden", "spgrid_golden.npz"))


@pytest.fixture(scope="session")
def cuda_lib():
    """The CUDA library; fails (never skips) when it is missing or no GPU is visible."""
    from ziran2019_b200 import abi, build
    build.build()
    lib = abi.product_lib()
    import ctypes
    cudart = None
    for name in ("libcudart.so", "libcudart.so.12"):
        try:
            cudart = ctypes.CDLL(name)
            break
        except OSError:
            continue
    if cudart is not None:
        n = ctypes.c_int(0)
        assert cudart.cudaGetDeviceCount(ctypes.byref(n)) == 0 and n.value > 0, "no CUDA device visible"
    return lib
