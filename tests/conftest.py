"""Test configuration: paths and the `gpu` marker.

`-m "not gpu"` runs the oracle against the golden vectors, the host logic and
the C-ABI load checks (no GPU needed); `-m gpu` runs the parity tests of the
CUDA path against the oracle and the golden vectors.
"""

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "prt-deeponet-gui_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libprtlb.so")


def load_golden(name):
    with np.load(os.path.join(GOLDEN, name + ".npz"), allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture
def golden():
    return load_golden


def gpu_available():
    try:
        import ctypes
        lib = ctypes.CDLL(os.path.join(PKG, "prtlb_gpu", "libprtlb.so"))
        n = ctypes.c_void_p()
        rc = lib.prt_create(0, ctypes.byref(n))
        if rc == 0:
            lib.prt_destroy(n)
            return True
    except OSError:
        pass
    return False
