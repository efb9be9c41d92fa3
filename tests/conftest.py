import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "radm2-solver-multi-gpu_b200")
for p in (PKG, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100) GPU and the built CUDA library")


ATOL = np.ones(59)
RTOL = np.full(59, 1.0e-3)

# Two instantiations of the fast solver (other block shape, schedule or placement) evaluate
# the same expressions, but the compiler may contract different multiply-add pairs in each,
# so their results agree to rounding level, not bit for bit: measured up to 4.8e-13 relative
# on the plain workloads.  The oracle bar (1e-10) is separate and tested on its own.
SAME_ARITH = 1e-12


def rel_err(a, b, floor=1.0):
    """|a-b| / max(|b|, floor): relative error with the solver's absolute tolerance
    (1 molec/cm^3) as the floor for species near zero."""
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


@pytest.fixture(scope="session")
def cells4k():
    from radm2b200 import inputs
    return inputs.make_cells(4096, 0, "plain", night_frac=0.0)
