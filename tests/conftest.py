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

# Instantiations of one solver form for another block shape, schedule or placement compile
# the same expressions; their results agree to 1e-13 relative (the oracle bar, 1e-10, is
# tested separately).
SAME_ARITH = 1e-13


def rel_err(a, b, floor=1.0):
    """|a-b| / max(|b|, floor): relative error with the solver's absolute tolerance
    (1 molec/cm^3) as the floor for species near zero."""
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


@pytest.fixture(scope="session")
def cells4k():
    from radm2b200 import inputs
    return inputs.make_cells(4096, 0, "plain", night_frac=0.0)
