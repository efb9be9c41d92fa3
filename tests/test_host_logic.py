"""Host-side logic on CPU: the seeded inputs are a pure function of (seed, cell), and the
oracle's IPAR/RPAR validation returns the reference's codes (mgpu.cu:3684-3811)."""
import numpy as np
import pytest

import oracle
import radm2b200
from radm2b200 import inputs


@pytest.mark.parametrize("workload", ["plain", "mixed"])
def test_any_subset_of_cells_is_reproducible(workload):
    full = inputs.make_cells(3000, 4, workload, 0.3)
    part = inputs.make_cells(700, 4, workload, 0.3, first_cell=1200)
    for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV", "cls"):
        assert np.array_equal(full[k][1200:1900], part[k]), k
    other = inputs.make_cells(700, 5, workload, 0.3, first_cell=1200)
    assert not np.array_equal(other["VAR"], part["VAR"])


def test_mixed_workload_classes_and_ranges():
    c = inputs.make_cells(20000, 3, "mixed")
    frac = np.bincount(c["cls"], minlength=4) / 20000.0
    assert abs(frac[1] - 0.2) < 0.02 and abs(frac[2] - 0.4) < 0.02 and abs(frac[3] - 0.4) < 0.02
    assert (c["JV"][c["cls"] == 3] == 0).all() and (c["JV"][c["cls"] != 3, 2] > 0).all()
    assert c["TEMP"].min() >= 220.0 and c["TEMP"].max() <= 310.0


def _code(ipar_mod=None, rpar_mod=None, atol=1.0, rtol=1e-3):
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    for k, v in (ipar_mod or {}).items():
        ipar[k] = v
    for k, v in (rpar_mod or {}).items():
        rpar[k] = v
    ok, _ = oracle.params(0.0, 600.0, np.full(59, atol), np.full(59, rtol), rpar, ipar)
    return ok


def test_parameter_validation_codes():
    assert _code() == 1
    assert _code(ipar_mod={2: -1}) == -1          # negative max steps
    assert _code(ipar_mod={3: 7}) == -2           # unknown method
    assert _code(rpar_mod={0: -1.0}) == -3        # Hmin < 0
    assert _code(rpar_mod={1: -1.0}) == -3        # Hmax < 0
    assert _code(rpar_mod={3: -0.5}) == -4        # FacMin < 0
    assert _code(rpar_mod={6: -0.9}) == -4        # FacSafe < 0
    assert _code(atol=0.0) == -5                  # AbsTol <= 0
    assert _code(rtol=1.0) == -5                  # RelTol >= 1
    assert _code(rtol=1e-20) == -5                # RelTol <= 10 * roundoff
