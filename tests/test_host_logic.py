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


def test_step_counters_saturate_instead_of_wrapping():
    """IPAR[10..16] are C ints in the reference's interface.  A 4M-cell, 24-split batch takes
    ~0.8e9 step attempts, so Nsol (3 per attempt) passes 2^31: the library's update (the one
    radm2_rosenbrock applies, called here on the host) saturates each slot at INT_MAX."""
    big = 10 ** 9
    ipar = np.zeros(20, dtype=np.int32)
    radm2b200.add_step_counters(ipar, big, 5, n_failed=2)
    assert ipar[13] == big and ipar[14] == 5
    assert ipar[12] == big + 5 and ipar[15] == big + 5      # Nstp, Ndec
    assert ipar[11] == big + 2                              # Njac: accepted + failed outer steps
    assert ipar[10] == (big + 2) + (big + 5)                # Nfun, autonomous
    assert ipar[16] == 2 ** 31 - 1                          # Nsol = 3 x 1e9 + 15: saturated
    radm2b200.add_step_counters(ipar, big, 0)               # a second integration
    assert ipar[13] == 2 * big and ipar[10] == 2 ** 31 - 1 and ipar[16] == 2 ** 31 - 1
    radm2b200.add_step_counters(ipar, big, 0)
    assert ipar[13] == 2 ** 31 - 1 and (ipar[10:17] > 0).all()  # never wraps negative
    assert ipar[17] == 0 and ipar[:10].sum() == 0
    # small counts add exactly, as before
    ipar = np.zeros(20, dtype=np.int32)
    radm2b200.add_step_counters(ipar, 7, 3, autonomous=False)
    assert list(ipar[10:17]) == [2 * 7 + 10, 7, 10, 7, 3, 10, 30]
