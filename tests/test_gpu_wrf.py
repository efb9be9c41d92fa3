"""WRF -> KPP conversion on the GPU (k_convert_wrf through radm2_convert_wrf) against the
oracle's restatement of dev_convert (mgpu.cu:513-646), and the reference's whole flow:
convert, rate constants, Rosenbrock."""
import ctypes

import numpy as np
import pytest

import oracle
import radm2b200
from conftest import rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
KEYS = ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")


def _check(got, exp):
    for k in ("VAR", "FIX", "TEMP", "JV"):  # products, quotients, clamps: bitwise
        assert np.array_equal(got[k], exp[k]), k
    # exp/pow of the device math library against the host's
    assert np.abs(got["RC_N2O5"] - exp["RC_N2O5"]).max() <= 1e-13 * np.abs(exp["RC_N2O5"]).max()


def test_convert_reference_grid_matches_oracle():
    f = inputs.make_wrf_fields(5)
    with radm2b200.Solver() as s:
        s.convert_wrf(f)
        assert s.ncell == 39 * 19 * 39
        _check(s.get_inputs(), oracle.convert_wrf(f))


def test_convert_other_grid_and_device_fields():
    import torch
    grid = (40, 12, 33, 3, 2, 5, 31, 9, 27)
    f = inputs.make_wrf_fields(8, ni=40, nk=12, nj=33)
    exp = oracle.convert_wrf(f, grid)
    with radm2b200.Solver() as s:
        s.convert_wrf(f, grid)
        _check(s.get_inputs(), exp)
    # the same from device-resident fields
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in f.items()}
    with radm2b200.Solver() as s:
        g = radm2b200.lib.WrfGrid(*grid)
        rc = s.lib.radm2_convert_wrf_device(s.h, ctypes.byref(g),
                                            *[ctypes.c_void_p(dev[k].data_ptr()) for k in ("ph", "chem", "rad", "phy",
                                                                                        "moist")])
        assert rc == 0
        s.ncell = 31 * 9 * 27
        s.synchronize()
        _check(s.get_inputs(), exp)


def test_bad_window_is_rejected():
    f = inputs.make_wrf_fields(1, ni=8, nk=4, nj=8)
    with radm2b200.Solver() as s:
        with pytest.raises(radm2b200.lib.RadmError):
            s.convert_wrf(f, (8, 4, 8, 4, 0, 4, 5, 4, 4))  # i0 + wi > ni


def test_reference_flow_convert_then_integrate():
    """convertWRFChemData -> updatingCoefficientWRFChemData -> Rosenbrock, as mgpu.cu:3891-3911
    runs them, on the GPU; a spread subset of cells re-run by the oracle."""
    f = inputs.make_wrf_fields(5)
    conv = oracle.convert_wrf(f)
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.convert_wrf(f)
        s.update_rconst()
        rc_gpu = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ierr = s.rosenbrock(0.0, 600.0, atol, rtol, rpar, ipar)
        assert ierr == 1
        y = s.get_state()
    idx = np.linspace(0, len(y) - 1, 64).astype(np.int64)
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, atol, rtol, rpar, ipar)
    y_o, _ = oracle.integrate(conv["VAR"][idx], conv["FIX"][idx], rc_gpu[idx], p)
    assert rel_err(y[idx], y_o).max() <= 1e-10
