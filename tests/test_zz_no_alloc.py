"""radm2_rosenbrock_noalloc: the integration entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc (code running under CUDA-graph
capture, frameworks that reserved all device memory up front, fixed-budget real-time
couplings).  This test allocates the caller's input/output buffers itself (the caller
owns those), calls the entry point through the C ABI twice in a row, and checks each
result against the context-based radm2_rosenbrock on the same cells, with the parity
tolerance the other solver tests use (1e-10 relative, floor 1 molec/cm^3).  The file is
collected last on purpose; it passes alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

import radm2b200
from conftest import ATOL, RTOL, rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
PARITY = 1e-10
NCELL = 3000  # not a multiple of the block size, below the 32768-cell limit


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _ip(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


def _soa(torch, a, ld):
    """Host per-cell array [n][m] -> device struct-of-arrays [m][ld]."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        a = a[:, None]
    t = torch.zeros((a.shape[1], ld), dtype=torch.float64)
    t[:, :a.shape[0]] = torch.from_numpy(np.ascontiguousarray(a.T))
    return t.cuda()


def _reference(cells):
    with radm2b200.Solver() as s:
        s.set_cells(cells)
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ierr = s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        return ierr, s.get_state(), s.cell_stats()["status"], ipar, rpar


def _noalloc(torch, lib, cells, ld):
    var = _soa(torch, cells["VAR"], ld)
    fix = _soa(torch, cells["FIX"], ld)
    temp = _soa(torch, cells["TEMP"], ld)
    rcn = _soa(torch, cells["RC_N2O5"], ld)
    jv = _soa(torch, cells["JV"], ld)
    status = torch.zeros(NCELL, dtype=torch.int32, device="cuda")
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    atol, rtol = np.ascontiguousarray(ATOL), np.ascontiguousarray(RTOL)
    stream = torch.cuda.current_stream().cuda_stream
    ierr = lib.radm2_rosenbrock_noalloc(NCELL, ld, var.data_ptr(), fix.data_ptr(), temp.data_ptr(), rcn.data_ptr(),
                                        jv.data_ptr(), 0.0, 600.0, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar),
                                        status.data_ptr(), stream)
    y = var[:, :NCELL].T.contiguous().cpu().numpy()
    return ierr, y, status.cpu().numpy(), ipar, rpar


def test_noalloc_matches_context_entry_point_twice():
    torch = pytest.importorskip("torch")
    lib = radm2b200.load()
    cells = inputs.make_cells(NCELL, 5, "plain", night_frac=0.3)
    ierr_ref, y_ref, st_ref, ipar_ref, rpar_ref = _reference(cells)
    assert ierr_ref == 1
    ld = 3008
    for call in range(2):  # the static area keeps the previous call's contents
        ierr, y, st, ipar, rpar = _noalloc(torch, lib, cells, ld)
        assert ierr == 1, (call, ierr)
        assert (st == 1).all() and (st == st_ref).all()
        assert rel_err(y, y_ref).max() <= PARITY, call
        assert ipar[13] == ipar_ref[13] and ipar[14] == ipar_ref[14]
        assert rpar[10] == rpar_ref[10] == 600.0


def test_noalloc_rejects_oversize_and_bad_parameters():
    torch = pytest.importorskip("torch")
    lib = radm2b200.load()
    cells = inputs.make_cells(64, 5, "plain")
    ipar, rpar = radm2b200.default_params()
    atol, rtol = np.ascontiguousarray(ATOL), np.ascontiguousarray(RTOL)
    big = 32768 + 32
    dummy = torch.zeros(59 * big, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    rc = lib.radm2_rosenbrock_noalloc(big, big, p, p, p, None, p, 0.0, 600.0, _dp(atol), _dp(rtol), _dp(rpar),
                                      _ip(ipar), None, None)
    assert rc == -105  # RADM2_E_TOOBIG
    ipar[3] = 7
    var = _soa(torch, cells["VAR"], 64)
    rc = lib.radm2_rosenbrock_noalloc(64, 64, var.data_ptr(), p, p, None, p, 0.0, 600.0, _dp(atol), _dp(rtol),
                                      _dp(rpar), _ip(ipar), None, None)
    assert rc == -2
