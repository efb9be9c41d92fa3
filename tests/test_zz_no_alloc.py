"""radm2_rosenbrock_noalloc: the integration entry point that allocates nothing.

Some callers may not allocate device memory while they run: a host framework that reserved
all of the GPU's memory for its own pool at start-up, or a coupling whose device memory
budget is fixed at initialisation.  This test allocates the caller's input/output buffers
itself (the caller owns those), calls the entry point through the C ABI several times in a
row, and checks each result against the context-based radm2_rosenbrock on the same cells and
against the CPU oracle: to 1e-13 relative against the context entry point running the same
solver kernel, and within the parity tolerance the other solver tests use against the oracle
(1e-10 relative, floor 1 molec/cm^3).  It also checks with cudaMemGetInfo that a call after the
first (the set-up call) leaves the device's free memory unchanged.  The file is collected
last on purpose; it passes alone in a fresh process and after the others.
"""
import ctypes

import numpy as np
import pytest

import oracle
import radm2b200
from conftest import ATOL, RTOL, SAME_ARITH, rel_err
from radm2b200 import inputs

pytestmark = pytest.mark.gpu
PARITY = 1e-10
MAX_CELLS = 32768


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
    """The context entry point on the same cells, with the solver variant the no-alloc call
    runs (persistent schedule, 32 threads, the working set in shared memory): IERR, states,
    statuses, rate constants, IPAR, RPAR."""
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT, block_threads=32,
                          placement=radm2b200.lib.PLACE_ALL_SMEM) as s:
        s.set_cells(cells)
        s.update_rconst()
        rc = s.get_rconst()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        ierr = s.rosenbrock(0.0, 600.0, ATOL, RTOL, rpar, ipar)
        return ierr, s.get_state(), s.cell_stats()["status"], rc, ipar, rpar


class _Call:
    """The caller's device buffers for one batch, and calls of the entry point on them."""

    def __init__(self, torch, lib, cells, ld, with_status=True):
        self.torch, self.lib, self.cells, self.ld = torch, lib, cells, ld
        self.n = len(cells["TEMP"])
        self.fix = _soa(torch, cells["FIX"], ld)
        self.temp = _soa(torch, cells["TEMP"], ld)
        self.rcn = _soa(torch, cells["RC_N2O5"], ld)
        self.jv = _soa(torch, cells["JV"], ld)
        self.var0 = _soa(torch, cells["VAR"], ld)
        self.var = self.var0.clone()
        self.status = torch.zeros(self.n, dtype=torch.int32, device="cuda") if with_status else None
        self.atol, self.rtol = np.ascontiguousarray(ATOL), np.ascontiguousarray(RTOL)

    def __call__(self):
        """One integration from the initial state.  Nothing here allocates device memory: the
        state is reset by an in-place copy and results are read back as whole buffers."""
        torch = self.torch
        self.var.copy_(self.var0)
        if self.status is not None:
            self.status.fill_(0)
        torch.cuda.synchronize()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        stream = torch.cuda.current_stream().cuda_stream
        ierr = self.lib.radm2_rosenbrock_noalloc(
            self.n, self.ld, self.var.data_ptr(), self.fix.data_ptr(), self.temp.data_ptr(), self.rcn.data_ptr(),
            self.jv.data_ptr(), 0.0, 600.0, _dp(self.atol), _dp(self.rtol), _dp(rpar), _ip(ipar),
            self.status.data_ptr() if self.status is not None else None, stream)
        y = np.ascontiguousarray(self.var.cpu().numpy()[:, :self.n].T)
        st = self.status.cpu().numpy() if self.status is not None else None
        return ierr, y, st, ipar, rpar


def _oracle(cells, rc, idx):
    ipar, rpar = radm2b200.default_params(hstart=6.0)
    ok, p = oracle.params(0.0, 600.0, ATOL, RTOL, rpar, ipar)
    assert ok == 1
    y_o, _ = oracle.integrate(cells["VAR"][idx], cells["FIX"][idx], rc[idx], p)
    return y_o


def test_noalloc_matches_context_entry_point_and_oracle_without_allocating():
    torch = pytest.importorskip("torch")
    lib = radm2b200.load()
    n = 3000  # not a multiple of the block size, below the limit
    cells = inputs.make_cells(n, 5, "plain", night_frac=0.3)
    ierr_ref, y_ref, st_ref, rc, ipar_ref, rpar_ref = _reference(cells)
    assert ierr_ref == 1
    y_orc = _oracle(cells, rc, np.arange(n))
    call = _Call(torch, lib, cells, 3008)
    free = []
    for k in range(3):  # the static area keeps the previous call's contents
        torch.cuda.synchronize()
        free.append(torch.cuda.mem_get_info()[0])
        ierr, y, st, ipar, rpar = call()
        assert ierr == 1, (k, ierr)
        assert (st == 1).all() and (st == st_ref).all()
        assert rel_err(y, y_ref).max() <= SAME_ARITH, k
        assert rel_err(y, y_orc).max() <= PARITY, k
        assert list(ipar[10:17]) == list(ipar_ref[10:17])
        assert rpar[10] == rpar_ref[10] == 600.0 and abs(rpar[11] - rpar_ref[11]) <= 1e-12 * rpar_ref[11]
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
    # the first call is the set-up (module load, address lookup); later calls allocate nothing
    assert free[1] == free[2] == free[3], free


def test_noalloc_without_status_array_at_the_size_limit():
    """status = NULL (the outcomes go to the static area and feed the statistics) at the
    largest batch, ncell = ld = RADM2_NOALLOC_MAX_CELLS: the persistent grid's block cap and
    the scratch sizing are exercised.  States and IPAR counters equal the context path's;
    every 64th cell is checked against the oracle."""
    torch = pytest.importorskip("torch")
    lib = radm2b200.load()
    cells = inputs.make_cells(MAX_CELLS, 8, "plain", night_frac=0.3)
    ierr_ref, y_ref, _, rc, ipar_ref, rpar_ref = _reference(cells)
    assert ierr_ref == 1
    call = _Call(torch, lib, cells, MAX_CELLS, with_status=False)
    for _ in range(2):
        ierr, y, _, ipar, rpar = call()
        assert ierr == 1
        assert rel_err(y, y_ref).max() <= SAME_ARITH
        assert list(ipar[10:17]) == list(ipar_ref[10:17])
        assert abs(rpar[11] - rpar_ref[11]) <= 1e-12 * rpar_ref[11]
    idx = np.arange(0, MAX_CELLS, 64)
    assert rel_err(y[idx], _oracle(cells, rc, idx)).max() <= PARITY


def test_noalloc_rejects_oversize_and_bad_parameters():
    torch = pytest.importorskip("torch")
    lib = radm2b200.load()
    cells = inputs.make_cells(64, 5, "plain")
    ipar, rpar = radm2b200.default_params()
    atol, rtol = np.ascontiguousarray(ATOL), np.ascontiguousarray(RTOL)
    big = MAX_CELLS + 32
    dummy = torch.zeros(59 * big, dtype=torch.float64, device="cuda")
    p = dummy.data_ptr()
    rc = lib.radm2_rosenbrock_noalloc(big, big, p, p, p, None, p, 0.0, 600.0, _dp(atol), _dp(rtol), _dp(rpar),
                                      _ip(ipar), None, None)
    assert rc == -105  # RADM2_E_TOOBIG
    rc = lib.radm2_rosenbrock_noalloc(64, big, p, p, p, None, p, 0.0, 600.0, _dp(atol), _dp(rtol), _dp(rpar),
                                      _ip(ipar), None, None)
    assert rc == -105  # the leading dimension counts against the limit too
    ipar[3] = 7
    var = _soa(torch, cells["VAR"], 64)
    rc = lib.radm2_rosenbrock_noalloc(64, 64, var.data_ptr(), p, p, None, p, 0.0, 600.0, _dp(atol), _dp(rtol),
                                      _dp(rpar), _ip(ipar), None, None)
    assert rc == -2
