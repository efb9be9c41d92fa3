"""ctypes binding of libradm2_b200.so (the C ABI in include/radm2.h).

This is the host-side mirror of the reference's entry points for Python
callers (tests, benchmark, the step-seeding trainer): `Solver.set_inputs`
stands for dev_convert's outputs (mgpu.cu:513-646), `Solver.update_rconst`
for updatingCoefficientWRFChemData (mgpu.cu:921-947) and `Solver.rosenbrock`
for Rosenbrock (mgpu.cu:3664-3848), with the same IPAR/RPAR arrays and IERR
codes.  The shared library is required: importing this module without it
raises, there is no fallback.
"""
import ctypes
import os

import numpy as np

NVAR, NFIX, NREACT, NPH, NJVS = 59, 2, 156, 28, 659
PREC_FP64, PREC_FP32LU = 0, 1
PLACE_GLOBAL, PLACE_LU_SMEM, PLACE_ALL_SMEM, PLACE_LU_TMEM = 0, 1, 3, 4
PLACE_LU_TMEM_WIDE = 10  # 256 LU slots in tensor memory, rate constants and state in shared memory
SCHED_STATIC, SCHED_PERSISTENT, SCHED_COOP = 0, 1, 2
RADM2_OK, RADM2_E_ARG, RADM2_E_CUDA, RADM2_E_NOMEM, RADM2_E_STATE, RADM2_E_NODEV, RADM2_E_TOOBIG = \
    0, -100, -101, -102, -103, -104, -105

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libradm2_b200.so")

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_F = ctypes.POINTER(ctypes.c_float)
NFEAT = 84


class Opts(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("precision", ctypes.c_int), ("refine_sweeps", ctypes.c_int),
                ("schedule", ctypes.c_int), ("block_threads", ctypes.c_int), ("blocks_per_sm", ctypes.c_int),
                ("float_coeffs", ctypes.c_int), ("placement", ctypes.c_int), ("min_blocks", ctypes.c_int),
                ("parity", ctypes.c_int), ("cells_per_thread", ctypes.c_int)]


class WrfGrid(ctypes.Structure):
    _fields_ = [(k, ctypes.c_int) for k in ("ni", "nk", "nj", "i0", "k0", "j0", "wi", "wk", "wj")]


class TuneEntry(ctypes.Structure):
    _fields_ = [("schedule", ctypes.c_int), ("block_threads", ctypes.c_int), ("placement", ctypes.c_int),
                ("min_blocks", ctypes.c_int), ("ms", ctypes.c_double), ("attempts", ctypes.c_longlong),
                ("cells_per_thread", ctypes.c_int)]


class Stats(ctypes.Structure):
    _fields_ = [("n_accepted", ctypes.c_longlong), ("n_rejected", ctypes.c_longlong),
                ("n_failed", ctypes.c_longlong), ("worst_status", ctypes.c_int), ("max_steps_cell", ctypes.c_int),
                ("texit_min", ctypes.c_double), ("hexit_min", ctypes.c_double)]


# Every symbol the header declares, with its signature.
SIGNATURES = {
    "radm2_opts_default": (ctypes.c_int, [ctypes.POINTER(Opts)]),
    "radm2_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(Opts)]),
    "radm2_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_error_string": (ctypes.c_char_p, [ctypes.c_int]),
    "radm2_last_error": (ctypes.c_char_p, [ctypes.c_void_p]),
    "radm2_set_stream": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "radm2_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_set_inputs": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, _D]),
    "radm2_set_state": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "radm2_get_state": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "radm2_set_inputs_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "radm2_get_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "radm2_set_state_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "radm2_update_rconst": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_get_rconst": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "radm2_set_rconst": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "radm2_rosenbrock": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.c_double, _D, _D, _D, _I]),
    "radm2_run_split": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, _D, _D, _D, _I,
                                       ctypes.c_int]),
    "radm2_get_cell_stats": (ctypes.c_int, [ctypes.c_void_p, _I, _I, _I, _D, _D]),
    "radm2_get_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Stats)]),
    "radm2_add_step_counters": (ctypes.c_int, [_I, ctypes.c_longlong, ctypes.c_longlong, ctypes.c_longlong,
                                               ctypes.c_int]),
    "radm2_set_cell_hstart": (ctypes.c_int, [ctypes.c_void_p, _D]),
    "radm2_set_cell_order": (ctypes.c_int, [ctypes.c_void_p, _I]),
    "radm2_fun": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D]),
    "radm2_jac": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D]),
    "radm2_decomp_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _D, _D, _I]),
    "radm2_set_kernel_timing": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "radm2_get_kernel_time": (ctypes.c_int, [ctypes.c_void_p, _D, _I]),
    "radm2_get_graph_kernels": (ctypes.c_int, [ctypes.c_void_p, _I]),
    "radm2_fma_peak": (ctypes.c_int, [ctypes.c_int, _D, _D]),
    "radm2_mlp_nparams": (ctypes.c_int, []),
    "radm2_mlp_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_uint]),
    "radm2_mlp_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_mlp_set_params": (ctypes.c_int, [ctypes.c_void_p, _F]),
    "radm2_mlp_get_params": (ctypes.c_int, [ctypes.c_void_p, _F]),
    "radm2_mlp_set_norm": (ctypes.c_int, [ctypes.c_void_p, _F, _F, _F, _F]),
    "radm2_mlp_forward": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F, _F]),
    "radm2_mlp_gradients": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _F, _F, _F, _F]),
    "radm2_mlp_train_step": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                            ctypes.c_float, _F]),
    "radm2_mlp_synchronize": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_mlp_set_h0_scale": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_float]),
    "radm2_mlp_set_tensor_path": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    "radm2_mlp_status": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_mlp_selftest_wait_limit": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_get_features": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, _F]),
    "radm2_seed_cells": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                                        ctypes.c_int]),
    "radm2_attach_mlp": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]),
    "radm2_get_ncell": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_rosenbrock_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_double,
                                             ctypes.c_double, _D, _D, _D, ctypes.POINTER(ctypes.c_int),
                                             ctypes.c_int]),
    "radm2_get_inputs": (ctypes.c_int, [ctypes.c_void_p, _D, _D, _D, _D, _D]),
    "radm2_wrf_grid_default": (ctypes.c_int, [ctypes.POINTER(WrfGrid)]),
    "radm2_convert_wrf": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WrfGrid), _D, _D, _D, _D, _D]),
    "radm2_convert_wrf_device": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(WrfGrid), ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]),
    "radm2_get_opts": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(Opts)]),
    "radm2_autotune": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_double, ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double),
                                      ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.POINTER(TuneEntry),
                                      ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "radm2_device_bytes": (ctypes.c_size_t, [ctypes.c_void_p]),
    "radm2_rosenbrock_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                                 ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double,
                                                 ctypes.c_double, _D, _D, _D, _I, ctypes.c_void_p, ctypes.c_void_p]),
    "radm2_selfcheck": (ctypes.c_int, []),
    "radm2_coop_selftest_wait_limit": (ctypes.c_int, [ctypes.c_void_p]),
    "radm2_version": (ctypes.c_char_p, []),
}

_lib = None


def load():
    """Load the shared library (raises OSError if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libradm2_b200.so not built (%s); run __graft_entry__.build()" % LIB_PATH)
        lib = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        _lib = lib
    return _lib


def fma_peak(device=0):
    """Measured CUDA-core FMA throughput (fp64_tflops, fp32_tflops)."""
    lib = load()
    a, b = ctypes.c_double(), ctypes.c_double()
    rc = lib.radm2_fma_peak(device, ctypes.byref(a), ctypes.byref(b))
    if rc != 0:
        raise RadmError(rc, lib.radm2_error_string(rc).decode())
    return a.value, b.value


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


def _c64(a, shape=None):
    a = np.ascontiguousarray(a, dtype=np.float64)
    if shape is not None:
        a = a.reshape(shape)
    return a


class RadmError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("radm2 error %d: %s" % (code, msg))
        self.code = code


def add_step_counters(ipar, n_accepted, n_rejected, n_failed=0, autonomous=True):
    """IPAR[10..16] += the statistics of an integration with these 64-bit step totals, each
    slot saturating at INT_MAX (the library's own update; no device needed)."""
    lib = load()
    assert ipar.dtype == np.int32 and ipar.flags.c_contiguous
    rc = lib.radm2_add_step_counters(_ip(ipar), int(n_accepted), int(n_rejected), int(n_failed),
                                     1 if autonomous else 0)
    if rc != 0:
        raise RadmError(rc, lib.radm2_error_string(rc).decode())
    return ipar


def default_params(hstart=0.0, max_steps=0, autonomous=True):
    """IPAR/RPAR as the reference driver sets them (mgpu.cu:3863-3873)."""
    ipar = np.zeros(20, dtype=np.int32)
    rpar = np.zeros(20, dtype=np.float64)
    ipar[0] = 1 if autonomous else 0
    ipar[2] = max_steps
    ipar[3] = 2
    rpar[2] = hstart
    return ipar, rpar


class Solver:
    """One device context of the batched solver."""

    def __init__(self, precision=PREC_FP64, schedule=SCHED_STATIC, refine_sweeps=1, block_threads=0,
                 blocks_per_sm=0, float_coeffs=1, device=0, placement=PLACE_GLOBAL, min_blocks=0, parity=0,
                 cells_per_thread=1):
        self.lib = load()
        o = Opts()
        self.lib.radm2_opts_default(ctypes.byref(o))
        o.device, o.precision, o.refine_sweeps, o.schedule = device, precision, refine_sweeps, schedule
        o.block_threads, o.blocks_per_sm, o.float_coeffs = block_threads, blocks_per_sm, float_coeffs
        o.placement = placement
        o.min_blocks = min_blocks
        o.parity = parity
        o.cells_per_thread = cells_per_thread
        h = ctypes.c_void_p()
        rc = self.lib.radm2_create(ctypes.byref(h), ctypes.byref(o))
        if rc != 0:
            raise RadmError(rc, self.lib.radm2_error_string(rc).decode())
        self.h = h
        self.ncell = 0

    def close(self):
        if getattr(self, "h", None):
            self.lib.radm2_destroy(self.h)  # detaches an attached network
            self.h = None
            self._mlp = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _check(self, rc):
        if rc != 0:
            raise RadmError(rc, "%s (%s)" % (self.lib.radm2_error_string(rc).decode(),
                                             self.lib.radm2_last_error(self.h).decode()))

    # ---- inputs / state
    def set_inputs(self, VAR, FIX, TEMP, RC_N2O5, JV):
        n = VAR.shape[0]
        VAR, FIX, TEMP, JV = _c64(VAR, (n, NVAR)), _c64(FIX, (n, NFIX)), _c64(TEMP, (n,)), _c64(JV, (n, NPH))
        rcn = None if RC_N2O5 is None else _c64(RC_N2O5, (n,))
        self._check(self.lib.radm2_set_inputs(self.h, n, _dp(VAR), _dp(FIX), _dp(TEMP),
                                              None if rcn is None else _dp(rcn), _dp(JV)))
        self.ncell = n

    def set_cells(self, cells):
        self.set_inputs(cells["VAR"], cells["FIX"], cells["TEMP"], cells["RC_N2O5"], cells["JV"])

    def set_state(self, VAR):
        VAR = _c64(VAR, (self.ncell, NVAR))
        self._check(self.lib.radm2_set_state(self.h, _dp(VAR)))

    def get_state(self, out=None):
        if out is None:
            out = np.empty((self.ncell, NVAR), dtype=np.float64)
        self._check(self.lib.radm2_get_state(self.h, _dp(out)))
        return out

    def get_state_device(self, ptr, ld):
        """Copy the species state to device memory var[59][ld] (ptr: device address)."""
        self._check(self.lib.radm2_get_state_device(self.h, ctypes.c_void_p(ptr), ld))

    def set_state_device(self, ptr, ld):
        self._check(self.lib.radm2_set_state_device(self.h, ctypes.c_void_p(ptr), ld))

    def update_rconst(self):
        self._check(self.lib.radm2_update_rconst(self.h))

    def get_rconst(self):
        out = np.empty((self.ncell, NREACT), dtype=np.float64)
        self._check(self.lib.radm2_get_rconst(self.h, _dp(out)))
        return out

    def set_rconst(self, rc):
        rc = _c64(rc, (self.ncell, NREACT))
        self._check(self.lib.radm2_set_rconst(self.h, _dp(rc)))

    # ---- integration
    def rosenbrock(self, tstart, tend, atol, rtol, rpar, ipar):
        """Mirror of Rosenbrock(): returns IERR; rpar/ipar (numpy) are updated in place."""
        atol, rtol = _c64(atol), _c64(rtol)
        assert rpar.dtype == np.float64 and ipar.dtype == np.int32
        return self.lib.radm2_rosenbrock(self.h, tstart, tend, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar))

    def run_split(self, nsplit, dt, atol, rtol, rpar, ipar, use_graph=True):
        atol, rtol = _c64(atol), _c64(rtol)
        return self.lib.radm2_run_split(self.h, nsplit, dt, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar),
                                        1 if use_graph else 0)

    def cell_stats(self):
        n = self.ncell
        st, na, nr = (np.empty(n, np.int32) for _ in range(3))
        hf, hx = np.empty(n), np.empty(n)
        self._check(self.lib.radm2_get_cell_stats(self.h, _ip(st), _ip(na), _ip(nr), _dp(hf), _dp(hx)))
        return {"status": st, "nacc": na, "nrej": nr, "hfirst": hf, "hexit": hx}

    def stats(self):
        s = Stats()
        self._check(self.lib.radm2_get_stats(self.h, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in Stats._fields_}

    def set_cell_hstart(self, h0):
        if h0 is None:
            self._check(self.lib.radm2_set_cell_hstart(self.h, None))
        else:
            h0 = _c64(h0, (self.ncell,))
            self._check(self.lib.radm2_set_cell_hstart(self.h, _dp(h0)))

    def set_cell_order(self, order):
        if order is None:
            self._check(self.lib.radm2_set_cell_order(self.h, None))
        else:
            order = np.ascontiguousarray(order, dtype=np.int32)
            self._check(self.lib.radm2_set_cell_order(self.h, _ip(order)))

    def synchronize(self):
        self._check(self.lib.radm2_synchronize(self.h))

    def set_stream(self, stream_ptr):
        self._check(self.lib.radm2_set_stream(self.h, ctypes.c_void_p(stream_ptr) if stream_ptr else None))

    def set_kernel_timing(self, enable=True):
        self._check(self.lib.radm2_set_kernel_timing(self.h, 1 if enable else 0))

    def kernel_time(self):
        """(device ms of solver-kernel launches, launch count) since the previous call."""
        ms, n = ctypes.c_double(), ctypes.c_int()
        self._check(self.lib.radm2_get_kernel_time(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def graph_kernels(self):
        """Kernel nodes of the cached split graph (kernels per replay; 0 = none cached)."""
        n = ctypes.c_int()
        self._check(self.lib.radm2_get_graph_kernels(self.h, ctypes.byref(n)))
        return n.value

    def device_bytes(self):
        return int(self.lib.radm2_device_bytes(self.h))

    def coop_selftest_wait_limit(self):
        """Cooperative kernel: one integration in which a warp of every block waits on a
        flag nothing sets; the bounded wait must run out and be reported (raises if not)."""
        self._check(self.lib.radm2_coop_selftest_wait_limit(self.h))

    # ---- learned seeding
    def features(self, dt):
        out = np.empty((self.ncell, NFEAT), dtype=np.float32)
        self._check(self.lib.radm2_get_features(self.h, dt, out.ctypes.data_as(_F)))
        return out

    def convert_wrf(self, fields, grid=None):
        """WRF fields (dict ph/chem/rad/phy/moist, each [nfield][nj][nk][ni], host) -> the
        context's cells (default grid: the reference's 48 x 20 x 48 domain and window)."""
        g = WrfGrid()
        if grid is None:
            self.lib.radm2_wrf_grid_default(ctypes.byref(g))
        else:
            g = WrfGrid(*grid)
        arrs = [np.ascontiguousarray(fields[k], dtype=np.float64) for k in ("ph", "chem", "rad", "phy", "moist")]
        self._check(self.lib.radm2_convert_wrf(self.h, ctypes.byref(g), *[_dp(a) for a in arrs]))
        self.ncell = g.wi * g.wk * g.wj

    def get_inputs(self):
        """The current per-cell inputs (reference layout)."""
        n = self.ncell
        out = {"VAR": np.empty((n, NVAR)), "FIX": np.empty((n, NFIX)), "TEMP": np.empty(n), "RC_N2O5": np.empty(n),
               "JV": np.empty((n, NPH))}
        self._check(self.lib.radm2_get_inputs(self.h, *[_dp(out[k]) for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")]))
        return out

    def rosenbrock_host(self, VAR, FIX, TEMP, RC_N2O5, JV, tstart, tend, atol, rtol, rpar, ipar, nchunk=8):
        """Integrate host arrays (reference layout) with copies overlapped with the solve;
        VAR (float64, C-contiguous) is overwritten with the result.  Returns IERR."""
        n = VAR.shape[0]
        if VAR.dtype != np.float64 or not VAR.flags.c_contiguous or VAR.shape[1] != NVAR:
            raise ValueError("VAR must be a C-contiguous float64 [n][59] array (updated in place)")
        FIX, TEMP, JV = _c64(FIX, (n, NFIX)), _c64(TEMP, (n,)), _c64(JV, (n, NPH))
        rcn = None if RC_N2O5 is None else _c64(RC_N2O5, (n,))
        atol, rtol = _c64(atol), _c64(rtol)
        ierr = self.lib.radm2_rosenbrock_host(self.h, n, _dp(VAR), _dp(FIX), _dp(TEMP),
                                              _dp(rcn) if rcn is not None else None, _dp(JV), tstart, tend,
                                              _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar), nchunk)
        self.ncell = n
        return ierr

    def opts(self):
        """The options in force (the autotuner rewrites schedule / block shape / placement)."""
        o = Opts()
        self._check(self.lib.radm2_get_opts(self.h, ctypes.byref(o)))
        return {k: getattr(o, k) for k, _ in Opts._fields_}

    def autotune(self, dt, atol, rtol, rpar=None, ipar=None, sample_cells=0):
        """Time every built variant on a strided sample of the current cells for one split;
        keep the fastest.  Returns the candidate table (ms = -1: did not run)."""
        if rpar is None or ipar is None:
            ipar, rpar = default_params()
        atol, rtol = _c64(atol), _c64(rtol)
        rpar, ipar = _c64(rpar), np.ascontiguousarray(ipar, dtype=np.int32)
        tab = (TuneEntry * 64)()
        n = ctypes.c_int()
        self._check(self.lib.radm2_autotune(self.h, dt, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar), sample_cells,
                                            tab, 64, ctypes.byref(n)))
        return [{k: getattr(tab[i], k) for k, _ in TuneEntry._fields_} for i in range(min(n.value, 64))]

    def attach_mlp(self, mlp, order=False):
        """Seed every following integration from the network (None detaches); order: False/0
        none, True/1 cells by predicted cost, 2 chunks of 32 cells by cost."""
        mode = 1 if order is True else int(order or 0)  # 0 none, 1 cells, 2 chunks of 32 cells
        self._check(self.lib.radm2_attach_mlp(self.h, mlp.h if mlp is not None else None, mode))
        self._mlp = mlp  # keep the network alive while attached

    def seed_cells(self, mlp, dt, h0=True, order=True):
        mode = 1 if order is True else int(order or 0)
        self._check(self.lib.radm2_seed_cells(self.h, mlp.h, dt, 1 if h0 else 0, mode))

    # ---- mechanism kernels
    def fun(self, V, FIX, RCT):
        n = V.shape[0]
        V, FIX, RCT = _c64(V, (n, NVAR)), _c64(FIX, (n, NFIX)), _c64(RCT, (n, NREACT))
        out = np.empty((n, NVAR))
        self._check(self.lib.radm2_fun(self.h, n, _dp(V), _dp(FIX), _dp(RCT), _dp(out)))
        return out

    def jac(self, V, FIX, RCT):
        n = V.shape[0]
        V, FIX, RCT = _c64(V, (n, NVAR)), _c64(FIX, (n, NFIX)), _c64(RCT, (n, NREACT))
        out = np.empty((n, NJVS))
        self._check(self.lib.radm2_jac(self.h, n, _dp(V), _dp(FIX), _dp(RCT), _dp(out)))
        return out

    def decomp_solve(self, G, X, precision=PREC_FP64):
        n = G.shape[0]
        G, X = _c64(G, (n, NJVS)).copy(), _c64(X, (n, NVAR)).copy()
        sing = np.empty(n, np.int32)
        self._check(self.lib.radm2_decomp_solve(self.h, n, precision, _dp(G), _dp(X), _ip(sing)))
        return G, X, sing


class Mlp:
    """The step-seeding network (radm2_mlp_* in the C ABI)."""

    def __init__(self, seed=0, device=0):
        self.lib = load()
        h = ctypes.c_void_p()
        rc = self.lib.radm2_mlp_create(ctypes.byref(h), device, seed)
        if rc != 0:
            raise RadmError(rc, self.lib.radm2_error_string(rc).decode())
        self.h = h
        self.nparams = self.lib.radm2_mlp_nparams()

    def close(self):
        # refused (RADM2_E_STATE) while a context still seeds from this network
        if getattr(self, "h", None) and self.lib.radm2_mlp_destroy(self.h) == RADM2_OK:
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, rc):
        if rc != 0:
            raise RadmError(rc, self.lib.radm2_error_string(rc).decode())

    @staticmethod
    def _f(a, shape=None):
        a = np.ascontiguousarray(a, dtype=np.float32)
        return a.reshape(shape) if shape is not None else a

    def params(self):
        out = np.empty(self.nparams, dtype=np.float32)
        self._check(self.lib.radm2_mlp_get_params(self.h, out.ctypes.data_as(_F)))
        return out

    def set_params(self, p):
        p = self._f(p, (self.nparams,))
        self._check(self.lib.radm2_mlp_set_params(self.h, p.ctypes.data_as(_F)))

    def set_norm(self, xmean, xstd, ymean, ystd):
        a = [self._f(v) for v in (xmean, xstd, ymean, ystd)]
        self._check(self.lib.radm2_mlp_set_norm(self.h, *[v.ctypes.data_as(_F) for v in a]))
        self.norm = a

    def forward(self, x):
        x = self._f(x, (-1, NFEAT))
        y = np.empty((x.shape[0], 2), dtype=np.float32)
        self._check(self.lib.radm2_mlp_forward(self.h, x.shape[0], x.ctypes.data_as(_F), y.ctypes.data_as(_F)))
        return y

    def gradients(self, x, t):
        x, t = self._f(x, (-1, NFEAT)), self._f(t, (-1, 2))
        g = np.empty(self.nparams, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(self.lib.radm2_mlp_gradients(self.h, x.shape[0], x.ctypes.data_as(_F), t.ctypes.data_as(_F),
                                                 g.ctypes.data_as(_F), ctypes.byref(loss)))
        return g, loss.value

    def train_step(self, n, x_dev_ptr, t_dev_ptr, lr, want_loss=False):
        loss = ctypes.c_float()
        self._check(self.lib.radm2_mlp_train_step(self.h, n, ctypes.c_void_p(x_dev_ptr), ctypes.c_void_p(t_dev_ptr),
                                                  lr, ctypes.byref(loss) if want_loss else None))
        return loss.value if want_loss else None

    def synchronize(self):
        self._check(self.lib.radm2_mlp_synchronize(self.h))

    def set_h0_scale(self, scale):
        self._check(self.lib.radm2_mlp_set_h0_scale(self.h, scale))

    def set_tensor_path(self, tcgen05=True):
        """Inference forward on tcgen05 with tensor-memory accumulators (default) or on
        mma.sync tiles; training always uses the mma.sync kernels."""
        self._check(self.lib.radm2_mlp_set_tensor_path(self.h, 1 if tcgen05 else 0))

    def status(self):
        """Raise if a tcgen05 forward gave up waiting on its tensor-core work."""
        self._check(self.lib.radm2_mlp_status(self.h))

    def selftest_wait_limit(self):
        """Run the tcgen05 forward with no tensor-core work issued: its bounded waits must
        run out, raise the status flag (cleared afterwards) and return."""
        self._check(self.lib.radm2_mlp_selftest_wait_limit(self.h))
