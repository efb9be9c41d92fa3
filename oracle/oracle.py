"""ctypes access to the CPU oracle and to the reference harness.

TEST INFRASTRUCTURE ONLY: imported by tests/, by the smoke check and by the
benchmark's CPU-baseline leg, never by the product.

  liboracle_radm2.so   the C restatement (radm2_oracle.c + gen/)       -- always
  _ref/libradm2_ref.so the reference's own mechanism functions, cut     -- only where
                       from mgpu.cu by build_ref.py                        it was built
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle_radm2.so")
REF_SO = os.path.join(HERE, "_ref", "libradm2_ref.so")
NVAR, NFIX, NREACT, NPH, NJVS = 59, 2, 156, 28, 659

_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)


class CellStats(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int), ("nacc", ctypes.c_int), ("nrej", ctypes.c_int),
                ("texit", ctypes.c_double), ("hexit", ctypes.c_double), ("hfirst", ctypes.c_double)]


class Params(ctypes.Structure):
    _fields_ = [("Tstart", ctypes.c_double), ("Tend", ctypes.c_double),
                ("AbsTol", ctypes.c_double * NVAR), ("RelTol", ctypes.c_double * NVAR),
                ("Hmin", ctypes.c_double), ("Hmax", ctypes.c_double), ("Hstart", ctypes.c_double),
                ("FacMin", ctypes.c_double), ("FacMax", ctypes.c_double), ("FacRej", ctypes.c_double),
                ("FacSafe", ctypes.c_double), ("Roundoff", ctypes.c_double),
                ("max_steps", ctypes.c_int), ("autonomous", ctypes.c_int), ("float_coeffs", ctypes.c_int)]


def _dp(a):
    return a.ctypes.data_as(_D)


def _ip(a):
    return a.ctypes.data_as(_I)


def _c(a, shape):
    return np.ascontiguousarray(a, dtype=np.float64).reshape(shape)


_lib = None


class WrfGrid(ctypes.Structure):
    """WRF field dimensions (i fastest) and the interior window converted to cells."""
    _fields_ = [(k, ctypes.c_int) for k in ("ni", "nk", "nj", "i0", "k0", "j0", "wi", "wk", "wj")]


# The reference's domain and window (mgpu.cu:513-536, 682-706).
REF_WRF_GRID = (48, 20, 48, 4, 0, 4, 39, 19, 39)


def _wrf_outputs(g):
    n = g.wi * g.wk * g.wj
    return {"VAR": np.zeros((n, NVAR)), "FIX": np.zeros((n, NFIX)), "TEMP": np.zeros(n), "RC_N2O5": np.zeros(n),
            "JV": np.zeros((n, NPH))}


def _wrf_fields(fields):
    return [np.ascontiguousarray(fields[k], dtype=np.float64) for k in ("ph", "chem", "rad", "phy", "moist")]


def convert_wrf(fields, grid=REF_WRF_GRID):
    """WRF fields (dict ph/chem/rad/phy/moist, each [nfield][nj][nk][ni]) -> per-cell inputs."""
    g = WrfGrid(*grid)
    out = _wrf_outputs(g)
    f = _wrf_fields(fields)
    lib().orc_convert_wrf(ctypes.byref(g), *[_dp(a) for a in f],
                          *[_dp(out[k]) for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")])
    return out


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise OSError("oracle not built: %s (make -C oracle)" % ORACLE_SO)
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_rconst.argtypes = [_D, ctypes.c_double, ctypes.c_double, ctypes.c_double, _D]
        L.orc_fun.argtypes = [_D, _D, _D, _D]
        L.orc_jac.argtypes = [_D, _D, _D, _D]
        L.orc_decomp.argtypes = [_D]
        L.orc_decomp.restype = ctypes.c_int
        L.orc_solve.argtypes = [_D, _D]
        L.orc_wlamch.restype = ctypes.c_double
        L.orc_integrate_batch.argtypes = [ctypes.c_int, _D, _D, _D, ctypes.POINTER(Params),
                                          ctypes.POINTER(CellStats), ctypes.c_int]
        L.orc_rconst_batch.argtypes = [ctypes.c_int, _D, _D, _D, _D, _D, ctypes.c_int]
        L.orc_rosenbrock.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D, _D, _I, ctypes.c_int, _D, _D, _D,
                                     ctypes.c_int, ctypes.POINTER(CellStats), ctypes.c_int]
        L.orc_rosenbrock.restype = ctypes.c_int
        L.orc_parse_params.argtypes = [ctypes.c_double, ctypes.c_double, _D, _D, _D, _I, ctypes.c_int,
                                       ctypes.POINTER(Params)]
        L.orc_parse_params.restype = ctypes.c_int
        L.orc_convert_wrf.argtypes = [ctypes.POINTER(WrfGrid), _D, _D, _D, _D, _D, _D, _D, _D, _D, _D]
        _lib = L
    return _lib


def lu_tables():
    L = lib()
    crow = (ctypes.c_int * (NVAR + 1)).in_dll(L, "orc_lu_crow")
    diag = (ctypes.c_int * NVAR).in_dll(L, "orc_lu_diag")
    icol = (ctypes.c_int * NJVS).in_dll(L, "orc_lu_icol")
    return np.array(crow), np.array(diag), np.array(icol)


def rconst(JV, TEMP, FIX, RC_N2O5, nthreads=0):
    n = len(TEMP)
    out = np.empty((n, NREACT))
    JV, TEMP, FIX = _c(JV, (n, NPH)), _c(TEMP, (n,)), _c(FIX, (n, NFIX))
    rcn = _c(RC_N2O5 if RC_N2O5 is not None else np.zeros(n), (n,))
    lib().orc_rconst_batch(n, _dp(JV), _dp(TEMP), _dp(FIX), _dp(rcn), _dp(out), nthreads)
    return out


def fun(V, F, RCT):
    V, F, RCT = _c(V, (NVAR,)), _c(F, (NFIX,)), _c(RCT, (NREACT,))
    out = np.empty(NVAR)
    lib().orc_fun(_dp(V), _dp(F), _dp(RCT), _dp(out))
    return out


def jac(V, F, RCT):
    V, F, RCT = _c(V, (NVAR,)), _c(F, (NFIX,)), _c(RCT, (NREACT,))
    out = np.empty(NJVS)
    lib().orc_jac(_dp(V), _dp(F), _dp(RCT), _dp(out))
    return out


def decomp(G):
    G = _c(G, (NJVS,)).copy()
    s = lib().orc_decomp(_dp(G))
    return G, s


def solve(LU, X):
    LU, X = _c(LU, (NJVS,)), _c(X, (NVAR,)).copy()
    lib().orc_solve(_dp(LU), _dp(X))
    return X


def params(tstart, tend, atol, rtol, rpar, ipar, float_coeffs=1):
    p = Params()
    atol, rtol = _c(atol, (-1,)), _c(rtol, (-1,))
    rpar = _c(rpar, (20,))
    ipar = np.ascontiguousarray(ipar, dtype=np.int32)
    rc = lib().orc_parse_params(tstart, tend, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar), float_coeffs,
                                ctypes.byref(p))
    return rc, p


def integrate(VAR, FIX, RCT, p, nthreads=0):
    """Integrate a batch in place on a copy; returns (VAR_out, stats dict)."""
    n = VAR.shape[0]
    Y = _c(VAR, (n, NVAR)).copy()
    FIX, RCT = _c(FIX, (n, NFIX)), _c(RCT, (n, NREACT))
    st = (CellStats * n)()
    lib().orc_integrate_batch(n, _dp(Y), _dp(FIX), _dp(RCT), ctypes.byref(p), st, nthreads)
    arr = np.ctypeslib.as_array(st)
    stats = {k: np.array(arr[k]) for k, _ in CellStats._fields_}
    return Y, stats


def rosenbrock(tstart, tend, atol, rtol, rpar, ipar, VAR, FIX, RCT, float_coeffs=1, nthreads=0):
    n = VAR.shape[0]
    Y = _c(VAR, (n, NVAR)).copy()
    FIX, RCT = _c(FIX, (n, NFIX)), _c(RCT, (n, NREACT))
    atol, rtol = _c(atol, (-1,)), _c(rtol, (-1,))
    st = (CellStats * n)()
    ierr = lib().orc_rosenbrock(tstart, tend, _dp(atol), _dp(rtol), _dp(rpar), _ip(ipar), n, _dp(Y), _dp(FIX),
                                _dp(RCT), float_coeffs, st, nthreads)
    arr = np.ctypeslib.as_array(st)
    return ierr, Y, {k: np.array(arr[k]) for k, _ in CellStats._fields_}


# ---------------------------------------------------------------- reference harness

_ref = None


def ref_available():
    return os.path.exists(REF_SO)


def ref():
    global _ref
    if _ref is None:
        R = ctypes.CDLL(REF_SO)
        R.ref_rconst.argtypes = [_D, _D, _D, _D, _D]
        R.ref_fun.argtypes = [_D, _D, _D, _D]
        R.ref_jac.argtypes = [_D, _D, _D, _D]
        R.ref_decomp.argtypes = [_D]
        R.ref_decomp.restype = ctypes.c_int
        R.ref_solve.argtypes = [_D, _D]
        R.ref_convert_wrf.argtypes = [_D] * 10
        _ref = R
    return _ref


def ref_rconst(jv, fix, rc_n2o5, temp):
    jv, fix = _c(jv, (NPH,)), _c(fix, (NFIX,))
    rcn, t = np.array([rc_n2o5], dtype=np.float64), np.array([temp], dtype=np.float64)
    out = np.empty(NREACT)
    ref().ref_rconst(_dp(jv), _dp(fix), _dp(rcn), _dp(t), _dp(out))
    return out


def ref_fun(V, F, RCT):
    V, F, RCT = _c(V, (NVAR,)), _c(F, (NFIX,)), _c(RCT, (NREACT,))
    out = np.empty(NVAR)
    ref().ref_fun(_dp(V), _dp(F), _dp(RCT), _dp(out))
    return out


def ref_jac(V, F, RCT):
    V, F, RCT = _c(V, (NVAR,)), _c(F, (NFIX,)), _c(RCT, (NREACT,))
    out = np.empty(NJVS)
    ref().ref_jac(_dp(V), _dp(F), _dp(RCT), _dp(out))
    return out


def ref_decomp(G):
    G = _c(G, (NJVS,)).copy()
    s = ref().ref_decomp(_dp(G))
    return G, s


def ref_solve(LU, X):
    LU, X = _c(LU, (NJVS,)), _c(X, (NVAR,)).copy()
    ref().ref_solve(_dp(LU), _dp(X))
    return X


def ref_convert_wrf(fields):
    """The reference's dev_convert over its own launch (the 48 x 20 x 48 domain only)."""
    g = WrfGrid(*REF_WRF_GRID)
    out = _wrf_outputs(g)
    f = _wrf_fields(fields)
    ref().ref_convert_wrf(*[_dp(a) for a in f], *[_dp(out[k]) for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")])
    return out
