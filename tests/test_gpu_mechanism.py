"""GPU mechanism kernels through the C ABI against the oracle.

The mirror kernels behind radm2_fun / radm2_jac / radm2_decomp_solve are compiled
without FMA contraction, so they must agree with the oracle bit for bit; the rate
constants use the device exp/pow/log10 and agree to a few ulp.
"""
import numpy as np
import pytest

import oracle
import radm2b200
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def solver():
    with radm2b200.Solver() as s:
        yield s


@pytest.fixture(scope="module")
def batch(cells4k):
    idx = np.arange(0, 4096, 16)
    c = {k: cells4k[k][idx] for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")}
    c["RCT"] = oracle.rconst(c["JV"], c["TEMP"], c["FIX"], c["RC_N2O5"])
    return c


def test_rconst(solver, cells4k):
    solver.set_cells(cells4k)
    solver.update_rconst()
    g = solver.get_rconst()
    o = oracle.rconst(cells4k["JV"], cells4k["TEMP"], cells4k["FIX"], cells4k["RC_N2O5"])
    nz = o != 0
    assert np.array_equal(g == 0, ~nz)
    assert (np.abs(g[nz] - o[nz]) / np.abs(o[nz])).max() < 1e-13


def test_fun_bitwise(solver, batch):
    g = solver.fun(batch["VAR"], batch["FIX"], batch["RCT"])
    for c in range(len(g)):
        assert np.array_equal(g[c], oracle.fun(batch["VAR"][c], batch["FIX"][c], batch["RCT"][c])), c


def test_jac_bitwise(solver, batch):
    g = solver.jac(batch["VAR"], batch["FIX"], batch["RCT"])
    for c in range(len(g)):
        assert np.array_equal(g[c], oracle.jac(batch["VAR"][c], batch["FIX"][c], batch["RCT"][c])), c


def _systems(batch, h=6.0):
    crow, diag, icol = oracle.lu_tables()
    n = len(batch["VAR"])
    G = np.empty((n, 659))
    B = np.empty((n, 59))
    for c in range(n):
        J = oracle.jac(batch["VAR"][c], batch["FIX"][c], batch["RCT"][c])
        G[c] = -J
        G[c, diag] += 1.0 / (h * 0.43586652150845899941601945119356)
        B[c] = oracle.fun(batch["VAR"][c], batch["FIX"][c], batch["RCT"][c])
    return G, B


def test_decomp_solve_fp64_bitwise(solver, batch):
    G, B = _systems(batch)
    LU, X, sing = solver.decomp_solve(G, B)
    assert not sing.any()
    for c in range(len(G)):
        lu, s = oracle.decomp(G[c])
        assert s == 0
        assert np.array_equal(LU[c], lu), c
        assert np.array_equal(X[c], oracle.solve(lu, B[c])), c


def _matvec(G, X):
    """G @ X for matrices in LU slot order (row-major CSR with the oracle's tables)."""
    crow, diag, icol = oracle.lu_tables()
    rows = np.repeat(np.arange(59), np.diff(crow))
    out = np.zeros_like(X)
    np.add.at(out.T, rows, (G * X[:, icol]).T)
    return out


def test_decomp_solve_fp32_refines(solver, batch):
    """The float factorisation is a good preconditioner: one FP64-residual refinement
    sweep, x1 = x0 + LU32^-1 (b - G x0), shrinks the error by orders of magnitude."""
    G, B = _systems(batch)
    _, X0, sing = solver.decomp_solve(G, B, precision=radm2b200.PREC_FP32LU)
    _, X64, _ = solver.decomp_solve(G, B)
    assert not sing.any()
    R = B - _matvec(G, X0)
    _, D, _ = solver.decomp_solve(G, R, precision=radm2b200.PREC_FP32LU)
    X1 = X0 + D
    e0 = np.abs(X0 - X64).max(axis=1) / np.abs(X64).max(axis=1)
    e1 = np.abs(X1 - X64).max(axis=1) / np.abs(X64).max(axis=1)
    assert np.median(e0) < 1e-2
    assert np.median(e1) < 1e-3 * np.median(e0) and (e1 <= e0).mean() > 0.95


def test_zero_pivot_reported(solver, batch):
    crow, diag, icol = oracle.lu_tables()
    G, B = _systems(batch)
    G = G[:4].copy()
    G[1, diag[30]] = 0.0
    _, _, sing = solver.decomp_solve(G, B[:4])
    assert list(sing) == [0, 31, 0, 0]
