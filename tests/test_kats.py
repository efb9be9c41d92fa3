"""Known-answer tests of the method's building blocks, on the CPU oracle:
the LU pattern reconstructs its matrix and its solve inverts it, the sparse Jacobian agrees
with central differences of the RHS (except the two slots where the reference's Jacobian
keeps a term its RHS drops), and the ROS-3 coefficient set has order 3 (embedded 2) and is
L-stable on y' = lambda y."""
import json
import os

import numpy as np
import pytest

import oracle
from conftest import PKG
from radm2b200 import inputs

MECH = json.load(open(os.path.join(PKG, "mech", "radm2_mech.json")))
QUIRK_SLOTS = (49, 51)  # H2O2 row: the reference Jacobian keeps the H2O2 + OH term its RHS drops


def _dense(vals, crow, icol):
    n = len(crow) - 1
    A = np.zeros((n, n))
    for r in range(n):
        for s in range(crow[r], crow[r + 1]):
            A[r, icol[s]] = vals[s]
    return A


@pytest.fixture(scope="module")
def cell():
    c = inputs.make_cells(4, 17, "mixed")
    rc = oracle.rconst(c["JV"], c["TEMP"], c["FIX"], c["RC_N2O5"])
    return c["VAR"][1], c["FIX"][1], rc[1]


def test_lu_reconstructs_matrix_and_solve_inverts_it(cell):
    V, F, RC = cell
    crow, diag, icol = oracle.lu_tables()
    J = oracle.jac(V, F, RC)
    G = -J
    G[diag] += 1.0 / (0.43586652150845899941601945119356 * 30.0)  # (hγ)^-1 for h = 30 s
    LU, sing = oracle.decomp(G)
    assert sing == 0
    A = _dense(LU, crow, icol)
    L = np.tril(A, -1) + np.eye(len(diag))
    U = np.triu(A)
    Gd = _dense(G, crow, icol)
    assert np.abs(L @ U - Gd).max() <= 1e-12 * np.abs(Gd).max()
    x = np.random.default_rng(2).normal(size=len(diag)) * (1.0 + np.abs(V))
    b = Gd @ x
    got = oracle.solve(LU, b)
    assert np.abs(got - x).max() <= 1e-9 * np.abs(x).max()


def test_jacobian_matches_central_differences(cell):
    """Mass-action rates are at most quadratic in each species, so central differences are
    exact up to rounding; the bound is rounding noise, from the row's term magnitudes."""
    V, F, RC = cell
    crow, diag, icol = oracle.lu_tables()
    irow = np.repeat(np.arange(len(diag)), np.diff(crow))
    J = oracle.jac(V, F, RC)
    row_terms = np.zeros(len(diag))  # sum_k |J_rk V_k| ~ magnitude of row r's RHS terms
    np.add.at(row_terms, irow, np.abs(J) * np.abs(V[icol]))
    fd, bound = np.zeros_like(J), np.zeros_like(J)
    for j in range(len(V)):
        h = 1e-2 * max(abs(V[j]), 1.0)
        vp, vm = V.copy(), V.copy()
        vp[j] += h
        vm[j] -= h
        col = (oracle.fun(vp, F, RC) - oracle.fun(vm, F, RC)) / (2 * h)
        for s_ in np.where(icol == j)[0]:
            fd[s_] = col[irow[s_]]
            bound[s_] = 1e-9 * abs(J[s_]) + 1e-13 * row_terms[irow[s_]] / h
    bad = np.abs(J - fd) > bound
    bad[list(QUIRK_SLOTS)] = False
    assert not bad.any(), [(int(s_), J[s_], fd[s_]) for s_ in np.where(bad)[0][:5]]
    # the two quirk slots differ by more than rounding: the term the RHS drops
    assert all(abs(J[s_] - fd[s_]) > 1e3 * bound[s_] for s_ in QUIRK_SLOTS)


def _ros3_step(z):
    """One ROS-3 step of y' = lambda*y from y = 1 with h*lambda = z, in the stage form the
    solver uses (KPP: (1/(h g) - lambda) K_s = f(Y + sum a K) + sum (c/h) K, NewF)."""
    r = MECH["ros3"]
    A, C, M, E = (np.array([float(x) for x in r[k]]) for k in ("ros_A", "ros_C", "ros_M", "ros_E"))
    g = float(r["ros_Gamma"][0])
    newf = r["ros_NewF"]
    h, lam = 1.0, z  # h = 1 without loss of generality
    K = []
    fval = None
    for s in range(3):
        if s == 0 or newf[s]:
            y = 1.0 + sum(A[s * (s - 1) // 2 + j] * K[j] for j in range(s))
            fval = lam * y
        rhs = fval + sum(C[s * (s - 1) // 2 + j] / h * K[j] for j in range(s))
        K.append(rhs / (1.0 / (h * g) - lam))
    return 1.0 + sum(M[s] * K[s] for s in range(3)), sum(E[s] * K[s] for s in range(3))


def test_ros3_order_and_embedded_order():
    zs = [-0.1, -0.05, -0.025, -0.0125, -0.00625]
    errs = [abs(_ros3_step(z)[0] - np.exp(z)) for z in zs]
    ests = [abs(_ros3_step(z)[1]) for z in zs]
    # local error O(z^4) (order 3): halving z divides it by ~16; error estimate O(z^3): ~8
    for a, b in zip(errs, errs[1:]):
        assert 14.0 < a / b < 18.0, errs
    for a, b in zip(ests, ests[1:]):
        assert 7.0 < a / b < 9.0, ests


def test_ros3_is_l_stable():
    for z in (-1e3, -1e6, -1e9):
        y, _ = _ros3_step(z)
        assert abs(y) < 10.0 / abs(z) ** 0.5 + 1e-6, (z, y)
    for z in (-0.5, -2.0, -10.0, -100.0):
        assert abs(_ros3_step(z)[0]) < 1.0
