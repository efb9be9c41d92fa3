"""The oracle against the reference's own code.

Two pins, both bit-for-bit:
  * the committed golden vectors in tests/golden/ref_mechanism.npz, produced by the
    reference's own dev_Update_RCONST / dev_Fun / dev_Jac_SP / dev_KppDecomp /
    dev_KppSolve compiled for the CPU (tests/golden/make_golden.py);
  * the live reference harness (oracle/_ref), where it was built.
"""
import os

import numpy as np
import pytest

import oracle
from conftest import ROOT

GOLDEN = os.path.join(ROOT, "tests", "golden", "ref_mechanism.npz")


def test_golden_vectors_bitwise():
    g = np.load(GOLDEN)
    n = g["VAR"].shape[0]
    rc = oracle.rconst(g["JV"], g["TEMP"], g["FIX"], g["RC_N2O5"])
    assert np.array_equal(rc, g["RCONST"])
    for c in range(n):
        V, F = g["VAR"][c], g["FIX"][c]
        assert np.array_equal(oracle.fun(V, F, rc[c]), g["VDOT"][c])
        J = oracle.jac(V, F, rc[c])
        assert np.array_equal(J, g["JVS"][c])
        LU, s = oracle.decomp(g["G"][c])
        assert s == 0 and np.array_equal(LU, g["LU"][c])
        assert np.array_equal(oracle.solve(LU, g["B"][c]), g["X"][c])


@pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built here")
def test_live_reference_harness_bitwise(cells4k):
    crow, diag, icol = oracle.lu_tables()
    idx = np.arange(0, 4096, 37)
    for c in idx:
        jv, fix, V = cells4k["JV"][c], cells4k["FIX"][c], cells4k["VAR"][c]
        r = oracle.ref_rconst(jv, fix, cells4k["RC_N2O5"][c], cells4k["TEMP"][c])
        assert np.array_equal(r, oracle.rconst(jv[None], cells4k["TEMP"][c:c + 1], fix[None],
                                               cells4k["RC_N2O5"][c:c + 1])[0])
        assert np.array_equal(oracle.ref_fun(V, fix, r), oracle.fun(V, fix, r))
        J = oracle.ref_jac(V, fix, r)
        assert np.array_equal(J, oracle.jac(V, fix, r))
        G = -J
        G[diag] += 1.0 / (37.0 * 0.43586652150845899941601945119356)
        L1, s1 = oracle.ref_decomp(G)
        L2, s2 = oracle.decomp(G)
        assert s1 == s2 == 0 and np.array_equal(L1, L2)
        b = oracle.fun(V, fix, r)
        assert np.array_equal(oracle.ref_solve(L1, b), oracle.solve(L2, b))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference harness not built here")
def test_zero_pivot_code_matches_reference():
    crow, diag, icol = oracle.lu_tables()
    G = np.random.default_rng(5).uniform(0.1, 1.0, 659)
    G[diag[17]] = 0.0
    _, s1 = oracle.ref_decomp(G)
    _, s2 = oracle.decomp(G)
    assert s1 == s2 == 18
