"""The operation streams of the cooperative kernel's table-driven LU and triangular solves
(mech/emit_coop.py), run on the CPU by a small interpreter with the kernel's semantics:
every role executes its stream in order and a WAIT blocks until the named row is DONE.
In the division form the result must equal the oracle's LU and solve (the row-by-row order
of mgpu.cu:2746-2779 and 2873-3090) bit for bit, for every role count built; the reciprocal
form within rounding of it."""
import os
import sys

import numpy as np
import pytest

import oracle
from conftest import PKG
from radm2b200 import inputs

sys.path.insert(0, os.path.join(PKG, "mech"))
import emit  # noqa: E402
import emit_coop  # noqa: E402

OP = {v: k for k, v in emit_coop.OPS.items()}


def decode(w):
    return OP[w >> 28], (w >> 18) & 1023, (w >> 8) & 1023, w & 255


def run_streams(streams, G, X=None, recip=True):
    """Execute role streams round-robin; G (LU slots) and X are updated in place."""
    pos = [0] * len(streams)
    done = set()
    sing = []
    finished = [False] * len(streams)
    while not all(finished):
        progressed = False
        for r, st in enumerate(streams):
            while not finished[r]:
                op, a, b, c = decode(st[pos[r]])
                if op == "WAIT":
                    if c not in done:
                        break
                    pos[r] += 1
                elif op == "END":
                    finished[r] = True
                elif op == "CHECK":
                    if G[a] == 0.0:
                        sing.append(a)
                    pos[r] += 1
                elif op == "PIVOT":
                    av = -G[a] * G[b] if recip else -G[a] / G[b]
                    G[a] = -av
                    for q in range(1, c + 1):
                        op2, s_ik, s_jk, _ = decode(st[pos[r] + q])
                        assert op2 == "UPD"
                        G[s_ik] = G[s_ik] + av * G[s_jk]
                    pos[r] += c + 1
                elif op == "RCP":
                    G[a] = 1.0 / G[a]
                    pos[r] += 1
                elif op == "DONE":
                    done.add(c)
                    pos[r] += 1
                elif op == "ROW":
                    acc = X[a]
                    for q in range(1, c + 1):
                        op2, s, j, _ = decode(st[pos[r] + q])
                        assert op2 == "TERM"
                        acc = acc - G[s] * X[j]
                    op3, k, d, _ = decode(st[pos[r] + c + 1])
                    if op3 == "STORE":
                        X[k] = acc
                    else:
                        assert op3 == "STORE_DIAG"
                        X[k] = acc * G[d] if recip else acc / G[d]
                    pos[r] += c + 2
                else:
                    raise AssertionError(op)
                progressed = True
        assert progressed or all(finished), "streams deadlock"
    return sing


def matrices(n):
    """Prepared matrices G = -J + I/(h gamma) of seeded mixed-regime cells, and right-hand sides."""
    cells = inputs.make_cells(n, 31, "mixed")
    rc = oracle.rconst(cells["JV"], cells["TEMP"], cells["FIX"], cells["RC_N2O5"])
    _, diag, _ = oracle.lu_tables()
    out = []
    rng = np.random.default_rng(5)
    for c in range(n):
        J = oracle.jac(cells["VAR"][c], cells["FIX"][c], rc[c])
        G = -J
        for d in diag:
            G[d] += 1.0 / (10.0 * 0.43586652150845899941601945119356)
        out.append((G, rng.normal(size=59)))
    return out


@pytest.mark.parametrize("nroles", emit_coop.ROLE_COUNTS)
def test_streams_equal_the_oracle(nroles):
    m = emit.load()
    lu = m["lu"]
    crow, diag, icol, nvar = lu["crow"], lu["diag"], lu["icol"], m["sizes"]["NVAR"]
    owner, _, _ = emit_coop.schedule_lu(crow, diag, icol, nvar, nroles)
    own_l, own_u, _, _ = emit_coop.schedule_solve(crow, diag, icol, nvar, nroles)
    for G0, b in matrices(6):
        # division form: the oracle's arithmetic, bit for bit
        G = G0.copy()
        assert run_streams(emit_coop.lu_op_streams(crow, diag, icol, nvar, owner, False), G, recip=False) == []
        Go, sing = oracle.decomp(G0)
        assert sing == 0
        assert np.array_equal(G, Go)
        fwd, bwd = emit_coop.solve_op_streams(crow, diag, icol, nvar, own_l, own_u, False)
        X = b.copy()
        run_streams(fwd, G, X, recip=False)
        run_streams(bwd, G, X, recip=False)
        assert np.array_equal(X, oracle.solve(Go, b))
        # reciprocal form: one rounding per pivot use away
        Gr = G0.copy()
        run_streams(emit_coop.lu_op_streams(crow, diag, icol, nvar, owner, True), Gr, recip=True)
        fwd, bwd = emit_coop.solve_op_streams(crow, diag, icol, nvar, own_l, own_u, True)
        Xr = b.copy()
        run_streams(fwd, Gr, Xr, recip=True)
        run_streams(bwd, Gr, Xr, recip=True)
        assert np.allclose(Xr, X, rtol=1e-9, atol=0)


def test_every_wait_names_a_row_the_phase_finishes():
    """A WAIT in a stream names a row some role of the same phase marks DONE (no wait can
    stall until the time limit)."""
    m = emit.load()
    lu = m["lu"]
    crow, diag, icol, nvar = lu["crow"], lu["diag"], lu["icol"], m["sizes"]["NVAR"]
    for nroles in emit_coop.ROLE_COUNTS:
        owner, _, _ = emit_coop.schedule_lu(crow, diag, icol, nvar, nroles)
        own_l, own_u, _, _ = emit_coop.schedule_solve(crow, diag, icol, nvar, nroles)
        fwd, bwd = emit_coop.solve_op_streams(crow, diag, icol, nvar, own_l, own_u, True)
        for streams in (emit_coop.lu_op_streams(crow, diag, icol, nvar, owner, True), fwd, bwd):
            done = {decode(w)[3] for st in streams for w in st if decode(w)[0] == "DONE"}
            waits = {decode(w)[3] for st in streams for w in st if decode(w)[0] == "WAIT"}
            assert waits <= done
