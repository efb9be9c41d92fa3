#!/usr/bin/env python3
"""Emit the role-split code of the cooperative solver kernel (csrc/radm2_coop.cuh).

The cooperative kernel keeps 32 cells per thread block on chip: one cell per lane, and
G warps per block.  Every warp ("role") runs the same lane-per-cell SIMT code, but each
phase of a step attempt is split between the G roles, so a cell's work is spread over G
lanes (one in each warp) and its LU, state and stage vectors stay in shared memory and
registers.  This module decides the split and writes it out as fragments:

  radm2_coop_g<G>_own.inc    species owned by each role (stage vectors, error terms):
                             OWN(k, species) per owned species, k = register slot
  radm2_coop_g<G>_fun.inc    RHS of the owned species, reference association order
                             (mgpu.cu:1103-1385): FUN_OUT(k, species, value)
  radm2_coop_g<G>_jac.inc    Jacobian slots of the role, G = -J (+ ghinv on the diagonal):
                             JAC_OUT / JAC_OUT_DIAG / JAC_OUT_ZERO (mgpu.cu:1685-2652)
  radm2_coop_g<G>_lu.inc     LU rows of the role (row-Doolittle blocks of mgpu.cu:2746-2779),
                             LU_WAIT(row) before a pivot row owned by another role is read,
                             LU_DONE(row) after a finished row is stored
  radm2_coop_g<G>_fwd.inc    forward substitution rows of the role and, after a block
  radm2_coop_g<G>_bwd.inc    barrier, backward rows (mgpu.cu:2873-3090 order); SOLVE_WAIT(row)
                             before another role's row is read, SOLVE_DONE(row) after a store

Each fragment is `switch (COOP_ROLE) { case r: ... }`; the kernel defines the accessor
macros.  Every expression keeps the reference's evaluation order, so each role computes
its share exactly as the single-thread code does.

Row assignment (LU and solves) is list scheduling on a cost model: rows are taken in
elimination order and each goes to the role that would finish it first, counting the
hand-off latency when a pivot row comes from another role.  Species and Jacobian slots
are balanced greedily by operation count, counting recomputed shared subexpressions.

Usage:  python emit_coop.py      (reads radm2_mech.json beside this file)
"""
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import emit  # noqa: E402

ROLE_COUNTS = (4, 8)

# Cost model (SM cycles) for the list scheduler.
C_LOAD = 2        # one shared-memory load issued (32 lanes x 8 B = 2 wavefronts)
C_STORE = 2
C_FMA = 8         # dependent FP64 multiply-add latency
C_DIV = 40        # reciprocal / division
C_HANDOFF = 160   # a row finished by another role: fence, flag, poll, reload

# Scheduling fences (COOP_FENCE) in the RHS: loads of one group of rates may not be hoisted
# above the previous group, which bounds the live set (the kernel runs at 255 registers).
FUN_FENCE_RATES = int(os.environ.get("RADM2_COOP_FUN_FENCE", "16"))


class Refs:
    """Collect the A (rate) or B (partial) references of an expression tree."""

    def __init__(self, arr):
        self.arr = arr

    def __call__(self, t, out=None):
        out = set() if out is None else out
        k = t[0]
        if k == "ref" and t[1] == self.arr:
            out.add(t[2])
        elif k == "bin":
            self(t[2], out)
            self(t[3], out)
        elif k == "neg":
            self(t[1], out)
        elif k == "call":
            for a in t[2]:
                self(a, out)
        return out


def balance(items, cost_own, needs, cost_need, nroles, cap=None):
    """Greedy balance: items (largest own cost first) go to the role with the least load
    after adding the item's own cost plus the shared subexpressions it newly needs there."""
    loads = [0.0] * nroles
    have = [set() for _ in range(nroles)]
    owned = [[] for _ in range(nroles)]
    for it in sorted(items, key=lambda x: (-cost_own[x], x)):
        best, bc = None, None
        for r in range(nroles):
            if cap is not None and len(owned[r]) >= cap:
                continue
            new = needs[it] - have[r]
            c = loads[r] + cost_own[it] + sum(cost_need[n] for n in new)
            if bc is None or c < bc:
                best, bc = r, c
        loads[best] = bc
        have[best] |= needs[it]
        owned[best].append(it)
    return [sorted(o) for o in owned], loads


def schedule_lu(crow, diag, icol, nvar, nroles):
    """Row -> role for the LU: rows in elimination order, each to the role that finishes it
    first.  Returns (owner, per-role finish time, makespan)."""
    owner = [None] * nvar
    ready = [0.0] * nvar
    free = [0.0] * nroles
    for i in range(nvar):
        n = crow[i + 1] - crow[i]
        piv = [icol[s] for s in range(crow[i], diag[i])]
        best = None
        for r in range(nroles):
            t = free[r] + n * C_LOAD
            for j in piv:
                t = max(t, ready[j] + (C_HANDOFF if owner[j] != r else 0))
                nu = crow[j + 1] - diag[j] - 1
                t += C_FMA + nu * (C_LOAD + 1) + C_FMA
            t += C_DIV + n * C_STORE
            if best is None or t < best[0] - 1e-9 or (abs(t - best[0]) < 1e-9 and free[r] < free[best[1]]):
                best = (t, r)
        t, r = best
        owner[i], ready[i], free[r] = r, t, t
    return owner, free, max(ready)


def schedule_solve(crow, diag, icol, nvar, nroles):
    """Rows -> roles for the forward substitution (rows with lower entries; the others keep
    b) and, after a block barrier, the backward substitution (all rows, last row first)."""
    lo = [[icol[s] for s in range(crow[i], diag[i])] for i in range(nvar)]
    up = [[icol[s] for s in range(diag[i] + 1, crow[i + 1])] for i in range(nvar)]

    def run(order, deps, active):
        own = [None] * nvar
        rdy = [0.0] * nvar
        free = [0.0] * nroles
        for i in order:
            if not active(i):
                continue
            best = None
            for r in range(nroles):
                t = free[r]
                for j in deps(i):
                    if active(j):
                        t = max(t, rdy[j] + (C_HANDOFF if own[j] != r else 0))
                    t += C_FMA
                t += C_FMA
                if best is None or t < best[0] - 1e-9:
                    best = (t, r)
            t, r = best
            own[i], rdy[i], free[r] = r, t, t
        return own, max(free)

    own_l, span_l = run(range(nvar), lambda i: lo[i], lambda i: bool(lo[i]))
    own_u, span_u = run(reversed(range(nvar)), lambda i: up[i], lambda i: True)
    return own_l, own_u, span_l, span_u


# ---- operation streams for the table-driven LU and solves
# One 32-bit word per operation: opcode (4 bits) | A (10 bits) | B (10 bits) | C (8 bits).
OPS = {"END": 0, "CHECK": 1, "WAIT": 2, "PIVOT": 3, "UPD": 4, "RCP": 5, "DONE": 6, "ROW": 7, "TERM": 8,
       "STORE": 9, "STORE_DIAG": 10}


def op_word(op, a=0, b=0, c=0):
    assert 0 <= a < 1024 and 0 <= b < 1024 and 0 <= c < 256, (op, a, b, c)
    return (OPS[op] << 28) | (a << 18) | (b << 8) | c


def lu_op_streams(crow, diag, icol, nvar, owner, recip):
    """Per role, the LU of its rows as operation words: CHECK(diag) at a row's start,
    WAIT(row) before the first pivot on a row another role owns, PIVOT(slot i,j; diag j;
    n) followed by n UPD(slot i,k; slot j,k), RCP(diag) (reciprocal form), DONE(row).  The
    same operations in the same order per slot as the unrolled row blocks."""
    nroles = max(owner) + 1
    streams = [[] for _ in range(nroles)]
    for ro in range(nroles):
        waited = set()
        out = streams[ro]
        for i in range(nvar):
            if owner[i] != ro:
                continue
            out.append(op_word("CHECK", diag[i]))
            col_slot = {icol[sl]: sl for sl in range(crow[i], crow[i + 1])}
            for kk in range(crow[i], diag[i]):
                j = icol[kk]
                if owner[j] != ro and j not in waited:
                    if recip or crow[j] != diag[j]:
                        out.append(op_word("WAIT", c=j))
                    waited.add(j)
                ups = list(range(diag[j] + 1, crow[j + 1]))
                out.append(op_word("PIVOT", kk, diag[j], len(ups)))
                for jj in ups:
                    out.append(op_word("UPD", col_slot[icol[jj]], jj))
            if recip:
                out.append(op_word("RCP", diag[i]))
            out.append(op_word("DONE", c=i))
        out.append(op_word("END"))
    return streams


def solve_op_streams(crow, diag, icol, nvar, own_l, own_u, recip):
    """Per role, the forward rows (ROW(k, n), n TERM(slot, j), STORE(k), DONE(k)) and, as a
    separate stream, the backward rows (... STORE_DIAG(k, diag k) ...), with WAIT(row) before
    another role's row is read.  Each row's terms in the unrolled order."""
    nroles = max(o for o in own_u if o is not None) + 1
    fwd = [[] for _ in range(nroles)]
    bwd = [[] for _ in range(nroles)]
    lo = [[s for s in range(crow[i], diag[i])] for i in range(nvar)]
    for ro in range(nroles):
        waited = set()
        out = fwd[ro]
        for k in range(nvar):
            if own_l[k] != ro:
                continue
            for s in lo[k]:
                j = icol[s]
                if lo[j] and own_l[j] != ro and j not in waited:
                    out.append(op_word("WAIT", c=j))
                    waited.add(j)
            out.append(op_word("ROW", k, 0, len(lo[k])))
            for s in lo[k]:
                out.append(op_word("TERM", s, icol[s]))
            out.append(op_word("STORE", k))
            out.append(op_word("DONE", c=k))
        out.append(op_word("END"))
        waited = set()
        out = bwd[ro]
        for k in reversed(range(nvar)):
            if own_u[k] != ro:
                continue
            ups = list(range(diag[k] + 1, crow[k + 1]))
            for s in ups:
                j = icol[s]
                if own_u[j] != ro and j not in waited:
                    out.append(op_word("WAIT", c=j))
                    waited.add(j)
            out.append(op_word("ROW", k, 0, len(ups)))
            for s in ups:
                out.append(op_word("TERM", s, icol[s]))
            out.append(op_word("STORE_DIAG", k, diag[k]))
            out.append(op_word("DONE", c=k))
        out.append(op_word("END"))
    return fwd, bwd


def flat(streams):
    """Concatenated words and the start of every role's stream."""
    words, starts = [], []
    for st in streams:
        starts.append(len(words))
        words.extend(st)
    return words, starts


def kref(arr, i):
    return {"RCT": "RC(%d)", "V": "V(%d)", "F": "FIX(%d)", "A": "a%d", "B": "b%d"}[arr] % i


def emit_role_code(m, G, out_dir):
    r = emit.Renderer(kref, emit.kernel_var)
    sz = m["sizes"]
    nvar = sz["NVAR"]
    lu = m["lu"]
    crow, diag, icol = lu["crow"], lu["diag"], lu["icol"]
    dset = set(diag)
    banner = emit.BANNER
    notes = []

    # ---- species: RHS sums (and the stage vectors of the same species)
    arefs = Refs("A")
    needs = {i: arefs(t) for i, t in enumerate(m["vdot"])}
    cost_own = {i: emit.count_flops(t) for i, t in enumerate(m["vdot"])}
    cost_a = {rx: max(1, emit.count_flops(t)) for rx, t in enumerate(m["rates"])}
    cap = -(-nvar // G) + 2
    own, loads = balance(range(nvar), cost_own, needs, cost_a, G, cap=cap)
    ns = max(len(o) for o in own)
    notes.append("species per role %s, RHS ops per role %s" % ([len(o) for o in own], [int(x) for x in loads]))

    body = [banner, "/* Species owned by each of %d roles: OWN(k, species), k = the role's slot. */\n" % G,
            "switch (COOP_ROLE) {\n"]
    for ro in range(G):
        body.append("case %d:\n" % ro)
        body.append("".join("  OWN(%d, %d)\n" % (k, s) for k, s in enumerate(own[ro])))
        body.append("  break;\n")
    body.append("default: break;\n}\n")
    emit.write(os.path.join(out_dir, "radm2_coop_g%d_own.inc" % G), body)

    # RHS, reaction-major per role: each rate is formed once and added into the accumulators
    # of the role's species that use it.  Every reference sum lists its reactions in
    # increasing order, so each accumulator sees the same operations in the same order as
    # the reference's left-to-right sum (bit-identical), and only the role's accumulators
    # stay live.
    chains = []
    for t in m["vdot"]:
        chain, node = [], t
        while node[0] == "bin" and node[1] in "+-":
            chain.append((node[1], node[3]))
            node = node[2]
        chain.append((None, node))
        chain.reverse()
        chains.append(chain)
    uses = {}
    for i, chain in enumerate(chains):
        for pos, (op, term) in enumerate(chain):
            rs = arefs(term)
            assert len(rs) == 1, (i, term)
            uses.setdefault(rs.pop(), []).append((i, pos, op, term))
    body = [banner, "/* RHS of each role's species, mgpu.cu:1103-1385, reaction-major (bit-identical to the\n"
            " * reference's sums).  Inputs: RC(r), V(i), FIX(k).  Output FUN_OUT(k, species, value) for owned\n"
            " * slot k. */\n",
            "switch (COOP_ROLE) {\n"]
    for ro in range(G):
        body.append("case %d: {\n" % ro)
        slot = {s_: k for k, s_ in enumerate(own[ro])}
        for s_ in own[ro]:
            body.append("  double vd%d;\n" % s_)
        nrx = 0
        for rx, t in enumerate(m["rates"]):
            mine = [u for u in uses.get(rx, []) if u[0] in slot]
            if not mine:
                continue
            if nrx and nrx % FUN_FENCE_RATES == 0:
                body.append("  COOP_FENCE;\n")
            nrx += 1
            body.append("  { const double a%d = %s;\n" % (rx, r(t)))
            for (i, pos, op, term) in mine:
                if pos == 0:
                    body.append("    vd%d = %s;\n" % (i, r(term)))
                else:
                    body.append("    vd%d = (vd%d %s %s);\n" % (i, i, op, r(term)))
            body.append("  }\n")
        for s_ in own[ro]:
            body.append("  FUN_OUT(%d, %d, vd%d);\n" % (slot[s_], s_, s_))
        body.append("} break;\n")
    body.append("default: break;\n}\n")
    emit.write(os.path.join(out_dir, "radm2_coop_g%d_fun.inc" % G), body)

    # ---- Jacobian slots
    brefs = Refs("B")
    slots = list(range(len(m["jvs"])))
    jneeds = {s: brefs(t) for s, t in enumerate(m["jvs"])}
    jcost = {s: emit.count_flops(t) + 1 for s, t in enumerate(m["jvs"])}
    bcost = {int(k): max(1, emit.count_flops(t)) for k, t in m["bvals"].items()}
    jown, jloads = balance(slots, jcost, jneeds, bcost, G)
    notes.append("Jacobian slots per role %s, ops %s" % ([len(o) for o in jown], [int(x) for x in jloads]))
    body = [banner, "/* Jacobian slots of each role, G = -J (+ ghinv on the diagonal), mgpu.cu:1685-2652\n"
            " * expressions.  Inputs: RC(r), V(i), FIX(k). */\n", "switch (COOP_ROLE) {\n"]
    for ro in range(G):
        body.append("case %d: {\n" % ro)
        need = sorted(set().union(*[jneeds[s] for s in jown[ro]])) if jown[ro] else []
        for b in need:
            body.append("  const double b%d = %s;\n" % (b, r(m["bvals"][str(b)])))
        for s in jown[ro]:
            t = m["jvs"][s]
            if emit.is_zero(t):
                body.append("  JAC_OUT_ZERO(%d, %d);\n" % (s, 1 if s in dset else 0))
            else:
                body.append("  %s(%d, %s);\n" % ("JAC_OUT_DIAG" if s in dset else "JAC_OUT", s, r(t)))
        body.append("} break;\n")
    body.append("default: break;\n}\n")
    emit.write(os.path.join(out_dir, "radm2_coop_g%d_jac.inc" % G), body)

    # ---- LU rows
    lu_owner, lu_free, lu_span = schedule_lu(crow, diag, icol, nvar, G)
    notes.append("LU rows per role %s, modelled makespan %d cycles" % (
        [lu_owner.count(ro) for ro in range(G)], int(lu_span)))
    for recip in (True, False):
        sfx = "" if recip else "_div"
        body = [banner, "/* LU rows of each role, the row-by-row elimination of mgpu.cu:2746-2779 (same blocks\n"
                " * as the single-thread form).  LU_WAIT(j) before row j's entries are read when another\n"
                " * role owns row j; LU_DONE(i) after row i is stored.  LU_PIVOT_CHECK(row, diag).%s */\n"
                % ("  Diagonal slots hold reciprocals on exit." if recip else ""), "switch (COOP_ROLE) {\n"]
        for ro in range(G):
            body.append("case %d: {\n" % ro)
            waited = set()
            for k in range(nvar):
                if lu_owner[k] != ro:
                    continue
                body.append("{ /* row %d */\n" % k)
                body.append("  LU_PIVOT_CHECK(%d, G(%d));\n" % (k, diag[k]))
                if crow[k] == diag[k]:
                    if recip:
                        body.append("  G(%d) = (LU_T)1 / G(%d);\n" % (diag[k], diag[k]))
                    body.append("  LU_DONE(%d);\n}\n" % k)
                    continue
                for sl in range(crow[k], crow[k + 1]):
                    body.append("  LU_T w%d = G(%d);\n" % (icol[sl], sl))
                for kk in range(crow[k], diag[k]):
                    j = icol[kk]
                    if lu_owner[j] != ro and j not in waited:
                        # rows with no elimination and no reciprocal are final from the start
                        if recip or crow[j] != diag[j]:
                            body.append("  LU_WAIT(%d);\n" % j)
                        waited.add(j)
                    if recip:
                        body.append("  { const LU_T a = -w%d * G(%d); w%d = -a;\n" % (j, diag[j], j))
                    else:
                        body.append("  { const LU_T a = -w%d / G(%d); w%d = -a;\n" % (j, diag[j], j))
                    for jj in range(diag[j] + 1, crow[j + 1]):
                        body.append("    w%d += a * G(%d);\n" % (icol[jj], jj))
                    body.append("  }\n")
                for sl in range(crow[k], crow[k + 1]):
                    if recip and sl == diag[k]:
                        body.append("  G(%d) = (LU_T)1 / w%d;\n" % (sl, icol[sl]))
                    else:
                        body.append("  G(%d) = w%d;\n" % (sl, icol[sl]))
                body.append("  LU_DONE(%d);\n}\n" % k)
            body.append("} break;\n")
        body.append("default: break;\n}\n")
        emit.write(os.path.join(out_dir, "radm2_coop_g%d_lu%s.inc" % (G, sfx)), body)

    # ---- triangular solves: forward rows, a block barrier, backward rows
    own_l, own_u, span_l, span_u = schedule_solve(crow, diag, icol, nvar, G)
    notes.append("solve rows per role: forward %s backward %s, modelled %d + %d cycles" % (
        [own_l.count(ro) for ro in range(G)], [own_u.count(ro) for ro in range(G)], int(span_l), int(span_u)))
    lo = [[s for s in range(crow[i], diag[i])] for i in range(nvar)]
    body = [banner, "/* Forward substitution rows of each role (unit lower factor), mgpu.cu:2873-3090 order,\n"
            " * in place on X(i).  SOLVE_WAIT(j) before X(j) of another role's row is read,\n"
            " * SOLVE_DONE(i) after X(i) is stored.  Rows without lower entries keep b. */\n",
            "switch (COOP_ROLE) {\n"]
    for ro in range(G):
        body.append("case %d: {\n" % ro)
        waited = set()
        for k in range(nvar):
            if own_l[k] != ro:
                continue
            for s in lo[k]:
                j = icol[s]
                if lo[j] and own_l[j] != ro and j not in waited:
                    body.append("  SOLVE_WAIT(%d);\n" % j)
                    waited.add(j)
            expr = "X(%d)" % k
            for s in lo[k]:
                expr = "(%s - G(%d) * X(%d))" % (expr, s, icol[s])
            body.append("  X(%d) = %s;\n  SOLVE_DONE(%d);\n" % (k, expr, k))
        body.append("} break;\n")
    body.append("default: break;\n}\n")
    emit.write(os.path.join(out_dir, "radm2_coop_g%d_fwd.inc" % G), body)
    for recip in (True, False):
        sfx = "" if recip else "_div"
        body = [banner, "/* Backward substitution rows of each role (upper factor), mgpu.cu:2873-3090 order, in\n"
                " * place on X(i), after every forward row is final.  SOLVE_WAIT(j) before X(j) of another\n"
                " * role's row is read, SOLVE_DONE(i) after X(i) is stored.%s */\n"
                % ("  Diagonal slots hold reciprocals." if recip else ""), "switch (COOP_ROLE) {\n"]
        for ro in range(G):
            body.append("case %d: {\n" % ro)
            waited = set()
            for k in reversed(range(nvar)):
                if own_u[k] != ro:
                    continue
                for s in range(diag[k] + 1, crow[k + 1]):
                    j = icol[s]
                    if own_u[j] != ro and j not in waited:
                        body.append("  SOLVE_WAIT(%d);\n" % j)
                        waited.add(j)
                expr = "X(%d)" % k
                for s in range(diag[k] + 1, crow[k + 1]):
                    expr = "(%s - G(%d) * X(%d))" % (expr, s, icol[s])
                body.append("  X(%d) = %s %s G(%d);\n  SOLVE_DONE(%d);\n" % (
                    k, expr, "*" if recip else "/", diag[k], k))
            body.append("} break;\n")
        body.append("default: break;\n}\n")
        emit.write(os.path.join(out_dir, "radm2_coop_g%d_bwd%s.inc" % (G, sfx)), body)

    # ---- operation streams of the table-driven LU and solves
    tabs = []
    for name, streams in (("lu", lu_op_streams(crow, diag, icol, nvar, lu_owner, True)),
                          ("lu_div", lu_op_streams(crow, diag, icol, nvar, lu_owner, False))):
        w, st = flat(streams)
        tabs.append((name, w, st))
    for recip in (True, False):
        fwd, bwd = solve_op_streams(crow, diag, icol, nvar, own_l, own_u, recip)
        if recip:
            w, st = flat(fwd)
            tabs.append(("fwd", w, st))
        w, st = flat(bwd)
        tabs.append(("bwd" if recip else "bwd_div", w, st))
    body = [banner, "/* Operation streams of the table-driven LU and triangular solves, %d roles: per\n"
            " * stream, the words of every role back to back and each role's first word.  Word:\n"
            " * opcode << 28 | A << 18 | B << 8 | C (see radm2_coop.cuh). */\n" % G]
    for name, w, st in tabs:
        body.append("static __device__ const unsigned coop_%s_ops[%d] = {%s};\n" % (
            name, len(w), ",".join("0x%08xu" % x for x in w)))
        body.append("static __device__ const int coop_%s_start[%d] = {%s};\n" % (name, len(st), ",".join(map(str, st))))
    emit.write(os.path.join(out_dir, "radm2_coop_g%d_ops.h" % G), body)
    notes.append("operation words: " + ", ".join("%s %d" % (n, len(w)) for n, w, _ in tabs))

    h = [banner, "#pragma once\n/* Cooperative kernel with %d roles: %s. */\n" % (G, "; ".join(notes)),
         "#define RADM2_COOP_G%d_NS %d  /* most species owned by one role */\n" % (G, ns)]
    emit.write(os.path.join(out_dir, "radm2_coop_g%d.h" % G), h)
    return notes


def main():
    m = emit.load()
    for G in ROLE_COUNTS:
        notes = emit_role_code(m, G, emit.CSRC_GEN)
        print("G=%d:" % G, "; ".join(notes))


if __name__ == "__main__":
    main()
