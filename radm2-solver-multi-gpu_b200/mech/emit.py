#!/usr/bin/env python3
"""Emit C / CUDA code for the RADM2 mechanism from mech/radm2_mech.json.

Two consumers, one mechanism table:

  csrc/gen/   fragments for the sm_100a kernels.  Each fragment is the body of
              a device function and talks to its caller only through accessor
              macros (V(i), RC(r), FIX(k), G(s), X(i), ...), so one fragment
              serves the FP64 kernel, the FP32-LU kernel and the test kernels,
              each with its own storage (registers, shared or global SoA).
              The LU decomposition and the solves are fully unrolled to the
              659-slot fill pattern.

  oracle/gen/ plain C functions for the CPU oracle (rates, RHS, Jacobian) and
              the CSR tables its table-driven LU / solve loops walk.

Expressions are rendered fully parenthesised from the parse trees, so both
sides evaluate every rate, RHS sum and Jacobian slot in the reference's own
association order (mgpu.cu:763-918, 1103-1385, 1685-2652).

Usage:  python emit.py      (reads radm2_mech.json beside this file)
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
REPO = os.path.dirname(PKG)
CSRC_GEN = os.path.join(PKG, "csrc", "gen")
ORACLE_GEN = os.path.join(REPO, "oracle", "gen")

BANNER = ("/* Generated by radm2-solver-multi-gpu_b200/mech/emit.py from mech/radm2_mech.json\n"
          " * (the RADM2 mechanism as encoded in the reference's mgpu.cu).  Do not edit. */\n")

# Rate-law helpers: reference name -> this project's implementation name.
CALLS = {"ARR2": "rk_arr2", "TROE": "rk_troe", "TROEE": "rk_troee",
         "THERMAL_T2": "rk_thermal_t2", "k46": "rk_k46", "pow": "pow", "exp": "exp"}


def lit(text):
    """Render a numeric literal as a C double literal with the same value."""
    if all(c.isdigit() for c in text):
        return text + ".0"
    return text


class Renderer:
    """Render an expression tree; `names` maps (array, index) / variables to C text."""

    def __init__(self, ref, var):
        self.ref = ref
        self.var = var

    def __call__(self, t):
        k = t[0]
        if k == "num":
            return lit(t[1])
        if k == "var":
            return self.var(t[1])
        if k == "ref":
            return self.ref(t[1], t[2])
        if k == "neg":
            return "(-" + self(t[1]) + ")"
        if k == "bin":
            return "(" + self(t[2]) + " " + t[1] + " " + self(t[3]) + ")"
        if k == "call":
            return CALLS[t[1]] + "(" + ", ".join(self(a) for a in t[2]) + ")"
        raise ValueError(k)


def count_flops(t):
    k = t[0]
    if k in ("num", "var", "ref"):
        return 0
    if k == "neg":
        return count_flops(t[1])
    if k == "bin":
        return 1 + count_flops(t[2]) + count_flops(t[3])
    if k == "call":
        return sum(count_flops(a) for a in t[2])
    raise ValueError(k)


def is_zero(t):
    return t[0] == "num" and float(t[1]) == 0.0


def load(path=os.path.join(HERE, "radm2_mech.json")):
    with open(path) as f:
        return json.load(f)



# The reference's Jacobian keeps reaction 33 (H2O2 + OH) in the H2O2 row although its RHS
# drops it: JVS[49] (row 13, col 13) has -B[43] = -k33 [OH], JVS[51] (13, 52) has
# -B[44] = -k33 [H2O2].
QUIRK_ROW, QUIRK_R, QUIRK_OH = 13, 33, 52

# LU scheduling fence spacing, in loads of U entries (see the decomposition emitter).
LU_FENCE_LOADS = int(os.environ.get("RADM2_LU_FENCE_LOADS", "48"))


def deriv(t):
    """Directional derivative of a rate expression along XIN (product rule over V factors)."""
    k = t[0]
    if k in ("num", "var"):
        return None
    if k == "ref":
        return ["ref", "XIN", t[2]] if t[1] == "V" else None
    if k == "bin" and t[1] == "*":
        da, db = deriv(t[2]), deriv(t[3])
        parts = []
        if da is not None:
            parts.append(["bin", "*", da, t[3]])
        if db is not None:
            parts.append(["bin", "*", t[2], db])
        if not parts:
            return None
        return parts[0] if len(parts) == 1 else ["bin", "+", parts[0], parts[1]]
    raise ValueError("rate expression not a product: %r" % (t,))


def subst_a(t, rx):
    """Replace A[rx] by da<rx> in an RHS term."""
    if t[0] == "ref" and t[1] == "A":
        assert t[2] == rx
        return ["ref", "DA", rx]
    if t[0] == "bin":
        return ["bin", t[1], subst_a(t[2], rx), subst_a(t[3], rx)]
    if t[0] == "neg":
        return ["neg", subst_a(t[1], rx)]
    return t


def _eval(t, env):
    k = t[0]
    if k == "num":
        return float(t[1])
    if k == "ref":
        return env[t[1]][t[2]]
    if k == "neg":
        return -_eval(t[1], env)
    if k == "bin":
        a, b = _eval(t[2], env), _eval(t[3], env)
        if t[1] == "+":
            return a + b
        if t[1] == "-":
            return a - b
        if t[1] == "*":
            return a * b
        return a / b
    raise ValueError(k)


def check_jacvec(m, chains, uses):
    """J_reference x (B partials, JVS slots, CSR) == directional-derivative form, on random data."""
    import random
    rnd = random.Random(7)
    lu = m["lu"]
    for _ in range(3):
        env = {"V": [rnd.uniform(0.5, 2.0) for _ in range(59)], "F": [rnd.uniform(0.5, 2.0) for _ in range(2)],
               "RCT": [rnd.uniform(0.5, 2.0) for _ in range(156)], "XIN": [rnd.uniform(-1, 1) for _ in range(59)]}
        env["B"] = {}
        for k, bt in m["bvals"].items():
            env["B"][int(k)] = _eval(bt, env)
        ref = [0.0] * 59
        for sl, t in enumerate(m["jvs"]):
            ref[lu["irow"][sl]] += _eval(t, env) * env["XIN"][lu["icol"][sl]]
        env["DA"] = {}
        for rx, t in enumerate(m["rates"]):
            d = deriv(t)
            env["DA"][rx] = _eval(d, env) if d is not None else 0.0
        got = [0.0] * 59
        for rx, lst in sorted(uses.items()):
            for (i, pos, op, term) in lst:
                v = _eval(subst_a(term, rx), env)
                got[i] = v if pos == 0 else (got[i] + v if op == "+" else got[i] - v)
        R = env["RCT"][QUIRK_R]
        got[QUIRK_ROW] -= R * env["V"][QUIRK_OH] * env["XIN"][QUIRK_ROW] + R * env["V"][QUIRK_ROW] * env["XIN"][QUIRK_OH]
        for i in range(59):
            assert abs(got[i] - ref[i]) <= 1e-9 * (1 + abs(ref[i])), (i, got[i], ref[i])


# ----------------------------------------------------------------------------- CUDA fragments

def kernel_ref(arr, i):
    return {"RCT": "RC(%d)", "V": "V(%d)", "F": "FIX(%d)", "A": "a%d", "B": "b%d",
            "jv": "JV(%d)", "XIN": "XIN(%d)", "DA": "da%d"}[arr] % i


def kernel_var(name):
    return {"TEMP": "TEMP", "C_M": "C_M", "rc_n2o5": "RC_N2O5"}[name]


def emit_cuda(m, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    r = Renderer(kernel_ref, kernel_var)
    sz = m["sizes"]
    lu = m["lu"]
    crow, diag, icol = lu["crow"], lu["diag"], lu["icol"]
    nvar = sz["NVAR"]
    flops = {}

    # --- header with sizes, tables and method coefficients
    h = [BANNER, "#pragma once\n"]
    for k in ("NVAR", "NFIX", "NREACT", "LU_NONZERO", "NPH", "NB"):
        h.append("#define RADM2_%s %d\n" % (k, sz[k]))
    h.append("#define RADM2_NJV_USED 21   /* photolysis rates 0..20 feed RCONST 0..20 */\n")
    ros = m["ros3"]
    for name, key in (("A", "ros_A"), ("C", "ros_C"), ("M", "ros_M"), ("E", "ros_E"),
                      ("ALPHA", "ros_Alpha"), ("GAMMA", "ros_Gamma")):
        for i, v in enumerate(ros[key]):
            h.append("#define RADM2_ROS_%s%d %s\n" % (name, i, lit(v)))
    h.append("#define RADM2_ROS_ELO %s\n" % lit(ros["ros_ELO"]))
    h.append("\n/* LU pattern (CSR over the 659 slots), recovered from mgpu.cu:2873-3090 */\n")
    h.append("#define RADM2_LU_CROW_INIT {%s}\n" % ",".join(map(str, crow)))
    h.append("#define RADM2_LU_DIAG_INIT {%s}\n" % ",".join(map(str, diag)))
    h.append("#define RADM2_LU_ICOL_INIT {%s}\n" % ",".join(map(str, icol)))
    h.append("#define RADM2_LU_DIAG_SLOTS(X) %s\n" % " ".join("X(%d,%d)" % (i, d) for i, d in enumerate(diag)))
    names = m["species"]
    h.append("#define RADM2_SPECIES_NAMES_INIT {%s}\n" % ",".join('"%s"' % n for n in names[:nvar]))

    # --- rate constants: RC_OUT(r, value)
    body = [BANNER, "/* 156 rate constants, mgpu.cu:763-918.  Inputs: JV(k), TEMP, C_M, RC_N2O5. */\n"]
    for i, t in enumerate(m["rconst"]):
        body.append("RC_OUT(%d, %s);\n" % (i, r(t)))
    write(os.path.join(out_dir, "radm2_rconst.inc"), body)

    # --- RHS, reaction-major: each rate A_r is formed once and immediately added into
    # the accumulators of the species it touches.  Every Vdot sum of the reference lists
    # its reactions in increasing order, so accumulating in reaction order applies the
    # same binary operations to each accumulator in the same order as the reference's
    # left-to-right sum (bit-identical), while only 59 accumulators stay live.
    body = [BANNER, "/* ODE right-hand side, mgpu.cu:1103-1385, reaction-major.  Inputs: RC(r), V(i), FIX(k).\n"
            " * Output VDOT_OUT(i, value) after all reactions. */\n"]
    f = 0
    chains = []
    for i, t in enumerate(m["vdot"]):
        chain = []
        node = t
        while node[0] == "bin" and node[1] in "+-":
            chain.append((node[1], node[3]))
            node = node[2]
        chain.append((None, node))
        chain.reverse()
        chains.append(chain)
        f += count_flops(t)
    uses = {}
    for i, chain in enumerate(chains):
        for pos, (op, term) in enumerate(chain):
            rs = set()
            def walk(x):
                if x[0] == "ref" and x[1] == "A":
                    rs.add(x[2])
                elif x[0] == "bin":
                    walk(x[2]); walk(x[3])
                elif x[0] == "neg":
                    walk(x[1])
            walk(term)
            assert len(rs) == 1, (i, term)
            uses.setdefault(rs.pop(), []).append((i, pos, op, term))
    for i in range(len(chains)):
        body.append("double vd%d;\n" % i)
    for rx, t in enumerate(m["rates"]):
        f += count_flops(t)
        if rx not in uses:
            continue
        body.append("{ const double a%d = %s;\n" % (rx, r(t)))
        for (i, pos, op, term) in uses[rx]:
            if pos == 0:
                body.append("  vd%d = %s;\n" % (i, r(term)))
            else:
                body.append("  vd%d = (vd%d %s %s);\n" % (i, i, op, r(term)))
        body.append("}\n")
    for i in range(len(chains)):
        body.append("VDOT_OUT(%d, vd%d);\n" % (i, i))
    flops["fun"] = f
    write(os.path.join(out_dir, "radm2_fun.inc"), body)

    # --- Jacobian in LU slot order, partial-major: each partial B_b is formed once and
    # added into the slots that use it.  Every JVS slot of the reference sums its
    # partials in increasing b, so accumulating in b order applies the same operations
    # to each slot in the same order (bit-identical); at most ~94 slots are open at once.
    # JAC_OUT(s, value) / JAC_OUT_DIAG(s, value) when a slot is complete; literal-zero
    # slots use JAC_OUT_ZERO(s, is_diag).
    dset = set(diag)
    body = [BANNER, "/* Sparse Jacobian in LU slot order, mgpu.cu:1685-2652, partial-major.\n"
            " * Inputs: RC(r), V(i), FIX(k). */\n"]
    f = 0
    juses = {}
    last_b = {}
    for sl, t in enumerate(m["jvs"]):
        if is_zero(t):
            body.append("JAC_OUT_ZERO(%d%s);\n" % (sl, ", 1" if sl in dset else ", 0"))
            continue
        f += count_flops(t)
        chain = []
        node = t
        while node[0] == "bin" and node[1] in "+-":
            chain.append((node[1], node[3]))
            node = node[2]
        chain.append((None, node))
        chain.reverse()
        for pos, (op, term) in enumerate(chain):
            bs = []

            def walkb(x):
                if x[0] == "ref" and x[1] == "B":
                    bs.append(x[2])
                elif x[0] == "bin":
                    walkb(x[2]); walkb(x[3])
                elif x[0] == "neg":
                    walkb(x[1])
            walkb(term)
            assert len(bs) == 1, (sl, term)
            juses.setdefault(bs[0], []).append((sl, pos, op, term, pos == len(chain) - 1))
    for k in sorted(m["bvals"], key=int):
        bt = m["bvals"][k]
        f += count_flops(bt)
        b = int(k)
        if b not in juses:
            continue
        body.append("{ const double b%d = %s;\n" % (b, r(bt)))
        for (sl, pos, op, term, is_last) in juses[b]:
            if pos == 0:
                expr = r(term)
            else:
                expr = "(js%d %s %s)" % (sl, op, r(term))
            if is_last:
                body.append("  %s(%d, %s);\n" % ("JAC_OUT_DIAG" if sl in dset else "JAC_OUT", sl, expr))
            elif pos == 0:
                body.append("  double js%d = %s;\n" % (sl, expr))
            else:
                body.append("  js%d = %s;\n" % (sl, expr))
        body.append("}\n")
    flops["jac"] = f
    # declarations of the open accumulators must precede their first use: hoist them.
    decl = sorted({int(x.split()[1][2:]) for x in body if x.startswith("  double js")})
    body = [x.replace("  double js", "  js") for x in body]
    body.insert(2, "".join("double js%d;\n" % sl for sl in decl))
    write(os.path.join(out_dir, "radm2_jac.inc"), body)

    # --- Jacobian-vector product J x for the FP64 residual of the FP32-LU refinement.
    # RADM2's rates are products of rate constants and concentrations, so J x is the exact
    # directional derivative of the RHS: dA_r = sum over its concentration factors of the
    # product rule, accumulated reaction-major like the RHS (59 live accumulators).  The
    # reference's Jacobian additionally keeps the H2O2 + OH loss in the H2O2 row that its
    # RHS drops (mgpu.cu:1275 vs 2011, 2013); those two slots are added explicitly.
    # check_jacvec() below verifies J_reference x == this on random data.
    body = [BANNER, "/* y = J(V) x, J the mgpu.cu:1685-2652 Jacobian, as the directional derivative of\n"
            " * the RHS plus the H2O2 row terms.  Inputs: RC, V, FIX, XIN(i).  Output JX_OUT(row, value). */\n"]
    f = 0
    for i in range(len(chains)):
        body.append("double jx%d;\n" % i)
    for rx, t in enumerate(m["rates"]):
        if rx not in uses:
            continue
        dt = deriv(t)
        f += count_flops(dt)
        body.append("{ const double da%d = %s;\n" % (rx, r(dt)))
        for (i, pos, op, term) in uses[rx]:
            dterm = subst_a(term, rx)
            f += count_flops(dterm)
            if pos == 0:
                body.append("  jx%d = %s;\n" % (i, r(dterm)))
            else:
                body.append("  jx%d = (jx%d %s %s);\n" % (i, i, op, r(dterm)))
        body.append("}\n")
    q = QUIRK_ROW
    body.append("jx%d = ((jx%d - (RC(%d) * V(%d)) * XIN(%d)) - (RC(%d) * V(%d)) * XIN(%d));\n"
                % (q, q, QUIRK_R, QUIRK_OH, q, QUIRK_R, q, QUIRK_OH))
    for i in range(len(chains)):
        body.append("JX_OUT(%d, jx%d);\n" % (i, i))
    flops["jacvec"] = f + 6
    write(os.path.join(out_dir, "radm2_jacvec.inc"), body)
    check_jacvec(m, chains, uses)

    for recip in (False, True):
        fd, fs = emit_lu(crow, diag, icol, nvar, out_dir, recip)
        if not recip:
            flops["decomp"], flops["solve"] = fd, fs
        emit_jaclu(m, crow, diag, icol, nvar, out_dir, recip)
    tcol = emit_tmem(crow, diag, icol, nvar, out_dir)
    for recip in (False, True):
        emit_lu_tm(crow, diag, icol, nvar, tcol, out_dir, recip)
    wcol = emit_tmem(crow, diag, icol, nvar, out_dir, TMEM_WIDE_SLOTS, "_wide")
    for recip in (False, True):
        emit_lu_tm(crow, diag, icol, nvar, wcol, out_dir, recip, "_wide")

    h.append("\n/* Algorithmic flop counts per call, counted from the emitted expressions */\n")
    for k, v in sorted(flops.items()):
        h.append("#define RADM2_FLOPS_%s %d\n" % (k.upper(), v))
    write(os.path.join(out_dir, "radm2_gen.h"), h)
    return flops


def emit_lu(crow, diag, icol, nvar, out_dir, recip):
    """Unrolled row-Doolittle LU (mgpu.cu:2746-2779 order) and the triangular solves
    (mgpu.cu:2873-3090 order).  With recip, each finished row stores the reciprocal of
    its pivot in the diagonal slot and the eliminations / back substitution multiply by
    it (one division per row instead of one per lower entry and per solve row)."""
    sfx = "_rcp" if recip else ""
    body = [BANNER, "/* In-place pivot-free LU of G on the fixed fill pattern, the row-by-row\n"
            " * elimination order of mgpu.cu:2746-2779, unrolled.  Accessors: G(s), LU_T (type),\n"
            " * LU_PIVOT_CHECK(row, diag_value); LU_STEP_FENCE ends each elimination step\n"
            " * (a compiler scheduling fence, or nothing).%s */\n"
            % ("\n * Reciprocal form: the diagonal slots hold 1/U(k,k) on exit." if recip else ""),
            "#ifndef LU_STEP_FENCE\n#define LU_STEP_FENCE do { } while (0)\n#endif\n"]
    f = 0
    since_fence = 0
    for k in range(nvar):
        body.append("{ /* row %d */\n" % k)
        body.append("  LU_PIVOT_CHECK(%d, G(%d));\n" % (k, diag[k]))
        if crow[k] == diag[k]:
            if recip:
                body.append("  G(%d) = (LU_T)1 / G(%d);\n" % (diag[k], diag[k]))
                f += 1
            body.append("}\n")  # no elimination, row unchanged
            continue
        for sl in range(crow[k], crow[k + 1]):
            body.append("  LU_T w%d = G(%d);\n" % (icol[sl], sl))
        for kk in range(crow[k], diag[k]):
            j = icol[kk]
            if recip:
                body.append("  { const LU_T a = -w%d * G(%d); w%d = -a;\n" % (j, diag[j], j))
            else:
                body.append("  { const LU_T a = -w%d / G(%d); w%d = -a;\n" % (j, diag[j], j))
            f += 1
            for jj in range(diag[j] + 1, crow[j + 1]):
                body.append("    w%d += a * G(%d);\n" % (icol[jj], jj))
                f += 2
            # A fence once LU_FENCE_LOADS loads have been issued since the last one: the
            # scheduler may overlap that many loads but no more (bounds the live set).
            since_fence += crow[j + 1] - diag[j]
            if since_fence >= LU_FENCE_LOADS:
                body.append("  LU_STEP_FENCE;\n")
                since_fence = 0
            body.append("  }\n")
        for sl in range(crow[k], crow[k + 1]):
            if recip and sl == diag[k]:
                body.append("  G(%d) = (LU_T)1 / w%d;\n" % (sl, icol[sl]))
                f += 1
            else:
                body.append("  G(%d) = w%d;\n" % (sl, icol[sl]))
        body.append("}\n")
    write(os.path.join(out_dir, "radm2_decomp%s.inc" % sfx), body)
    fdec = f

    body = [BANNER, "/* Solve (LU) x = b in place on X(i), mgpu.cu:2873-3090 order.  Accessors: G(s), X(i).%s */\n"
            % (" Diagonal slots hold reciprocals." if recip else "")]
    f = 0
    for k in range(nvar):
        if crow[k] == diag[k]:
            continue
        expr = "X(%d)" % k
        for sl in range(crow[k], diag[k]):
            expr = "(%s - G(%d) * X(%d))" % (expr, sl, icol[sl])
            f += 2
        body.append("X(%d) = %s;\n" % (k, expr))
    for k in reversed(range(nvar)):
        expr = "X(%d)" % k
        for sl in range(diag[k] + 1, crow[k + 1]):
            expr = "(%s - G(%d) * X(%d))" % (expr, sl, icol[sl])
            f += 2
        body.append("X(%d) = %s %s G(%d);\n" % (k, expr, "*" if recip else "/", diag[k]))
        f += 1
    write(os.path.join(out_dir, "radm2_solve%s.inc" % sfx), body)
    return fdec, f


TMEM_SLOTS = 128  # doubles of tensor memory per thread (256 32-bit columns)
TMEM_WIDE_SLOTS = 256  # one 128-thread CTA per SM owning all 512 columns


def lu_slot_accesses(crow, diag, icol, nvar):
    """Loads and stores of each LU slot in one step attempt of the thread-per-cell solver:
    the Jacobian's store, the factorisation's row loads, stores and pivot-row reads
    (emit_lu's order; a row without eliminations touches only its pivot), and the three
    stage solves' reads."""
    acc = [1] * len(icol)
    for k in range(nvar):
        if crow[k] == diag[k]:
            acc[diag[k]] += 2
            continue
        for s in range(crow[k], crow[k + 1]):
            acc[s] += 2
        for kk in range(crow[k], diag[k]):
            j = icol[kk]
            acc[diag[j]] += 1
            for jj in range(diag[j] + 1, crow[j + 1]):
                acc[jj] += 1
    for k in range(nvar):
        for s in range(crow[k], crow[k + 1]):
            acc[s] += 3
    return acc


def emit_tmem(crow, diag, icol, nvar, out_dir, nslot=TMEM_SLOTS, tag=""):
    """The LU slots a thread keeps in its tensor-memory row: the nslot most accessed per
    step attempt (ties by slot index), each a double in two 32-bit columns.  tag "" is the
    128-slot map (PLACE_LU_TMEM), "_wide" the 256-slot map (PLACE_LU_TMEM_WIDE)."""
    acc = lu_slot_accesses(crow, diag, icol, nvar)
    hot = sorted(range(len(icol)), key=lambda s: (-acc[s], s))[:nslot]
    col = [-1] * len(icol)
    for i, s in enumerate(sorted(hot)):
        col[s] = 2 * i
    up = tag.upper()
    body = [BANNER, "/* Tensor-memory placement of the LU slots (PLACE_LU_TMEM%s): the %d slots with the\n"
            " * most loads and stores per step attempt (%d of %d), slot s at 32-bit column\n"
            " * radm2_tmem%s_col[s] of the thread's row, -1: global scratch. */\n"
            % (up, nslot, sum(acc[s] for s in hot), sum(acc), tag),
            "#pragma once\n#define RADM2_TMEM%s_SLOTS %d\n" % (up, nslot),
            "static constexpr short radm2_tmem%s_col[%d] = {%s};\n" % (tag, len(col), ",".join(map(str, col)))]
    write(os.path.join(out_dir, "radm2_tmem%s.h" % tag), body)
    return col


TM_GROUP = 16  # doubles per tensor-memory load statement (32 registers)


def tm_runs(slots, col):
    """Split a list of slots into runs of tensor-memory slots with consecutive columns
    (global slots are left out)."""
    runs, cur = [], []
    for s in slots:
        if col[s] >= 0 and cur and col[s] == col[cur[-1]] + 2:
            cur.append(s)
        else:
            if cur:
                runs.append(cur)
            cur = [s] if col[s] >= 0 else []
    if cur:
        runs.append(cur)
    return runs


def tm_pieces(run, col):
    """A run as (first slot index in the run, doubles) pieces of 1, 2, 4 or 8 doubles, each
    starting on a column that is a multiple of its own width."""
    out, i = [], 0
    while i < len(run):
        c = col[run[i]]
        for p in (8, 4, 2, 1):
            if p <= len(run) - i and c % (2 * p) == 0:
                out.append((i, p))
                i += p
                break
    return out


def tm_load(pairs, col, ind):
    """Load tensor-memory slots into already declared doubles: pairs [(slot, var)] in slot
    order.  One statement per TM_GROUP doubles: its loads, then one wait, so the values are
    never read before they arrive."""
    var = dict(pairs)
    pieces = []
    for run in tm_runs([s for s, _ in pairs], col):
        pieces += [(run[i:i + p], p) for i, p in tm_pieces(run, col)]
    lines, group, n = [], [], 0
    for pc in pieces + [None]:
        if pc is None or n + pc[1] > TM_GROUP:
            if group:
                nout = 2 * n
                text, outs, ins, k = [], [], [], 0
                for gi, (sl, p) in enumerate(group):
                    regs = ",".join("%%%d" % (k + r) for r in range(2 * p))
                    text.append("tcgen05.ld.sync.aligned.32x32b.x%d.b32 {%s}, [%%%d];" % (2 * p, regs, nout + gi))
                    for s in sl:
                        outs.append('"=r"(tl%d), "=r"(th%d)' % (s, s))
                    ins.append('"r"(TM_BASE + %du)' % col[sl[0]])
                    k += 2 * p
                text.append("tcgen05.wait::ld.sync.aligned;")
                slots = [s for sl, _ in group for s in sl]
                lines.append("%s{ unsigned %s;\n" % (ind, ", ".join("tl%d, th%d" % (s, s) for s in slots)))
                lines.append('%s  asm volatile("%s" : %s : %s);\n' % (ind, "\\n\\t".join(text), ", ".join(outs),
                                                                      ", ".join(ins)))
                for s in slots:
                    lines.append("%s  %s = __hiloint2double((int)th%d, (int)tl%d);\n" % (ind, var[s], s, s))
                lines.append("%s}\n" % ind)
            group, n = [], 0
        if pc is not None:
            group.append(pc)
            n += pc[1]
    return lines


def tm_store(pairs, col, ind):
    """Store doubles into tensor-memory slots: pairs [(slot, expression)] in slot order.
    The stores are asynchronous; the caller waits for them before the slots are read."""
    val = dict(pairs)
    lines = []
    for run in tm_runs([s for s, _ in pairs], col):
        for i, p in tm_pieces(run, col):
            sl = run[i:i + p]
            regs = ",".join("%%%d" % (1 + r) for r in range(2 * p))
            ins = ['"r"(TM_BASE + %du)' % col[sl[0]]]
            for s in sl:
                ins.append('"r"(__double2loint(%s)), "r"(__double2hiint(%s))' % (val[s], val[s]))
            lines.append('%sasm volatile("tcgen05.st.sync.aligned.32x32b.x%d.b32 [%%0], {%s};" :: %s);\n'
                         % (ind, 2 * p, regs, ", ".join(ins)))
    return lines


def emit_lu_tm(crow, diag, icol, nvar, col, out_dir, recip, tag=""):
    """The LU and triangular solves of emit_lu (reciprocal or division form) for the
    tensor-memory placement: the same operations in the same order, with the tensor-memory
    slots of a row (or of a pivot row's U part) read by wide tcgen05 loads with one wait per
    group instead of one load and one wait each.  Global slots go through G(s).  TM_BASE is
    the thread's first column address; every statement is warp-collective."""
    sfx = "_rcp" if recip else ""
    body = [BANNER, "/* Pivot-free LU (mgpu.cu:2746-2779 order, %s) with tensor-memory slots\n"
            " * (radm2_tmem.h) loaded and stored in groups.  Accessors: G(s) (global slots), LU_T,\n"
            " * TM_BASE, LU_PIVOT_CHECK(row, value), LU_STEP_FENCE. */\n"
            % ("reciprocal pivots" if recip else "pivot divisions"),
            "#ifndef LU_STEP_FENCE\n#define LU_STEP_FENCE do { } while (0)\n#endif\n"]
    wait_st = '  asm volatile("tcgen05.wait::st.sync.aligned;");\n'
    since_fence = 0
    for k in range(nvar):
        body.append("{ /* row %d */\n" % k)
        d = diag[k]
        if crow[k] == d:  # no elimination: the pivot check, and in reciprocal form 1/pivot
            if col[d] >= 0:
                body.append("  LU_T w%d;\n" % k)
                body += tm_load([(d, "w%d" % k)], col, "  ")
                body.append("  LU_PIVOT_CHECK(%d, w%d);\n" % (k, k))
                if recip:
                    body += tm_store([(d, "((LU_T)1 / w%d)" % k)], col, "  ")
                    body.append(wait_st)
            else:
                body.append("  LU_PIVOT_CHECK(%d, G(%d));\n" % (k, d))
                if recip:
                    body.append("  G(%d) = (LU_T)1 / G(%d);\n" % (d, d))
            body.append("}\n")
            continue
        row = list(range(crow[k], crow[k + 1]))
        for sl in row:
            if col[sl] >= 0:
                body.append("  LU_T w%d;\n" % icol[sl])
            else:
                body.append("  LU_T w%d = G(%d);\n" % (icol[sl], sl))
        body += tm_load([(sl, "w%d" % icol[sl]) for sl in row if col[sl] >= 0], col, "  ")
        body.append("  LU_PIVOT_CHECK(%d, w%d);\n" % (k, k))
        for kk in range(crow[k], d):
            j = icol[kk]
            seg = [diag[j]] + list(range(diag[j] + 1, crow[j + 1]))
            tms = [s for s in seg if col[s] >= 0]
            body.append("  {\n")
            if tms:
                body.append("    LU_T %s;\n" % ", ".join("u%d" % s for s in tms))
                body += tm_load([(s, "u%d" % s) for s in tms], col, "    ")
            ref = lambda s: ("u%d" % s) if col[s] >= 0 else ("G(%d)" % s)  # noqa: E731
            body.append("    const LU_T a = -w%d %s %s; w%d = -a;\n" % (j, "*" if recip else "/", ref(diag[j]), j))
            for jj in range(diag[j] + 1, crow[j + 1]):
                body.append("    w%d += a * %s;\n" % (icol[jj], ref(jj)))
            since_fence += crow[j + 1] - diag[j]
            if since_fence >= LU_FENCE_LOADS:
                body.append("  LU_STEP_FENCE;\n")
                since_fence = 0
            body.append("  }\n")
        out = []
        for sl in row:
            v = "((LU_T)1 / w%d)" % icol[sl] if (recip and sl == d) else "w%d" % icol[sl]
            if col[sl] >= 0:
                out.append((sl, v))
            else:
                body.append("  G(%d) = %s;\n" % (sl, v))
        if out:
            body += tm_store(out, col, "  ")
            body.append(wait_st)
        body.append("}\n")
    write(os.path.join(out_dir, "radm2_decomp%s_tm%s.inc" % (sfx, tag)), body)

    body = [BANNER, "/* Solve (LU) x = b in place on X(i) (mgpu.cu:2873-3090 order, %s)\n"
            " * with tensor-memory slots loaded in groups.  Accessors: G(s), X(i), TM_BASE. */\n"
            % ("reciprocal pivots" if recip else "pivot divisions")]
    for k in range(nvar):
        if crow[k] == diag[k]:
            continue
        seg = list(range(crow[k], diag[k]))
        tms = [s for s in seg if col[s] >= 0]
        body.append("{\n")
        if tms:
            body.append("  double %s;\n" % ", ".join("g%d" % s for s in tms))
            body += tm_load([(s, "g%d" % s) for s in tms], col, "  ")
        expr = "X(%d)" % k
        for sl in seg:
            expr = "(%s - %s * X(%d))" % (expr, ("g%d" % sl) if col[sl] >= 0 else ("G(%d)" % sl), icol[sl])
        body.append("  X(%d) = %s;\n}\n" % (k, expr))
    for k in reversed(range(nvar)):
        seg = [diag[k]] + list(range(diag[k] + 1, crow[k + 1]))
        tms = [s for s in seg if col[s] >= 0]
        body.append("{\n")
        if tms:
            body.append("  double %s;\n" % ", ".join("g%d" % s for s in tms))
            body += tm_load([(s, "g%d" % s) for s in tms], col, "  ")
        ref = lambda s: ("g%d" % s) if col[s] >= 0 else ("G(%d)" % s)  # noqa: E731
        expr = "X(%d)" % k
        for sl in range(diag[k] + 1, crow[k + 1]):
            expr = "(%s - %s * X(%d))" % (expr, ref(sl), icol[sl])
        body.append("  X(%d) = %s %s %s;\n}\n" % (k, expr, "*" if recip else "/", ref(diag[k])))
    write(os.path.join(out_dir, "radm2_solve%s_tm%s.inc" % (sfx, tag)), body)


def slot_chain(t):
    """A Jacobian slot's expression as its left-to-right chain [(None, t0), (op, t1), ...]."""
    chain = []
    node = t
    while node[0] == "bin" and node[1] in "+-":
        chain.append((node[1], node[3]))
        node = node[2]
    chain.append((None, node))
    chain.reverse()
    return chain


def term_b(term):
    """The one partial B_b a Jacobian term multiplies."""
    bs = []

    def walkb(x):
        if x[0] == "ref" and x[1] == "B":
            bs.append(x[2])
        elif x[0] == "bin":
            walkb(x[2]); walkb(x[3])
        elif x[0] == "neg":
            walkb(x[1])
    walkb(term)
    assert len(bs) == 1, term
    return bs[0]


def count_loads(t):
    """Array reads (RC, V) in an expression."""
    if t[0] == "ref":
        return 1 if t[1] in ("RCT", "V") else 0
    if t[0] == "bin":
        return count_loads(t[2]) + count_loads(t[3])
    if t[0] == "neg":
        return count_loads(t[1])
    if t[0] == "call":
        return sum(count_loads(a) for a in t[2])
    return 0


def emit_jaclu(m, crow, diag, icol, nvar, out_dir, recip):
    """Jacobian and LU fused row by row: row k's slots of G = -J + ghinv I are formed in
    registers (each slot the same left-to-right sum of its partials as the partial-major
    Jacobian, so the same value), its pivot is checked, the row is eliminated against the
    finished rows above it exactly as emit_lu does, and only then stored.  The matrix is
    written once per factorisation instead of written by the Jacobian and read back by
    the LU; the price is that a partial feeding several rows is formed once per row."""
    sfx = "_rcp" if recip else ""
    r = Renderer(kernel_ref, kernel_var)
    dset = set(diag)
    body = [BANNER, "/* Jacobian (mgpu.cu:1685-2652) and pivot-free LU (mgpu.cu:2746-2779) fused row by\n"
            " * row.  Inputs: RC(r), V(i), FIX(k).  Accessors: G(s), LU_T; JAC_VAL(e),\n"
            " * JAC_VAL_DIAG(e) and JAC_VAL_ZERO(is_diag) turn a Jacobian slot into a slot of G;\n"
            " * LU_PIVOT_CHECK(row, diag_value); LU_STEP_FENCE bounds the loads in flight.%s */\n"
            % ("\n * Reciprocal form: the diagonal slots hold 1/U(k,k) on exit." if recip else ""),
            "#ifndef LU_STEP_FENCE\n#define LU_STEP_FENCE do { } while (0)\n#endif\n"]
    since_fence = 0
    for k in range(nvar):
        body.append("{ /* row %d */\n" % k)
        for sl in range(crow[k], crow[k + 1]):
            t = m["jvs"][sl]
            c = icol[sl]
            if is_zero(t):
                body.append("  LU_T w%d = JAC_VAL_ZERO(%d);\n" % (c, 1 if sl in dset else 0))
                continue
            chain = slot_chain(t)
            defs = []
            expr = None
            for pos, (op, term) in enumerate(chain):
                b = term_b(term)
                bt = m["bvals"][str(b)]
                defs.append("const double b%d = %s;" % (b, r(bt)))
                since_fence += count_loads(bt)
                expr = r(term) if pos == 0 else "(%s %s %s)" % (expr, op, r(term))
            body.append("  LU_T w%d;\n  { %s\n    w%d = %s(%s); }\n"
                        % (c, "\n    ".join(defs), c, "JAC_VAL_DIAG" if sl in dset else "JAC_VAL", expr))
            if since_fence >= LU_FENCE_LOADS:
                body.append("  LU_STEP_FENCE;\n")
                since_fence = 0
        body.append("  LU_PIVOT_CHECK(%d, w%d);\n" % (k, k))
        for kk in range(crow[k], diag[k]):
            j = icol[kk]
            if recip:
                body.append("  { const LU_T a = -w%d * G(%d); w%d = -a;\n" % (j, diag[j], j))
            else:
                body.append("  { const LU_T a = -w%d / G(%d); w%d = -a;\n" % (j, diag[j], j))
            for jj in range(diag[j] + 1, crow[j + 1]):
                body.append("    w%d += a * G(%d);\n" % (icol[jj], jj))
            since_fence += crow[j + 1] - diag[j]
            if since_fence >= LU_FENCE_LOADS:
                body.append("  LU_STEP_FENCE;\n")
                since_fence = 0
            body.append("  }\n")
        for sl in range(crow[k], crow[k + 1]):
            if recip and sl == diag[k]:
                body.append("  G(%d) = (LU_T)1 / w%d;\n" % (sl, icol[sl]))
            else:
                body.append("  G(%d) = w%d;\n" % (sl, icol[sl]))
        body.append("}\n")
    write(os.path.join(out_dir, "radm2_jaclu%s.inc" % sfx), body)


# ----------------------------------------------------------------------------- oracle C

def oracle_ref(arr, i):
    return {"RCT": "RCT[%d]", "V": "V[%d]", "F": "F[%d]", "A": "A[%d]", "B": "B[%d]",
            "jv": "jv[%d]"}[arr] % i


def oracle_var(name):
    return {"TEMP": "TEMP", "C_M": "C_M", "rc_n2o5": "rc_n2o5"}[name]


def emit_oracle(m, out_dir):
    os.makedirs(out_dir, exist_ok=True)
    r = Renderer(oracle_ref, oracle_var)
    sz = m["sizes"]
    lu = m["lu"]
    c = [BANNER, '#include "../radm2_oracle.h"\n#include <math.h>\n\n']
    c.append("/* LU pattern tables (CSR), recovered from mgpu.cu:2873-3090 */\n")
    c.append("const int orc_lu_crow[%d] = {%s};\n" % (len(lu["crow"]), ",".join(map(str, lu["crow"]))))
    c.append("const int orc_lu_diag[%d] = {%s};\n" % (len(lu["diag"]), ",".join(map(str, lu["diag"]))))
    c.append("const int orc_lu_icol[%d] = {%s};\n\n" % (len(lu["icol"]), ",".join(map(str, lu["icol"]))))
    c.append("/* Rate constants: mgpu.cu:763-918 (dev_Update_RCONST) */\n")
    c.append("void orc_rconst(const double *jv, double TEMP, double C_M, double rc_n2o5, double *RCT)\n{\n")
    for i, t in enumerate(m["rconst"]):
        c.append("  RCT[%d] = %s;\n" % (i, r(t)))
    c.append("}\n\n")
    c.append("/* ODE right-hand side: mgpu.cu:1103-1385 (dev_Fun) */\n")
    c.append("void orc_fun(const double *V, const double *F, const double *RCT, double *Vdot)\n{\n")
    c.append("  double A[%d];\n" % sz["NREACT"])
    for i, t in enumerate(m["rates"]):
        c.append("  A[%d] = %s;\n" % (i, r(t)))
    for i, t in enumerate(m["vdot"]):
        c.append("  Vdot[%d] = %s;\n" % (i, r(t)))
    c.append("}\n\n")
    c.append("/* Sparse Jacobian in LU slot order: mgpu.cu:1685-2652 (dev_Jac_SP) */\n")
    c.append("void orc_jac(const double *V, const double *F, const double *RCT, double *JVS)\n{\n")
    c.append("  double B[%d];\n" % sz["NB"])
    for k in sorted(m["bvals"], key=int):
        c.append("  B[%s] = %s;\n" % (k, r(m["bvals"][k])))
    for s, t in enumerate(m["jvs"]):
        c.append("  JVS[%d] = %s;\n" % (s, r(t)))
    c.append("}\n")
    w = m["wrf"]
    src_id = {"chem": 0, "rad": 1}
    c.append("\n/* WRF -> KPP conversion tables, mgpu.cu:513-646 (dev_convert): species i takes field\n"
             " * orc_wrf_var_src[i][1] of the chem (0) or rad (1) array; jv k takes ph field orc_wrf_jv_src[k]. */\n")
    c.append("const int orc_wrf_var_src[%d][2] = {%s};\n" % (
        len(w["var_src"]), ",".join("{%d,%d}" % (src_id[a], f) for a, f in w["var_src"])))
    c.append("const int orc_wrf_jv_src[%d] = {%s};\n" % (len(w["jv_src"]), ",".join(map(str, w["jv_src"]))))
    write(os.path.join(out_dir, "radm2_oracle_gen.c"), c)


def emit_wrf(m, out_dir):
    """WRF -> KPP conversion tables for the kernels (mgpu.cu:513-646, 682-706)."""
    w = m["wrf"]
    src_id = {"chem": 0, "rad": 1}
    d, g = w["dims"], w["window"]
    h = [BANNER, "#pragma once\n/* WRF -> KPP conversion, %s.\n"
         " * Fields are field-major with i fastest: field[f][nj][nk][ni].  Species v takes\n"
         " * conv * max(src[f], 0) with src 0 = chem, 1 = rad; photolysis slot k takes ph[f] / 60. */\n"
         % w["citation"]]
    h.append("#define RADM2_WRF_VAR_SRC(X) %s\n" % " ".join("X(%d,%d,%d)" % (v, src_id[a], f)
                                                          for v, (a, f) in enumerate(w["var_src"])))
    h.append("#define RADM2_WRF_JV_SRC(X) %s\n" % " ".join("X(%d,%d)" % (k, f) for k, f in enumerate(w["jv_src"])))
    h.append("#define RADM2_WRF_NCHEM_USED %d\n" % (1 + max(f for a, f in w["var_src"] if a == "chem")))
    h.append("#define RADM2_WRF_NRAD_USED %d\n" % (1 + max(f for a, f in w["var_src"] if a == "rad")))
    h.append("#define RADM2_WRF_NPH_USED %d\n" % (1 + max(w["jv_src"])))
    h.append("/* the reference's domain (ni, nk, nj) and interior window (i0, k0, j0, wi, wk, wj) */\n")
    h.append("#define RADM2_WRF_REF_GRID_INIT {%d, %d, %d, %d, %d, %d, %d, %d, %d}\n" % (
        d["ni"], d["nk"], d["nj"], g["i0"], g["k0"], g["j0"], g["wi"], g["wk"], g["wj"]))
    write(os.path.join(out_dir, "radm2_wrf.h"), h)


def write(path, parts):
    with open(path, "w") as f:
        f.write("".join(parts))


def main():
    m = load()
    flops = emit_cuda(m, CSRC_GEN)
    emit_wrf(m, CSRC_GEN)
    emit_oracle(m, ORACLE_GEN)
    print("emitted", CSRC_GEN, ORACLE_GEN, flops)


if __name__ == "__main__":
    main()
