#!/usr/bin/env python3
"""Extract the RADM2 mechanism tables from the reference's mgpu.cu into JSON.

The reference encodes its chemistry as KPP-generated straight-line C inside
CUDA kernels.  This script reads that text and records the mechanism as data:

  * species / photolysis / fixed-species index maps   mgpu.cu:52-79, 125-193
  * the 156 rate-constant expressions                 mgpu.cu:763-918  (dev_Update_RCONST)
  * the 156 reaction rates A[r] and 59 Vdot sums       mgpu.cu:1103-1385 (dev_Fun)
  * the Jacobian partials B[b] and 659 JVS slots      mgpu.cu:1685-2652 (dev_Jac_SP)
  * the LU sparsity pattern, recovered from the        mgpu.cu:2873-3090 (dev_KppSolve)
    fully unrolled triangular solves (the reference
    declares LU_DIAG/CROW/ICOL but never fills them,  mgpu.cu:197-207)
  * the ROS-3 method coefficients                     mgpu.cu:1007-1062 (Ros3)

Every expression is kept as a parse tree so the emitter (emit.py) can render
it with exactly the reference's association order; nothing is simplified.
The output, mech/radm2_mech.json, is committed: the build and the GPU runs do
not need the reference.

Usage:  python gen_mech.py /path/to/mgpu.cu
"""
import ast
import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))

# Expected LU structure of the RADM2 mechanism (row starts and diagonal slots).
EXPECT_CROW = [0, 3, 9, 26, 29, 31, 33, 35, 37, 39, 41, 43, 46, 49, 52, 55, 57, 62, 66, 71, 75, 79,
               84, 88, 92, 104, 120, 124, 128, 132, 140, 148, 156, 170, 180, 187, 194, 204, 216,
               229, 238, 245, 267, 298, 305, 318, 329, 343, 368, 378, 393, 435, 464, 511, 541,
               569, 586, 602, 625, 659]
EXPECT_DIAG = [0, 3, 9, 26, 29, 31, 33, 35, 37, 39, 41, 43, 46, 49, 52, 55, 57, 62, 67, 71, 75, 81,
               84, 88, 94, 105, 120, 124, 128, 132, 140, 149, 158, 170, 181, 188, 196, 208, 220,
               230, 239, 252, 283, 299, 310, 323, 334, 356, 370, 384, 426, 456, 504, 535, 564,
               582, 599, 623, 658]


def strip_comments(text):
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    return text


def function_body(src, signature_regex):
    """Return the text between the braces of the first function matching the regex."""
    m = re.search(signature_regex, src)
    if not m:
        raise SystemExit("function not found: " + signature_regex)
    i = src.index("{", m.end())
    depth = 0
    for j in range(i, len(src)):
        if src[j] == "{":
            depth += 1
        elif src[j] == "}":
            depth -= 1
            if depth == 0:
                return src[i + 1:j]
    raise SystemExit("unbalanced braces after " + signature_regex)


def to_tree(node):
    """Convert a Python ast expression node (C expressions parse as Python here) to JSON."""
    if isinstance(node, ast.Expression):
        return to_tree(node.body)
    if isinstance(node, ast.Constant):
        if isinstance(node.value, bool) or not isinstance(node.value, (int, float)):
            raise ValueError("unexpected constant %r" % (node.value,))
        return ["num", repr(node.value) if isinstance(node.value, float) else str(node.value)]
    if isinstance(node, ast.Name):
        return ["var", node.id]
    if isinstance(node, ast.Subscript):
        idx = node.slice
        if not isinstance(idx, ast.Constant):
            raise ValueError("non-constant subscript")
        return ["ref", node.value.id, int(idx.value)]
    if isinstance(node, ast.UnaryOp):
        if isinstance(node.op, ast.USub):
            return ["neg", to_tree(node.operand)]
        if isinstance(node.op, ast.UAdd):
            return to_tree(node.operand)
        raise ValueError("unary op")
    if isinstance(node, ast.BinOp):
        ops = {ast.Add: "+", ast.Sub: "-", ast.Mult: "*", ast.Div: "/"}
        return ["bin", ops[type(node.op)], to_tree(node.left), to_tree(node.right)]
    if isinstance(node, ast.Call):
        name = node.func.id
        args = [to_tree(a) for a in node.args]
        if name in ("X", "JVS") and len(args) == 1 and args[0][0] == "num":
            return ["ref", name, int(args[0][1])]
        return ["call", name, args]
    raise ValueError("unsupported node %s" % type(node).__name__)


def parse_expr(text):
    text = re.sub(r"MY_I(?:_A)?\((\d+)\)", r"\1", text)
    text = " ".join(text.split())
    return to_tree(ast.parse(text, mode="eval"))


def assignments(body, lhs_names):
    """Yield (name, index, tree) for statements 'NAME[k] = expr;' in body, in order."""
    body = strip_comments(body)
    body = "\n".join(l for l in body.split("\n") if not l.strip().startswith("#"))
    pat = re.compile(r"^\s*(%s)\s*\[\s*MY_I(?:_A)?\((\d+)\)\s*\]\s*=\s*(.*)$" % "|".join(lhs_names), re.S)
    for stmt in body.split(";"):
        m = pat.match(stmt)
        if m:
            yield m.group(1), int(m.group(2)), parse_expr(m.group(3))


def refs_in(tree, name, out=None):
    if out is None:
        out = []
    if tree[0] == "ref" and tree[1] == name:
        out.append(tree[2])
    elif tree[0] == "bin":
        refs_in(tree[2], name, out)
        refs_in(tree[3], name, out)
    elif tree[0] == "neg":
        refs_in(tree[1], name, out)
    elif tree[0] == "call":
        for a in tree[2]:
            refs_in(a, name, out)
    return out


def subtraction_chain(tree):
    """Flatten ((x - t1) - t2) - ... into (x, [t1, t2, ...])."""
    terms = []
    while tree[0] == "bin" and tree[1] == "-":
        terms.append(tree[3])
        tree = tree[2]
    terms.reverse()
    return tree, terms


def jvs_times_x(term):
    if term[0] == "bin" and term[1] == "*" and term[2][0] == "ref" and term[2][1] == "JVS" \
            and term[3][0] == "ref" and term[3][1] == "X":
        return term[2][2], term[3][2]
    raise ValueError("unexpected solve term %r" % (term,))


def extract_lu_pattern(solve_body):
    """Recover the CSR LU pattern from the unrolled forward/backward solves."""
    body = strip_comments(solve_body)
    body = "\n".join(l for l in body.split("\n") if not l.strip().startswith("#"))
    stmts = [s for s in body.split(";") if re.match(r"^\s*X\(\d+\)\s*=", s)]
    entries = {}  # slot -> (row, col)
    diag = {}
    fwd_rows, bwd_rows = [], []
    for s in stmts:
        lhs, rhs = s.split("=", 1)
        k = int(re.search(r"\d+", lhs).group())
        tree = to_tree(ast.parse(" ".join(rhs.split()), mode="eval"))
        if tree[0] == "bin" and tree[1] == "/":
            # backward: (X(k) - sum U(k,j) X(j)) / JVS(d)
            num, den = tree[2], tree[3]
            assert den[0] == "ref" and den[1] == "JVS"
            head, terms = subtraction_chain(num)
            assert head == ["ref", "X", k]
            diag[k] = den[2]
            entries[den[2]] = (k, k)
            for t in terms:
                slot, col = jvs_times_x(t)
                assert col > k
                entries[slot] = (k, col)
            bwd_rows.append(k)
        else:
            head, terms = subtraction_chain(tree)
            assert head == ["ref", "X", k]
            for t in terms:
                slot, col = jvs_times_x(t)
                assert col < k
                entries[slot] = (k, col)
            fwd_rows.append(k)
    nvar = len(diag)
    nslot = len(entries)
    assert sorted(entries) == list(range(nslot)), "LU slots are not a dense 0..n-1 range"
    icol = [entries[s][1] for s in range(nslot)]
    irow = [entries[s][0] for s in range(nslot)]
    crow = []
    for r in range(nvar):
        slots = [s for s in range(nslot) if irow[s] == r]
        assert slots == list(range(slots[0], slots[-1] + 1)), "row %d not contiguous" % r
        cols = [icol[s] for s in slots]
        assert cols == sorted(cols), "row %d columns not sorted" % r
        crow.append(slots[0])
    crow.append(nslot)
    ludiag = [diag[r] for r in range(nvar)]
    return {"crow": crow, "diag": ludiag, "icol": icol, "irow": irow,
            "forward_rows": fwd_rows, "backward_rows": bwd_rows}


def check_closed(pattern):
    """Symbolic elimination (row Doolittle) must not create entries outside the pattern."""
    crow, diag, icol = pattern["crow"], pattern["diag"], pattern["icol"]
    nvar = len(diag)
    for k in range(nvar):
        present = set(icol[crow[k]:crow[k + 1]])
        for kk in range(crow[k], diag[k]):
            j = icol[kk]
            for jj in range(diag[j] + 1, crow[j + 1]):
                if icol[jj] not in present:
                    return False
    return True


def main():
    if len(sys.argv) != 2:
        raise SystemExit("usage: python gen_mech.py /path/to/mgpu.cu")
    src_path = sys.argv[1]
    with open(src_path) as f:
        src = f.read()

    defines = dict(re.findall(r"#define\s+(\w+)\s+\(?(-?\d+)\)?\s*(?://.*)?$", src, flags=re.M))
    nvar, nfix, nreact = int(defines["NVAR"]), int(defines["NFIX"]), int(defines["NREACT"])
    lu_nonzero, nonzero, nph = int(defines["LU_NONZERO"]), int(defines["NONZERO"]), int(defines["NPH"])
    species = {}
    for name, idx in re.findall(r"#define\s+ind_(\w+)\s+(\d+)", src):
        species[int(idx)] = name
    photolysis = {}
    for name, idx in re.findall(r"#define\s+Pj_(\w+)\s+(\d+)", src):
        photolysis[int(idx)] = name

    rconst_body = function_body(src, r"__global__\s+void\s+dev_Update_RCONST\s*\(")
    rconst = {i: t for _, i, t in assignments(rconst_body, ["RCONST"])}
    assert sorted(rconst) == list(range(nreact))

    fun_body = function_body(src, r"__global__\s+void\s+dev_Fun\s*\(")
    rates, vdot = {}, {}
    for name, i, t in assignments(fun_body, ["A", "Vdot"]):
        (rates if name == "A" else vdot)[i] = t
    assert sorted(rates) == list(range(nreact)) and sorted(vdot) == list(range(nvar))

    jac_body = function_body(src, r"__global__\s+void\s+dev_Jac_SP\s*\(")
    bvals, jvs = {}, {}
    for name, i, t in assignments(jac_body, ["B", "JVS"]):
        (bvals if name == "B" else jvs)[i] = t
    assert sorted(jvs) == list(range(lu_nonzero))

    solve_body = function_body(src, r"__global__\s+void\s+dev_KppSolve\s*\(")
    pattern = extract_lu_pattern(solve_body)
    assert pattern["crow"] == EXPECT_CROW, "LU_CROW mismatch"
    assert pattern["diag"] == EXPECT_DIAG, "LU_DIAG mismatch"
    assert check_closed(pattern), "LU pattern is not closed under elimination"

    ros_body = function_body(src, r"void\s+Ros3\s*\(")
    ros = {}
    for arr, idx, val in re.findall(r"(ros_\w+)\[(\d+)\]\s*=\s*\(double\)\s*\(?([-0-9.eE+]+)\)?\s*;", ros_body):
        ros.setdefault(arr, {})[int(idx)] = val
    ros_tab = {k: [v[i] for i in sorted(v)] for k, v in ros.items()}
    nf = re.findall(r"ros_NewF\[(\d+)\]\s*=\s*(\d+)", ros_body)
    ros_tab["ros_NewF"] = [int(v) for _, v in sorted(nf)]
    ros_tab["ros_ELO"] = re.search(r"\*ros_ELO\s*=\s*\(double\)\s*([0-9.]+)", ros_body).group(1)
    ros_tab["ros_S"] = int(re.search(r"\*ros_S\s*=\s*(\d+)", ros_body).group(1))

    # WRF -> KPP conversion (dev_convert, mgpu.cu:513-646): which WRF field feeds each
    # species and photolysis slot, the field dimensions, and the interior window the
    # launch in convertWRFChemData (mgpu.cu:682-706) covers.
    conv_body = strip_comments(function_body(src, r"__global__\s+void\s+dev_convert\s*\("))
    var_src = {}
    for a, arr, b in re.findall(r"VAR\[MY_I\((\d+)\)\]\s*=\s*conv\s*\*\s*MAX\(\(wrf(chem|rad)data\[\(\((\d+)\)\*",
                                conv_body):
        assert int(a) not in var_src
        var_src[int(a)] = [arr, int(b)]
    assert sorted(var_src) == list(range(nvar)), "dev_convert must set every species"
    jv_src = {}
    for n, m2, div in re.findall(r"jv\[MY_I\((\d+)\)\]\s*=\s*\(wrfphdata\[\(\((\d+)\)\*[^;]*\)\s*/\s*([0-9.]+)\s*;",
                                 conv_body):
        assert float(div) == 60.0
        jv_src[int(n)] = int(m2)
    assert sorted(jv_src) == list(range(nph))
    dims = re.search(r"wrfphydata\[\(\(2\)\*(\d+)\*(\d+)\*(\d+) \+ \(j\)\*(\d+)\*(\d+) \+ \(k\)\*(\d+)", conv_body)
    nj_, nk_, ni_ = int(dims.group(1)), int(dims.group(2)), int(dims.group(3))
    offs = {v: int(o) for v, o in re.findall(r"\b([ijk])\s*\+=\s*(\d+)\s*;", conv_body)}
    launch = function_body(src, r"void\s+convertWRFChemData\s*\(")
    gy = int(re.search(r"gridDim\.y\s*=\s*(\d+)", launch).group(1))
    gx = int(re.search(r"gridDim\.x\s*=\s*(\d+)", launch).group(1))
    bx = int(re.search(r"blockDim\.x\s*=\s*(\d+)", launch).group(1))
    wrf = {"citation": "mgpu.cu:513-646 (dev_convert), 682-706 (convertWRFChemData)",
           "var_src": [var_src[i] for i in range(nvar)], "jv_src": [jv_src[i] for i in range(nph)],
           "dims": {"ni": ni_, "nk": nk_, "nj": nj_},
           "window": {"i0": offs["i"], "k0": offs["k"], "j0": offs["j"], "wi": bx, "wk": gx, "wj": gy}}

    # Structural facts used by tests and the emitter.
    lower = sum(1 for s in range(lu_nonzero) if pattern["icol"][s] < pattern["irow"][s])
    upper = sum(1 for s in range(lu_nonzero) if pattern["icol"][s] > pattern["irow"][s])
    # (row, col) of each JVS slot must be consistent with the Fun RHS dependencies.
    out = {
        "source": "mgpu.cu (Rizkyanno/RADM2-Solver-Multi-GPU), extracted by mech/gen_mech.py",
        "citations": {
            "rconst": "mgpu.cu:763-918", "fun": "mgpu.cu:1103-1385", "jac": "mgpu.cu:1685-2652",
            "solve": "mgpu.cu:2873-3090", "decomp": "mgpu.cu:2746-2779", "ros3": "mgpu.cu:1007-1062",
            "species": "mgpu.cu:125-193", "photolysis": "mgpu.cu:52-79",
        },
        "sizes": {"NVAR": nvar, "NFIX": nfix, "NREACT": nreact, "LU_NONZERO": lu_nonzero,
                  "NONZERO": nonzero, "NPH": nph, "NB": max(bvals) + 1,
                  "n_lower": lower, "n_upper": upper},
        "species": [species[i] for i in range(nvar + nfix)],
        "photolysis": [photolysis[i] for i in range(nph)],
        "rconst": [rconst[i] for i in range(nreact)],
        "rates": [rates[i] for i in range(nreact)],
        "vdot": [vdot[i] for i in range(nvar)],
        "bvals": {str(k): bvals[k] for k in sorted(bvals)},
        "jvs": [jvs[i] for i in range(lu_nonzero)],
        "lu": pattern,
        "ros3": ros_tab,
        "wrf": wrf,
    }
    dst = os.path.join(HERE, "radm2_mech.json")
    with open(dst, "w") as f:
        json.dump(out, f, separators=(",", ":"))
        f.write("\n")
    print("wrote %s: %d rconst, %d rates, %d vdot, %d B, %d JVS, LU %d slots (%d lower, %d upper)"
          % (dst, len(rconst), len(rates), len(vdot), len(bvals), len(jvs), lu_nonzero, lower, upper))


if __name__ == "__main__":
    main()
