"""Structural known-answer tests of the extracted mechanism and the emitted code."""
import json
import os
import subprocess
import sys

import numpy as np

from conftest import PKG, ROOT

MECH = os.path.join(PKG, "mech", "radm2_mech.json")

CROW = [0, 3, 9, 26, 29, 31, 33, 35, 37, 39, 41, 43, 46, 49, 52, 55, 57, 62, 66, 71, 75, 79, 84, 88, 92, 104, 120,
        124, 128, 132, 140, 148, 156, 170, 180, 187, 194, 204, 216, 229, 238, 245, 267, 298, 305, 318, 329, 343,
        368, 378, 393, 435, 464, 511, 541, 569, 586, 602, 625, 659]
DIAG = [0, 3, 9, 26, 29, 31, 33, 35, 37, 39, 41, 43, 46, 49, 52, 55, 57, 62, 67, 71, 75, 81, 84, 88, 94, 105, 120,
        124, 128, 132, 140, 149, 158, 170, 181, 188, 196, 208, 220, 230, 239, 252, 283, 299, 310, 323, 334, 356,
        370, 384, 426, 456, 504, 535, 564, 582, 599, 623, 658]


def mech():
    with open(MECH) as f:
        return json.load(f)


def test_sizes_and_counts():
    m = mech()
    s = m["sizes"]
    assert (s["NVAR"], s["NFIX"], s["NREACT"], s["LU_NONZERO"], s["NPH"]) == (59, 2, 156, 659, 28)
    assert (s["n_lower"], s["n_upper"]) == (304, 296)
    assert len(m["rconst"]) == 156 and len(m["rates"]) == 156 and len(m["vdot"]) == 59 and len(m["jvs"]) == 659
    # Jacobian partials B[0..279] with the gaps of derivatives w.r.t. fixed species.
    assert sorted(set(range(280)) - set(map(int, m["bvals"]))) == [22, 26, 28, 42, 48]


def test_lu_pattern():
    lu = mech()["lu"]
    assert lu["crow"] == CROW and lu["diag"] == DIAG
    icol = lu["icol"]
    for k in range(59):
        cols = icol[CROW[k]:CROW[k + 1]]
        assert cols == sorted(cols) and icol[DIAG[k]] == k
    # closed under row-Doolittle elimination
    for k in range(59):
        present = set(icol[CROW[k]:CROW[k + 1]])
        for kk in range(CROW[k], DIAG[k]):
            j = icol[kk]
            assert set(icol[DIAG[j] + 1:CROW[j + 1]]) <= present


def test_h2o2_quirk_is_kept():
    """Vdot[13] lacks -A[33] (H2O2 + OH) while the Jacobian keeps its terms (mgpu.cu:1275, 2011, 2013)."""
    m = mech()
    s = json.dumps(m["vdot"][13])
    assert '["ref", "A", 33]' not in s
    assert '["ref", "B", 43]' in json.dumps(m["jvs"][49]) and '["ref", "B", 44]' in json.dumps(m["jvs"][51])


def test_ros3_coefficients():
    r = mech()["ros3"]
    assert r["ros_S"] == 3 and r["ros_NewF"] == [1, 1, 0] and float(r["ros_ELO"]) == 3.0
    assert float(r["ros_Gamma"][0]) == 0.43586652150845899941601945119356
    assert float(r["ros_M"][1]) == 6.1697947043828245592553615689730


def test_emitted_code_is_current(tmp_path):
    """Re-emitting from the committed JSON reproduces the committed generated sources."""
    sys.path.insert(0, os.path.join(PKG, "mech"))
    import emit
    m = emit.load(MECH)
    emit.emit_cuda(m, str(tmp_path / "csrc"))
    emit.emit_oracle(m, str(tmp_path / "oracle"))
    for name in os.listdir(tmp_path / "csrc"):
        with open(tmp_path / "csrc" / name) as a, open(os.path.join(PKG, "csrc", "gen", name)) as b:
            assert a.read() == b.read(), name
    with open(tmp_path / "oracle" / "radm2_oracle_gen.c") as a, \
            open(os.path.join(ROOT, "oracle", "gen", "radm2_oracle_gen.c")) as b:
        assert a.read() == b.read()


def test_flop_counts():
    hdr = open(os.path.join(PKG, "csrc", "gen", "radm2_gen.h")).read()
    for key, val in (("FUN", 1085), ("JAC", 1272), ("DECOMP", 3588), ("SOLVE", 1259)):
        assert "#define RADM2_FLOPS_%s %d" % (key, val) in hdr
