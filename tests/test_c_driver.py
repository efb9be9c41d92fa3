"""The C ABI from plain C: examples/c_driver.c compiles with gcc against include/radm2.h
and links against the library (CPU); on a GPU it integrates cells handed to it in the
reference's per-cell layout and matches the Python binding bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import radm2b200
from conftest import PKG, ROOT
from radm2b200 import inputs

SRC = os.path.join(PKG, "examples", "c_driver.c")


@pytest.fixture(scope="module")
def driver(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("c") / "c_driver")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-Wall", "-Werror", "-I", os.path.join(ROOT, "include"), SRC,
                           "-o", exe, "-L", PKG, "-lradm2_b200", "-Wl,-rpath," + PKG])
    return exe


def test_c_driver_builds_against_the_header(driver):
    assert os.access(driver, os.X_OK)


@pytest.mark.gpu
def test_c_driver_matches_python_binding(driver, tmp_path):
    cells = inputs.make_cells(3000, 31, "mixed")
    n = len(cells["TEMP"])
    fin, fout = str(tmp_path / "in.bin"), str(tmp_path / "out.bin")
    with open(fin, "wb") as f:
        f.write(np.int32(n).tobytes())
        for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV"):
            f.write(np.ascontiguousarray(cells[k], dtype=np.float64).tobytes())
    out = subprocess.run([driver, fin, fout], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    raw = open(fout, "rb").read()
    y_c = np.frombuffer(raw[:n * 59 * 8], dtype=np.float64).reshape(n, 59)
    ipar_c = np.frombuffer(raw[n * 59 * 8:], dtype=np.int32)
    with radm2b200.Solver(schedule=radm2b200.SCHED_PERSISTENT) as s:
        s.set_cells(cells)
        s.update_rconst()
        ipar, rpar = radm2b200.default_params(hstart=6.0)
        assert s.rosenbrock(0.0, 600.0, np.ones(59), np.full(59, 1e-3), rpar, ipar) == 1
        y = s.get_state()
    assert np.array_equal(y_c, y)
    assert list(ipar_c[10:17]) == list(ipar[10:17])
