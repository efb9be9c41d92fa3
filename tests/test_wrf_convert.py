"""WRF -> KPP conversion (mgpu.cu:513-646): the oracle against the reference's own
dev_convert (compiled for the CPU), bit for bit, and against the committed fixture."""
import os

import numpy as np
import pytest

import oracle
from radm2b200 import inputs

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "wrf_convert.npz")
KEYS = ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")


@pytest.fixture(scope="module")
def fields():
    return inputs.make_wrf_fields(5)


def test_oracle_matches_reference_dev_convert(fields):
    if not oracle.ref_available():
        pytest.skip("reference harness not built here")
    a, b = oracle.convert_wrf(fields), oracle.ref_convert_wrf(fields)
    for k in KEYS:
        assert np.array_equal(a[k], b[k]), k


def test_oracle_matches_golden_fixture():
    g = np.load(GOLDEN)
    f = inputs.make_wrf_fields(int(g["seed"]))
    out = oracle.convert_wrf(f)
    idx = g["cells"]
    for k in KEYS:
        assert np.array_equal(out[k][idx], g[k]), k


def test_conversion_semantics(fields):
    out = oracle.convert_wrf(fields)
    assert out["VAR"].shape == (39 * 19 * 39, 59)
    assert (out["VAR"] >= 0).all() and (out["VAR"] == 0).any()  # negative mixing ratios clamped
    # cell p = (j'*19 + k')*39 + i' reads point (i0+i', k0+k', j0+j')
    p = (7 * 19 + 3) * 39 + 11
    i, k, j = 4 + 11, 0 + 3, 4 + 7
    assert out["TEMP"][p] == fields["phy"][1, j, k, i]
    assert out["JV"][p, 5] == fields["ph"][5, j, k, i] / 60.0
    rho = fields["phy"][2, j, k, i]
    assert out["FIX"][p, 1] == (1.0e-3 * (1.0 / 28.97) * 6.022e23) * rho
    # a window of another grid converts the same points
    g2 = (48, 20, 48, 15, 3, 11, 1, 1, 1)
    one = oracle.convert_wrf(fields, g2)
    for key in KEYS:
        assert np.array_equal(one[key][0], out[key][p]), key


def test_reference_text_files_round_trip(tmp_path):
    from radm2b200 import wrf_io
    f = inputs.make_wrf_fields(9, ni=6, nk=3, nj=5)
    wrf_io.save_text_fields(f, str(tmp_path))
    g = wrf_io.load_text_fields(str(tmp_path), dims=(5, 3, 6))
    for k in ("ph", "chem", "rad", "phy", "moist"):
        assert np.array_equal(f[k], g[k]), k


def test_binary_fields_round_trip_and_text_conversion(tmp_path):
    """The binary form holds exactly the arrays of the text files (read, mapped, or
    converted from a text directory) and rejects a truncated or foreign file."""
    from radm2b200 import wrf_io
    f = inputs.make_wrf_fields(10, ni=6, nk=3, nj=5)
    keys = ("ph", "chem", "rad", "phy", "moist")
    wrf_io.save_binary_fields(f, str(tmp_path / "bin"))
    for mmap in (False, True):
        g = wrf_io.load_binary_fields(str(tmp_path / "bin"), mmap=mmap)
        for k in keys:
            assert g[k].shape == f[k].shape and np.array_equal(np.asarray(g[k]), f[k]), k
    wrf_io.save_text_fields(f, str(tmp_path / "txt"))
    wrf_io.text_to_binary(str(tmp_path / "txt"), str(tmp_path / "conv"), dims=(5, 3, 6))
    h = wrf_io.load_binary_fields(str(tmp_path / "conv"))
    for k in keys:
        assert np.array_equal(h[k], f[k]), k
    # the converted fields feed the conversion exactly like the originals
    grid = (5, 3, 6, 1, 0, 1, 3, 2, 3)
    a, b = oracle.convert_wrf(f, grid), oracle.convert_wrf(h, grid)
    for key in KEYS:
        assert np.array_equal(a[key], b[key]), key
    chem = tmp_path / "bin" / "wrfchem.bin"
    data = chem.read_bytes()
    chem.write_bytes(data[:-8])
    with pytest.raises(ValueError):
        wrf_io.load_binary_fields(str(tmp_path / "bin"))
    chem.write_bytes(b"NOTAWRF!" + data[8:])
    with pytest.raises(ValueError):
        wrf_io.load_binary_fields(str(tmp_path / "bin"))
