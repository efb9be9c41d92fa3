"""The C-ABI library loads on a machine without a GPU and exports every function
declared in include/radm2.h (no compute calls here)."""
import ctypes
import os
import re

import radm2b200
from conftest import ROOT
from radm2b200 import lib as rlib


def declared_functions():
    text = open(os.path.join(ROOT, "include", "radm2.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\s*\**\s*(radm2_\w+)\s*\(", text, flags=re.M)))


def test_header_symbols_exported():
    names = declared_functions()
    assert len(names) >= 30
    lib = ctypes.CDLL(rlib.LIB_PATH)
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header():
    assert set(declared_functions()) <= set(rlib.SIGNATURES)


def test_no_device_is_reported_not_crashed():
    lib = radm2b200.load()
    assert lib.radm2_version().decode().startswith("radm2-b200")
    assert lib.radm2_error_string(-8).decode() == "Matrix is repeatedly singular"
    # without a GPU, context creation fails cleanly with an error code
    import torch
    if not torch.cuda.is_available():
        h = ctypes.c_void_p()
        rc = lib.radm2_create(ctypes.byref(h), None)
        assert rc == -104


def test_kernel_layouts_in_bounds():
    """Every built solver variant's per-thread working-set offsets fit its allocation
    (host-side arithmetic over the same layout constants the kernels use)."""
    assert radm2b200.load().radm2_selfcheck() == 0


def test_error_codes_match_header():
    text = open(os.path.join(ROOT, "include", "radm2.h")).read()
    codes = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define (RADM2_(?:OK|E_\w+))\s+\(?(-?\d+)\)?", text)}
    assert len(codes) == 7
    for name, val in codes.items():
        assert getattr(rlib, name) == val, name


def test_placement_constants_match_header():
    """RADM2_PLACE_* values agree between the header, the Python binding and the bench's
    --placement names."""
    import importlib.util
    text = open(os.path.join(ROOT, "include", "radm2.h")).read()
    places = {m.group(1): int(m.group(2)) for m in re.finditer(r"#define RADM2_(PLACE_\w+)\s+(\d+)", text)}
    assert places == {"PLACE_GLOBAL": 0, "PLACE_LU_SMEM": 1, "PLACE_ALL_SMEM": 3, "PLACE_LU_TMEM": 4,
                      "PLACE_LU_TMEM_WIDE": 10}
    for name, val in places.items():
        assert getattr(rlib, name) == val, name
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    assert set(bench.PLACEMENTS.values()) == set(places.values())
    assert set(bench.TMEM_NAMES) == {places["PLACE_LU_TMEM"], places["PLACE_LU_TMEM_WIDE"]}
