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


def test_option_validation_before_device_lookup():
    """radm2_create checks its options before it looks for a device: on a machine without a
    GPU an invalid combination returns RADM2_E_ARG and a valid one RADM2_E_NODEV (with a GPU
    the valid ones create a context, covered by the GPU tests)."""
    import torch
    if torch.cuda.is_available():
        return
    lib = radm2b200.load()

    def create(**kw):
        o = rlib.Opts()
        lib.radm2_opts_default(ctypes.byref(o))
        for k, v in kw.items():
            setattr(o, k, v)
        h = ctypes.c_void_p()
        return lib.radm2_create(ctypes.byref(h), ctypes.byref(o))

    wide, pers = rlib.PLACE_LU_TMEM_WIDE, radm2b200.SCHED_PERSISTENT
    ok = [dict(placement=wide, schedule=pers), dict(placement=wide, schedule=pers, parity=1),
          dict(placement=rlib.PLACE_LU_TMEM), dict(placement=rlib.PLACE_LU_TMEM, parity=1)]
    bad = [dict(placement=wide), dict(placement=wide, schedule=radm2b200.SCHED_COOP),
           dict(placement=wide, schedule=pers, precision=radm2b200.PREC_FP32LU),
           dict(placement=wide, schedule=pers, cells_per_thread=2), dict(placement=7),
           dict(placement=rlib.PLACE_LU_TMEM, precision=radm2b200.PREC_FP32LU),
           dict(parity=1, placement=rlib.PLACE_LU_SMEM)]
    for kw in ok:
        assert create(**kw) == rlib.RADM2_E_NODEV, kw
    for kw in bad:
        assert create(**kw) == rlib.RADM2_E_ARG, kw
