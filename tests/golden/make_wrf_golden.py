#!/usr/bin/env python3
"""Generate tests/golden/wrf_convert.npz from the reference's own dev_convert.

Runs the reference harness (oracle/_ref/libradm2_ref.so, built by oracle/build_ref.py
from mgpu.cu) on seeded WRF-like fields (radm2b200.inputs.make_wrf_fields, seed 5) over
the reference's 48 x 20 x 48 domain, and stores the outputs of 400 spread cells.  The
fields themselves are regenerated from the seed by the test.

Usage:  python oracle/build_ref.py && python tests/golden/make_wrf_golden.py
"""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "radm2-solver-multi-gpu_b200"))
import oracle  # noqa: E402
from radm2b200 import inputs  # noqa: E402


def main():
    seed = 5
    out = oracle.ref_convert_wrf(inputs.make_wrf_fields(seed))
    n = out["TEMP"].shape[0]
    cells = np.linspace(0, n - 1, 400).astype(np.int64)
    arrays = {k: out[k][cells] for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")}
    arrays.update(seed=np.int64(seed), cells=cells)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wrf_convert.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
