#!/usr/bin/env python3
"""Generate tests/golden/ref_mechanism.npz from the reference's own code.

Runs the reference harness (oracle/_ref/libradm2_ref.so: mgpu.cu's
dev_Update_RCONST, dev_Fun, dev_Jac_SP, dev_KppDecomp and dev_KppSolve compiled
for the CPU by oracle/build_ref.py) on 48 seeded cells and stores inputs and
outputs.  Needs the reference sources once, to build the harness; the
committed .npz does not.

Usage:  python oracle/build_ref.py && python tests/golden/make_golden.py
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
    cells = inputs.make_cells(48, 7, "mixed")
    crow, diag, icol = oracle.lu_tables()
    n = 48
    out = {k: [] for k in ("RCONST", "VDOT", "JVS", "G", "LU", "B", "X")}
    for c in range(n):
        rc = oracle.ref_rconst(cells["JV"][c], cells["FIX"][c], cells["RC_N2O5"][c], cells["TEMP"][c])
        V, F = cells["VAR"][c], cells["FIX"][c]
        vdot = oracle.ref_fun(V, F, rc)
        J = oracle.ref_jac(V, F, rc)
        G = -J
        G[diag] += 1.0 / (1.0 * (0.5 + c) * 0.43586652150845899941601945119356)
        LU, s = oracle.ref_decomp(G)
        assert s == 0
        X = oracle.ref_solve(LU, vdot)
        for k, v in zip(("RCONST", "VDOT", "JVS", "G", "LU", "B", "X"), (rc, vdot, J, G, LU, vdot, X)):
            out[k].append(v)
    arrays = {k: np.array(v) for k, v in out.items()}
    arrays.update({k: cells[k] for k in ("VAR", "FIX", "TEMP", "RC_N2O5", "JV")})
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "ref_mechanism.npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, {k: v.shape for k, v in arrays.items()})


if __name__ == "__main__":
    main()
