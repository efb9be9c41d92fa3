"""Per-phase cycle breakdown of the FP64 persistent solver kernel.

Uses the profiling build of the library (``make -C csrc phase`` builds
libradm2_b200_phase.so, the same kernels with clock64() counters around each phase)
and prints the share of warp cycles spent in each phase of a step attempt.

    python -m radm2b200.phase_profile [ncell]
"""
import ctypes
import os
import sys
import time

import numpy as np

from . import inputs
from . import lib as L

PHASES = ["cell load/store, time-loop test, Fcn0", "Jacobian -> G", "LU", "stage 1 solve",
          "stage 2 RHS + solve", "stage 3 solve", "error norm, step control"]


def main(ncell=1048576):
    L.LIB_PATH = os.path.join(os.path.dirname(L.LIB_PATH), "libradm2_b200_phase.so")
    lib = L.load()
    lib.radm2_phase_clocks.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    cells = inputs.make_cells(ncell, 1, "plain", 0.3)
    atol, rtol = np.ones(59), np.full(59, 1e-3)
    nw = 1 << 16
    buf = (ctypes.c_ulonglong * (8 * nw))()
    with L.Solver(schedule=L.SCHED_PERSISTENT, block_threads=128) as s:
        s.set_cells(cells)
        s.update_rconst()
        s.synchronize()
        lib.radm2_phase_clocks(buf, nw, 1)
        ipar, rpar = L.default_params(hstart=6.0)
        t = time.time()
        ierr = s.rosenbrock(0.0, 600.0, atol, rtol, rpar, ipar)
        dt = time.time() - t
        lib.radm2_phase_clocks(buf, nw, 0)
    a = np.frombuffer(buf, dtype=np.uint64).reshape(nw, 8).astype(np.float64)
    tot = a.sum(axis=0)
    print("ierr %d, %d cells, one 600 s split, %.1f ms (counters on)" % (ierr, ncell, dt * 1e3))
    for i, name in enumerate(PHASES):
        print("  %-40s %5.1f%%" % (name, 100.0 * tot[i] / tot[:7].sum()))


if __name__ == "__main__":
    main(int(sys.argv[1]) if len(sys.argv) > 1 else 1048576)
