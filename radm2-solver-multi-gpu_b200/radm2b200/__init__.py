"""B200 batched RADM2 Rosenbrock chemistry solver: Python host mirror.

    lib      ctypes binding of libradm2_b200.so (include/radm2.h)
    inputs   seeded synthetic cell inputs in the reference's per-cell layout
    seeding  step traces, training and use of the step-seeding network
"""
from . import inputs  # noqa: F401
from .lib import (NFIX, NJVS, NPH, NREACT, NVAR, PREC_FP32LU, PREC_FP64, SCHED_COOP, SCHED_PERSISTENT,  # noqa: F401
                  SCHED_STATIC, Mlp, RadmError, Solver, add_step_counters, default_params, fma_peak, load)
