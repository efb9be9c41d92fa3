// Instantiations of the fused solver kernel in reference arithmetic (radm2_opts.parity):
// fp64 LU with the pivot divisions kept, built without multiply-add contraction
// (Makefile: -DRADM2_LU_RECIP=0 --fmad=false), persistent schedule.
#define RADM2_ARITH 1
#include "radm2_solver_inst.h"

#define RADM2_T double
#define RADM2_S SCHED_PERSISTENT
RADM2_DEFINE_SOLVER(fp64x_persistent, RADM2_VARIANTS_FP64X_PERS)
