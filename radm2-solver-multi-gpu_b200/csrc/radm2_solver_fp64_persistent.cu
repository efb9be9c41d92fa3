// Instantiations of the fused solver kernel: fp64 LU, persistent schedule.
#include "radm2_solver_inst.h"

#define RADM2_T double
#define RADM2_S SCHED_PERSISTENT
RADM2_DEFINE_SOLVER(fp64_persistent, RADM2_VARIANTS_FP64_PERS)
