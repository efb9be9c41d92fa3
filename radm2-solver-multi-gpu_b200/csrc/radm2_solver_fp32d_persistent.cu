// Instantiations of the fused solver kernel: fp32 LU without the refinement code (used
// when refine_sweeps = 0), persistent schedule.
#define RADM2_IR 0
#include "radm2_solver_inst.h"

#define RADM2_T float
#define RADM2_S SCHED_PERSISTENT
RADM2_DEFINE_SOLVER(fp32d_persistent, RADM2_VARIANTS_FP32)
