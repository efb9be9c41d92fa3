// Instantiations of the fused solver kernel: fp32 LU, static schedule.
#include "radm2_solver_inst.h"

#define RADM2_T float
#define RADM2_S SCHED_STATIC
RADM2_DEFINE_SOLVER(fp32_static, RADM2_VARIANTS_FP32)
