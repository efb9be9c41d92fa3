// Instantiations of the fused solver kernel: fp64 LU, persistent schedule.
#include "radm2_solver_inst.h"

#define RADM2_T double
#define RADM2_S SCHED_PERSISTENT
RADM2_DEFINE_SOLVER(fp64_persistent, RADM2_VARIANTS_FP64)

#ifdef RADM2_PHASE_CLOCKS
// Profiling build only: read (and optionally clear) the per-warp phase cycle counters of
// this file's kernels.
extern "C" int radm2_phase_clocks(unsigned long long *out, int nwarps, int clear)
{
    const size_t bytes = sizeof(unsigned long long) * 8 * (size_t)nwarps;
    cudaError_t e = cudaMemcpyFromSymbol(out, radm2::phase_clocks, bytes);
    if (e == cudaSuccess && clear) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, radm2::phase_clocks);
        if (e == cudaSuccess) e = cudaMemset(p, 0, sizeof(radm2::phase_clocks));
    }
    return (int)e;
}
#endif
