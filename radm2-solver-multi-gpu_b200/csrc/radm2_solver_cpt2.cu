// Instantiations of the two-cells-per-thread solver kernel (radm2_solver_cpt2.cuh): FP64,
// global placement, 64 or 128 threads per block, both schedules.
#include "radm2_internal.h"
#include "radm2_solver_cpt2.cuh"

namespace radm2 {

namespace {

template <int BS, int SCHED>
cudaError_t launch_cpt2(const SolveArgs &a, int grid, cudaStream_t st)
{
    (void)cudaGetLastError();  // a stale error from another library is not this launch's
    k_rosenbrock_cpt2<BS, SCHED><<<grid, BS, 0, st>>>(a);
    return cudaGetLastError();
}

template <int BS, int SCHED>
cudaError_t info_cpt2(SolverInfo *out)
{
    cudaFuncAttributes at{};
    cudaError_t e = cudaFuncGetAttributes(&at, k_rosenbrock_cpt2<BS, SCHED>);
    if (e != cudaSuccess) return e;
    int blocks = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_rosenbrock_cpt2<BS, SCHED>, BS, 0);
    if (e != cudaSuccess) return e;
    out->regs = at.numRegs;
    out->local_bytes = (int)at.localSizeBytes;
    out->blocks_per_sm = blocks;
    out->global_words = 2 * Layout<double, PLACE_GLOBAL>::global_words;  // per thread: two cells
    out->smem_bytes = 0;
    return cudaSuccess;
}

}  // namespace

cudaError_t launch_solver_cpt2(const SolveArgs &a, int bs, int sched, int grid, cudaStream_t st)
{
    if (bs == 64) return sched ? launch_cpt2<64, SCHED_PERSISTENT>(a, grid, st) : launch_cpt2<64, SCHED_STATIC>(a, grid, st);
    if (bs == 128)
        return sched ? launch_cpt2<128, SCHED_PERSISTENT>(a, grid, st) : launch_cpt2<128, SCHED_STATIC>(a, grid, st);
    return cudaErrorInvalidValue;
}

cudaError_t solver_info_cpt2(int bs, int sched, SolverInfo *out)
{
    if (bs == 64) return sched ? info_cpt2<64, SCHED_PERSISTENT>(out) : info_cpt2<64, SCHED_STATIC>(out);
    if (bs == 128) return sched ? info_cpt2<128, SCHED_PERSISTENT>(out) : info_cpt2<128, SCHED_STATIC>(out);
    return cudaErrorInvalidValue;
}

int solver_layout_check_cpt2()
{
    // a block of BS threads is a virtual block of 2 x BS lanes on the thread-per-cell layout
    return layout_check<double, PLACE_GLOBAL>(128) | layout_check<double, PLACE_GLOBAL>(256);
}

}  // namespace radm2
