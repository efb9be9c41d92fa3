// Launch and query helpers shared by the solver instantiation files.  Each file
// instantiates one (precision, schedule) pair for a list of (block size, placement)
// combinations; combinations whose shared memory would exceed 227 KB are not built.
#pragma once

#include "radm2_internal.h"
#include "radm2_solver.cuh"

namespace radm2 {

template <int BS, typename LUT, int SCHED, int PLACE, int MINB, int IR, int ARITH>
cudaError_t launch_one(const SolveArgs &a, int grid, cudaStream_t st)
{
    auto k = k_rosenbrock<BS, LUT, SCHED, PLACE, MINB, IR, ARITH>;
    const size_t smem = (size_t)Layout<LUT, PLACE>::smem_words * sizeof(double) * BS;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    (void)cudaGetLastError();  // a stale error from another library is not this launch's
    k<<<grid, BS, smem, st>>>(a);
    return cudaGetLastError();
}

template <int BS, typename LUT, int SCHED, int PLACE, int MINB, int IR, int ARITH>
cudaError_t info_one(SolverInfo *out)
{
    auto k = k_rosenbrock<BS, LUT, SCHED, PLACE, MINB, IR, ARITH>;
    const size_t smem = (size_t)Layout<LUT, PLACE>::smem_words * sizeof(double) * BS;
    cudaFuncAttributes at{};
    cudaError_t e = cudaFuncGetAttributes(&at, k);
    if (e != cudaSuccess) return e;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    int blocks = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k, BS, smem);
    if (e != cudaSuccess) return e;
    // tensor-memory LU slots: 256 columns per 128 threads, 512 per SM
    if ((PLACE & PLACE_LU_TMEM) && blocks * (BS / 128) > 2) blocks = 2 / (BS / 128);
    if ((PLACE & PLACE_LU_TMEM_256) && blocks > 1) blocks = 1;  // all 512 columns per CTA
    out->regs = at.numRegs;
    out->local_bytes = (int)at.localSizeBytes;
    out->blocks_per_sm = blocks;
    out->global_words = Layout<LUT, PLACE>::global_words;
    out->smem_bytes = (int)smem;
    return cudaSuccess;
}

template <int BS, typename LUT, int SCHED, int PLACE, int MINB>
int check_one()
{
    return layout_check<LUT, PLACE>(BS);
}

}  // namespace radm2

// The built (block size, placement, min blocks) lists, RADM2_VARIANTS_FP64 / _FP32, are in
// radm2_internal.h (the autotuner walks them too).  An instantiation file sets RADM2_T
// (LU type), RADM2_S (schedule) and, for FP32 LU without the refinement code, RADM2_IR 0.
#ifndef RADM2_IR
#define RADM2_IR 1
#endif
// 1 in the files built in reference arithmetic (see k_rosenbrock's ARITH)
#ifndef RADM2_ARITH
#define RADM2_ARITH 0
#endif

#define RADM2_KEY(BS_, PL_, MB_) ((BS_) * 256 + (MB_) * 16 + (PL_))  // = variant_key
#define RADM2_CASE_LAUNCH(BS_, PL_, MB_) \
    case RADM2_KEY(BS_, PL_, MB_): return launch_one<BS_, RADM2_T, RADM2_S, PL_, MB_, RADM2_IR, RADM2_ARITH>(a, grid, st);
#define RADM2_CASE_INFO(BS_, PL_, MB_) \
    case RADM2_KEY(BS_, PL_, MB_): return info_one<BS_, RADM2_T, RADM2_S, PL_, MB_, RADM2_IR, RADM2_ARITH>(out);
#define RADM2_CHECK(BS_, PL_, MB_) bad |= check_one<BS_, RADM2_T, RADM2_S, PL_, MB_>();

#define RADM2_DEFINE_SOLVER(NAME, LIST)                                                                  \
    namespace radm2 {                                                                                    \
    cudaError_t launch_solver_##NAME(const SolveArgs &a, int key, int grid, cudaStream_t st)           \
    {                                                                                                    \
        switch (key) {                                                                       \
            LIST(RADM2_CASE_LAUNCH)                                                                      \
            default: return cudaErrorInvalidValue;                                                       \
        }                                                                                                \
    }                                                                                                    \
    cudaError_t solver_info_##NAME(int key, SolverInfo *out)                                            \
    {                                                                                                    \
        switch (key) {                                                                       \
            LIST(RADM2_CASE_INFO)                                                                        \
            default: return cudaErrorInvalidValue;                                                       \
        }                                                                                                \
    }                                                                                                    \
    int solver_layout_check_##NAME()                                                                     \
    {                                                                                                    \
        int bad = 0;                                                                                     \
        LIST(RADM2_CHECK)                                                                                \
        return bad;                                                                                      \
    }                                                                                                    \
    }
