// Instantiation of the cooperative solver kernel: 16 roles per block of 32 cells.
#define RADM2_COOP_G 16
#define RADM2_COOP_RECIP 1
#define RADM2_COOP_KERNEL k_rosenbrock_coop_g16
#include "radm2_internal.h"
#include "radm2_coop.cuh"

namespace radm2 {

cudaError_t launch_solver_coop_g16(const SolveArgs &a, int grid, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(k_rosenbrock_coop_g16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)COOP_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    (void)cudaGetLastError();  // a stale error from another library is not this launch's
    k_rosenbrock_coop_g16<<<grid, 32 * RADM2_COOP_G, COOP_SMEM_BYTES, st>>>(a);
    return cudaGetLastError();
}

cudaError_t solver_info_coop_g16(SolverInfo *out)
{
    cudaFuncAttributes at{};
    cudaError_t e = cudaFuncGetAttributes(&at, k_rosenbrock_coop_g16);
    if (e != cudaSuccess) return e;
    e = cudaFuncSetAttribute(k_rosenbrock_coop_g16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)COOP_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    int blocks = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, k_rosenbrock_coop_g16, 32 * RADM2_COOP_G, COOP_SMEM_BYTES);
    if (e != cudaSuccess) return e;
    out->regs = at.numRegs;
    out->local_bytes = (int)at.localSizeBytes;
    out->blocks_per_sm = blocks;
    out->global_words = 0;
    out->smem_bytes = (int)COOP_SMEM_BYTES;
    return cudaSuccess;
}

}  // namespace radm2
