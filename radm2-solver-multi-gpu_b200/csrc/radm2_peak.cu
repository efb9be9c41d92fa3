// CUDA-core FMA throughput microbenchmark: the FP64 / FP32 denominators of the
// solver's roofline (the solver runs on the CUDA cores, not the tensor cores).
// Every thread runs 8 independent FMA chains; the grid covers every SM several times.
#include <cuda_runtime.h>

#include "../../include/radm2.h"

namespace {

template <typename T>
__global__ void __launch_bounds__(256) k_fma_chains(int iters, T seed, T *sink)
{
    T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6,
      a7 = a0 + 7;
    const T m = (T)0.999999, c = (T)1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            a0 = a0 * m + c;
            a1 = a1 * m + c;
            a2 = a2 * m + c;
            a3 = a3 * m + c;
            a4 = a4 * m + c;
            a5 = a5 * m + c;
            a6 = a6 * m + c;
            a7 = a7 * m + c;
        }
    }
    const T s = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
    if (s == (T)-1) sink[0] = s;  // keeps the chains alive; never true
}

template <typename T>
double measure(int nsm, int iters)
{
    T *sink = nullptr;
    if (cudaMalloc(&sink, sizeof(T)) != cudaSuccess) return -1.0;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int blocks = nsm * 8, threads = 256;
    double best = 0.0;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        k_fma_chains<T><<<blocks, threads>>>(iters, (T)1.0, sink);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
        if (rep > 0 && ms > 0.f && flops / (ms * 1e-3) > best) best = flops / (ms * 1e-3);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(sink);
    return best * 1e-12;
}

}  // namespace

extern "C" int radm2_fma_peak(int device, double *fp64_tflops, double *fp32_tflops)
{
    if (!fp64_tflops || !fp32_tflops) return RADM2_E_ARG;
    cudaDeviceProp prop;
    if (cudaSetDevice(device) != cudaSuccess || cudaGetDeviceProperties(&prop, device) != cudaSuccess)
        return RADM2_E_NODEV;
    *fp64_tflops = measure<double>(prop.multiProcessorCount, 4096);
    *fp32_tflops = measure<float>(prop.multiProcessorCount, 8192);
    return (*fp64_tflops > 0 && *fp32_tflops > 0) ? RADM2_OK : RADM2_E_CUDA;
}
