// Step-seeding network: features of each cell's state -> (log h0, log accepted steps).
//
// MLP 96 (84 features, zero padded) -> 128 -> 128 -> 128 -> 8 (2 outputs, zero padded),
// GELU hidden activations, BF16 weights and activations on the tensor cores with FP32
// accumulation, FP32 master weights and Adam moments.  Inference (k_forward_tc) issues
// tcgen05.mma with the accumulators in tensor memory; training (k_forward keeping the
// pre-activations, k_backward) uses mma.sync m16n8k16 tiles.  Forward and backward are
// fused over all four layers; weights live in shared memory (transposed, k contiguous).
#include <cuda_bf16.h>

#include <cstring>
#include <vector>

#include "../../include/radm2.h"
#include "radm2_internal.h"

namespace radm2 {
namespace mlp {

constexpr int NIN = 96, NFEAT = 84, W = 128, NOUT = 8, NY = 2;
constexpr int ROWS = 64;            // samples per CTA
constexpr int KP_IN = NIN + 8;      // padded k stride (bf16) for the input layer
constexpr int KP = W + 8;           // padded k stride for hidden layers
// parameter offsets (floats) in the flat master vector
constexpr int OFF_W1 = 0, OFF_B1 = OFF_W1 + NIN * W;
constexpr int OFF_W2 = OFF_B1 + W, OFF_B2 = OFF_W2 + W * W;
constexpr int OFF_W3 = OFF_B2 + W, OFF_B3 = OFF_W3 + W * W;
constexpr int OFF_W4 = OFF_B3 + W, OFF_B4 = OFF_W4 + W * NOUT;
constexpr int NPARAM = OFF_B4 + NOUT;

// Shared-memory image of the transposed bf16 weights: WT[n][k] with k contiguous.
constexpr int S_WT1 = 0;                     // W x KP_IN
constexpr int S_WT2 = S_WT1 + W * KP_IN;     // W x KP
constexpr int S_WT3 = S_WT2 + W * KP;        // W x KP
constexpr int S_WT4 = S_WT3 + W * KP;        // NOUT x KP
constexpr int S_WEND = S_WT4 + NOUT * KP;    // bf16 elements
constexpr int S_ACT = S_WEND;                // activations: ROWS x KP bf16 (x, h1, h2, h3 reuse)
constexpr int S_ACT2 = S_ACT + ROWS * KP;    // second activation buffer
constexpr int S_TOTAL = S_ACT2 + ROWS * KP;  // bf16 elements
constexpr int SMEM_BYTES = S_TOTAL * 2 + (W * 3 + NOUT) * 4 + NIN * 8;  // + biases + feature norm
// The forward kernel runs 12 warps per CTA (192 rows per tile) over the one staged weight
// image: 3x the warps of the training kernels, for latency hiding in the 1-CTA-per-SM
// footprint (98 KB of weights + 8.7 KB of activations per warp).
constexpr int FWD_WARPS = 12, FWD_ROWS = FWD_WARPS * 16;
constexpr int FS_ACT = S_WEND, FS_ACT2 = FS_ACT + FWD_ROWS * KP, FS_TOTAL = FS_ACT2 + FWD_ROWS * KP;
constexpr int FWD_SMEM_BYTES = FS_TOTAL * 2 + (W * 3 + NOUT) * 4 + NIN * 8;
static_assert(FWD_SMEM_BYTES <= 227 * 1024, "forward kernel shared memory");

__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi)
{
    __nv_bfloat162 v = __floats2bfloat162_rn(lo, hi);
    return *reinterpret_cast<uint32_t *>(&v);
}

__device__ __forceinline__ uint32_t ld32(const __nv_bfloat16 *p) { return *reinterpret_cast<const uint32_t *>(p); }

__device__ __forceinline__ uint32_t pack2(const __nv_bfloat16 *lo, const __nv_bfloat16 *hi)
{
    const uint32_t a = *reinterpret_cast<const unsigned short *>(lo);
    const uint32_t b = *reinterpret_cast<const unsigned short *>(hi);
    return a | (b << 16);
}

// D = A(16x16, row) * B(16x8, col) + C, bf16 inputs, fp32 accumulate.
__device__ __forceinline__ void mma16816(float *c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x)
{
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// Warp computes its 16 rows of Z = A(16 x K) * WT^T (K x N): acc[nt][4] for N/8 n-tiles.
// A: activation rows in smem (stride KA), WT: transposed weights (stride KW).
template <int K, int N>
__device__ __forceinline__ void warp_gemm(float (*acc)[4], const __nv_bfloat16 *A, int KA, const __nv_bfloat16 *WT,
                                          int KW)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int nt = 0; nt < N / 8; nt++) acc[nt][0] = acc[nt][1] = acc[nt][2] = acc[nt][3] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < K; k0 += 16) {
        const uint32_t a0 = ld32(A + g * KA + k0 + 2 * t);
        const uint32_t a1 = ld32(A + (g + 8) * KA + k0 + 2 * t);
        const uint32_t a2 = ld32(A + g * KA + k0 + 8 + 2 * t);
        const uint32_t a3 = ld32(A + (g + 8) * KA + k0 + 8 + 2 * t);
#pragma unroll
        for (int nt = 0; nt < N / 8; nt++) {
            const __nv_bfloat16 *w = WT + (nt * 8 + g) * KW + k0 + 2 * t;
            mma16816(acc[nt], a0, a1, a2, a3, ld32(w), ld32(w + 8));
        }
    }
}

struct Net {
    const float *params;          // fp32 master [NPARAM]
    const __nv_bfloat16 *wt;      // bf16 transposed weights image [S_WEND]
    const float *xmean, *xstd;    // feature normalisation [NIN]
};

// Stage the bf16 weight image, biases and feature normalisation into shared memory.
__device__ void load_net(const Net &net, __nv_bfloat16 *sw, float *sb, float *snorm)
{
    const uint4 *src = reinterpret_cast<const uint4 *>(net.wt);
    uint4 *dst = reinterpret_cast<uint4 *>(sw);
    for (int i = threadIdx.x; i < S_WEND / 8; i += blockDim.x) dst[i] = src[i];
    for (int i = threadIdx.x; i < W; i += blockDim.x) {
        sb[i] = net.params[OFF_B1 + i];
        sb[W + i] = net.params[OFF_B2 + i];
        sb[2 * W + i] = net.params[OFF_B3 + i];
    }
    for (int i = threadIdx.x; i < NOUT; i += blockDim.x) sb[3 * W + i] = net.params[OFF_B4 + i];
    for (int i = threadIdx.x; i < NIN; i += blockDim.x) {
        snorm[i] = net.xmean[i];
        snorm[NIN + i] = net.xstd[i];
    }
}

// Forward over all layers for the CTA's rows.  Saves pre-activations z1..z3 (fp32) and the
// outputs when the pointers are set (training).
__global__ void __launch_bounds__(FWD_WARPS * 32) k_forward(Net net, int n, const float *__restrict__ x,
                                                            float *__restrict__ y,
                                                 float *__restrict__ z1, float *__restrict__ z2,
                                                 float *__restrict__ z3)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16 *sw = reinterpret_cast<__nv_bfloat16 *>(smraw);
    float *sb = reinterpret_cast<float *>(smraw + FS_TOTAL * 2);
    float *snorm = sb + 3 * W + NOUT;
    load_net(net, sw, sb, snorm);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    __nv_bfloat16 *act = sw + FS_ACT + warp * 16 * KP;  // this warp's 16 rows
    __nv_bfloat16 *act2 = sw + FS_ACT2 + warp * 16 * KP;
    const int ntiles = (n + FWD_ROWS - 1) / FWD_ROWS;
    // the weights are staged once per CTA; the CTA walks row tiles
#pragma unroll 1
    for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
    const int row0 = tile * FWD_ROWS + warp * 16;
    __syncwarp();
    // normalised inputs -> bf16
    for (int i = lane; i < 16 * NIN; i += 32) {
        const int r = i / NIN, k = i % NIN, gr = row0 + r;
        float v = 0.f;
        if (gr < n && k < NFEAT) v = (x[(size_t)gr * NFEAT + k] - snorm[k]) / snorm[NIN + k];
        act[r * KP + k] = __float2bfloat16_rn(v);
    }
    __syncwarp();
    float acc[16][4];
    float *zs[3] = {z1, z2, z3};
    const __nv_bfloat16 *wts[3] = {sw + S_WT1, sw + S_WT2, sw + S_WT3};
    const int kws[3] = {KP_IN, KP, KP};
#pragma unroll 1
    for (int l = 0; l < 3; l++) {
        __nv_bfloat16 *in = (l & 1) ? act2 : act;
        __nv_bfloat16 *out = (l & 1) ? act : act2;
        if (l == 0)
            warp_gemm<NIN, W>(acc, in, KP, wts[0], kws[0]);
        else
            warp_gemm<W, W>(acc, in, KP, wts[l], kws[l]);
        __syncwarp();
#pragma unroll
        for (int nt = 0; nt < 16; nt++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = g + 8 * h, c = nt * 8 + 2 * t, gr = row0 + r;
                const float v0 = acc[nt][2 * h] + sb[l * W + c], v1 = acc[nt][2 * h + 1] + sb[l * W + c + 1];
                if (zs[l] && gr < n) {
                    zs[l][(size_t)gr * W + c] = v0;
                    zs[l][(size_t)gr * W + c + 1] = v1;
                }
                *reinterpret_cast<uint32_t *>(out + r * KP + c) = pack_bf16(gelu(v0), gelu(v1));
            }
        }
        __syncwarp();
    }
    // output layer: h3 is in act2 (l = 2 wrote `out` = act2)
    float acc4[1][4];
    warp_gemm<W, NOUT>(acc4, act2, KP, sw + S_WT4, KP);
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int r = g + 8 * h, c = 2 * t, gr = row0 + r;
        if (gr < n && c < NY) {
            y[(size_t)gr * NY + c] = acc4[0][2 * h] + sb[3 * W + c];
            if (c + 1 < NY) y[(size_t)gr * NY + c + 1] = acc4[0][2 * h + 1] + sb[3 * W + c + 1];
        }
    }
    }  // tiles
}

// dW[m][nn] += sum over the warp's 16 rows of A[row][m] * B[row][nn]  (A^T B, K = 16 rows).
// A rows in smem (stride KA, M columns), B rows in smem (stride KB, NN columns); the
// products are accumulated into the fp32 gradient (global atomics).
template <int M, int NN>
__device__ __forceinline__ void warp_outer(float *grad, int ldg, const __nv_bfloat16 *A, int KA,
                                           const __nv_bfloat16 *B, int KB, int nvalid)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll 1
    for (int mt = 0; mt < M / 16; mt++) {
        // A' = A^T: (m, k=row) -> A[row][m]
        const int m0 = mt * 16 + g, m1 = m0 + 8;
        const uint32_t a0 = pack2(A + (2 * t) * KA + m0, A + (2 * t + 1) * KA + m0);
        const uint32_t a1 = pack2(A + (2 * t) * KA + m1, A + (2 * t + 1) * KA + m1);
        const uint32_t a2 = pack2(A + (2 * t + 8) * KA + m0, A + (2 * t + 9) * KA + m0);
        const uint32_t a3 = pack2(A + (2 * t + 8) * KA + m1, A + (2 * t + 9) * KA + m1);
#pragma unroll 4
        for (int nt = 0; nt < NN / 8; nt++) {
            const int nn = nt * 8 + g;
            const uint32_t b0 = pack2(B + (2 * t) * KB + nn, B + (2 * t + 1) * KB + nn);
            const uint32_t b1 = pack2(B + (2 * t + 8) * KB + nn, B + (2 * t + 9) * KB + nn);
            float c[4] = {0.f, 0.f, 0.f, 0.f};
            mma16816(c, a0, a1, a2, a3, b0, b1);
            const int col = nt * 8 + 2 * t;
            if (col < nvalid) {
                atomicAdd(&grad[(size_t)(mt * 16 + g) * ldg + col], c[0]);
                atomicAdd(&grad[(size_t)(mt * 16 + g + 8) * ldg + col], c[2]);
            }
            if (col + 1 < nvalid) {
                atomicAdd(&grad[(size_t)(mt * 16 + g) * ldg + col + 1], c[1]);
                atomicAdd(&grad[(size_t)(mt * 16 + g + 8) * ldg + col + 1], c[3]);
            }
        }
    }
}

// dH (16 x M) = dZ (16 x NN) * W^T where W is [M][NN] (stored transposed: WT[NN][M]).
template <int NN, int M>
__device__ __forceinline__ void warp_gemm_wt(float (*acc)[4], const __nv_bfloat16 *dZ, int KZ,
                                             const __nv_bfloat16 *WT, int KW)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
#pragma unroll
    for (int mt = 0; mt < M / 8; mt++) acc[mt][0] = acc[mt][1] = acc[mt][2] = acc[mt][3] = 0.f;
#pragma unroll
    for (int k0 = 0; k0 < NN; k0 += 16) {
        const uint32_t a0 = ld32(dZ + g * KZ + k0 + 2 * t);
        const uint32_t a1 = ld32(dZ + (g + 8) * KZ + k0 + 2 * t);
        const uint32_t a2 = ld32(dZ + g * KZ + k0 + 8 + 2 * t);
        const uint32_t a3 = ld32(dZ + (g + 8) * KZ + k0 + 8 + 2 * t);
#pragma unroll
        for (int mt = 0; mt < M / 8; mt++) {
            // B(k = j, n = i) = W[i][j] = WT[j][i]
            const int i = mt * 8 + g;
            const uint32_t b0 = pack2(WT + (k0 + 2 * t) * KW + i, WT + (k0 + 2 * t + 1) * KW + i);
            const uint32_t b1 = pack2(WT + (k0 + 2 * t + 8) * KW + i, WT + (k0 + 2 * t + 9) * KW + i);
            mma16816(acc[mt], a0, a1, a2, a3, b0, b1);
        }
    }
}

// ---------------------------------------------------------------- tcgen05 forward
// The inference forward on the 5th-generation tensor cores.  A CTA holds the transposed
// weights once in shared memory and runs TC_G independent tile pipelines (4 warps each,
// 128 rows per tile): per layer, one thread issues K/16 `tcgen05.mma.kind::f16`
// (BF16 x BF16 -> FP32) with A = the tile's activations and B = the weights, both in the
// canonical K-major no-swizzle layout, and D = a 128 x N FP32 accumulator in the pipeline's
// 128 tensor-memory columns (lane = row).  `tcgen05.commit` arms the pipeline's mbarrier;
// the epilogue reads D back with `tcgen05.ld` (warp w: lanes 32(w%4)..+31), adds the bias,
// applies GELU and writes the next layer's BF16 activations in place (the MMA that read
// them has completed).  While one pipeline waits on its MMAs the others run their
// epilogues.  Every wait is bounded and reports through *err.
//
// Canonical K-major layout (no swizzle): element (r, k) of an [R][K] BF16 operand at byte
// ((r / 8) * (K / 8) + k / 8) * 128 + (r % 8) * 16 + (k % 8) * 2: 8 x 16-byte core matrices,
// K-adjacent ones 128 B apart (leading byte offset), 8-row groups K * 16 B apart (stride
// byte offset).
constexpr int TC_M = 128;                      // tile rows = TMEM lanes
constexpr int TC_G = 4;                        // tile pipelines per CTA (4 warps each)
constexpr int TC_THREADS = TC_G * TC_M;
constexpr int TC_N4 = 16;                      // output layer N (2 outputs, padded)
constexpr int TB_W1 = 0;                       // W1^T [128][96]
constexpr int TB_W2 = TB_W1 + W * NIN * 2;     // W2^T [128][128]
constexpr int TB_W3 = TB_W2 + W * W * 2;       // W3^T [128][128]
constexpr int TB_W4 = TB_W3 + W * W * 2;       // W4^T [16][128]
constexpr int TB_ACT = TB_W4 + TC_N4 * W * 2;  // per pipeline: activations [128][128] (layer 1 reads k < 96)
constexpr int TB_BIAS = TB_ACT + TC_G * TC_M * W * 2;  // floats: 3 x 128 + 8
constexpr int TB_NORM = TB_BIAS + (3 * W + NOUT) * 4;  // floats: mean[96], std[96]
constexpr int TB_MBAR = TB_NORM + 2 * NIN * 4;         // per pipeline, 8 bytes
constexpr int TB_TMEM = TB_MBAR + 8 * TC_G;
constexpr int TB_FLAG = TB_TMEM + 4;                   // per pipeline: a wait gave up
constexpr int TC_SMEM = TB_FLAG + 4 * TC_G;
constexpr int TC_TMEM_COLS = 128 * TC_G;
constexpr long TC_WAIT_LIMIT = 1L << 22;         // try_wait rounds before a wait gives up
constexpr long long TC_WAIT_CYCLES = 4000000000LL;  // and SM cycles (~2 s): a try_wait round
                                                    // may suspend for a hardware-defined time
static_assert(TB_ACT % 16 == 0 && TB_W2 % 16 == 0 && TB_W4 % 16 == 0 && TB_MBAR % 8 == 0, "operand alignment");
static_assert(TC_SMEM <= 227 * 1024, "tcgen05 forward shared memory");
static_assert(TC_TMEM_COLS <= 512, "tensor memory columns");
static_assert(NFEAT % 4 == 0 && NIN % 8 == 0, "feature rows in 16-byte groups");

__host__ __device__ constexpr int canon_off(int r, int k, int K)
{
    return ((r >> 3) * (K >> 3) + (k >> 3)) * 128 + (r & 7) * 16 + (k & 7) * 2;
}

// Shared-memory matrix descriptor: start, leading (K) and stride (8-row) byte offsets in
// 16-byte units, descriptor version 1, no swizzle.
__host__ __device__ constexpr uint64_t umma_desc(uint32_t saddr, int K)
{
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((128 >> 4) & 0x3FFF) << 16) |
           ((uint64_t)(((K / 8) * 128 >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// Instruction descriptor: FP32 accumulator, BF16 A and B, both K-major, M x N.
__host__ __device__ constexpr uint32_t umma_idesc(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

// Last byte a K=16 MMA step reads from an operand of `rows` rows laid out with extent K:
// 8-row groups at stride K*16 B, two K-adjacent core matrices 128 B apart, 8 rows of 16 B.
__host__ __device__ constexpr int umma_last_byte(int step, int rows, int K)
{
    return step * 256 + (rows / 8 - 1) * (K / 8) * 128 + 128 + 7 * 16 + 15;
}
static_assert(umma_last_byte(W / 16 - 1, TC_M, W) < TC_M * W * 2, "A operand inside its buffer");
static_assert(umma_last_byte(NIN / 16 - 1, W, NIN) < W * NIN * 2, "W1 operand inside its buffer");
static_assert(umma_last_byte(W / 16 - 1, W, W) < W * W * 2, "W2/W3 operand inside its buffer");
static_assert(umma_last_byte(W / 16 - 1, TC_N4, W) < TC_N4 * W * 2, "W4 operand inside its buffer");

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem_d),
        "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t phase, long limit)
{
    const long long t0 = clock64();
    for (long it = 0; it < limit && clock64() - t0 < TC_WAIT_CYCLES; it++) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, P1;\n\t}\n"
            : "=r"(ok)
            : "r"(addr), "r"(phase)
            : "memory");
        if (ok) return true;
    }
    return false;
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory"); }
// barrier of one tile pipeline's 4 warps (named barrier 1 + g)
__device__ __forceinline__ void group_sync(int g) { asm volatile("bar.sync %0, %1;\n" ::"r"(1 + g), "r"(TC_M) : "memory"); }

// Copy a transposed weight matrix WT[rows][k < kvalid] (row stride ks, bf16) into the
// canonical layout [rows_pad][K]; rows and columns beyond the source are zero.
__device__ void stage_canon(unsigned char *dst, const __nv_bfloat16 *src, int rows, int rows_pad, int kvalid, int ks,
                            int K)
{
    for (int i = threadIdx.x; i < rows_pad * (K / 8); i += blockDim.x) {
        const int r = i / (K / 8), k0 = (i % (K / 8)) * 8;
        uint4 v = make_uint4(0, 0, 0, 0);
        if (r < rows && k0 < kvalid) v = *reinterpret_cast<const uint4 *>(src + (size_t)r * ks + k0);
        *reinterpret_cast<uint4 *>(dst + canon_off(r, k0, K)) = v;
    }
}

// wait_limit bounds every mbarrier wait (TC_WAIT_LIMIT in production).  idle != 0 is the
// self-test of that bound: no tensor-core work is issued or committed, so the first wait of
// every pipeline runs out, raises *err and the kernel returns with nothing in flight.
__global__ void __launch_bounds__(TC_THREADS) k_forward_tc(Net net, int n, const float *__restrict__ x,
                                                          float *__restrict__ y, int *__restrict__ err,
                                                          long wait_limit, int idle)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    float *sb = reinterpret_cast<float *>(sm + TB_BIAS);
    float *snorm = reinterpret_cast<float *>(sm + TB_NORM);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + TB_TMEM);
    const int tid = threadIdx.x, warp = tid >> 5;
    const int g = warp >> 2, gt = tid & (TC_M - 1);  // pipeline, thread within it (= tile row)
    volatile int *gflag = reinterpret_cast<volatile int *>(sm + TB_FLAG) + g;
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(sm);
    const uint32_t mbar = sbase + TB_MBAR + 8 * g;
    unsigned char *act = sm + TB_ACT + g * (TC_M * W * 2);
    const uint32_t act_s = sbase + TB_ACT + g * (TC_M * W * 2);

    // weights (canonical, once per CTA), biases, normalisation
    stage_canon(sm + TB_W1, net.wt + S_WT1, W, W, NIN, KP_IN, NIN);
    stage_canon(sm + TB_W2, net.wt + S_WT2, W, W, W, KP, W);
    stage_canon(sm + TB_W3, net.wt + S_WT3, W, W, W, KP, W);
    stage_canon(sm + TB_W4, net.wt + S_WT4, NOUT, TC_N4, W, KP, W);
    for (int i = tid; i < W; i += blockDim.x) {
        sb[i] = net.params[OFF_B1 + i];
        sb[W + i] = net.params[OFF_B2 + i];
        sb[2 * W + i] = net.params[OFF_B3 + i];
    }
    for (int i = tid; i < NOUT; i += blockDim.x) sb[3 * W + i] = net.params[OFF_B4 + i];
    for (int i = tid; i < NIN; i += blockDim.x) {
        snorm[i] = net.xmean[i];
        snorm[NIN + i] = net.xstd[i];
    }
    if (gt == 0) {
        *gflag = 0;
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(mbar) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
    // one warp owns the tensor-memory allocation; the shared-memory footprint keeps one CTA
    // per SM and no other kernel of the library uses tensor memory, so the 512 columns are free
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(sbase + TB_TMEM),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
    }
    proxy_fence();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tmem_slot + (uint32_t)(128 * g);            // this pipeline's columns
    const uint32_t trow = tmem + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's lanes
    uint32_t phase = 0;
    const uint32_t idesc_h = umma_idesc(TC_M, W), idesc_o = umma_idesc(TC_M, TC_N4);
    const int ntiles = (n + TC_M - 1) / TC_M;
    const bool xvec = (reinterpret_cast<uintptr_t>(x) & 15) == 0;

#pragma unroll 1
    for (int tile = blockIdx.x * TC_G + g; tile < ntiles && !*gflag; tile += gridDim.x * TC_G) {
        const int row0 = tile * TC_M;
        // normalised inputs -> bf16 activations (k < 96; features >= 84 are zero)
        for (int i = gt; i < TC_M * (NIN / 8); i += TC_M) {
            const int r = i / (NIN / 8), k0 = (i % (NIN / 8)) * 8, gr = row0 + r;
            float v[8];
#pragma unroll
            for (int q = 0; q < 2; q++) {  // rows are NFEAT * 4 = 336 bytes: 16-byte groups stay aligned
                const int k = k0 + 4 * q;
                float4 f = make_float4(0.f, 0.f, 0.f, 0.f);
                if (gr < n && k < NFEAT) {
                    if (xvec) {
                        f = __ldg(reinterpret_cast<const float4 *>(x + (size_t)gr * NFEAT + k));
                    } else {
                        const float *xs = x + (size_t)gr * NFEAT + k;
                        f = make_float4(xs[0], xs[1], xs[2], xs[3]);
                    }
                }
                v[4 * q] = f.x, v[4 * q + 1] = f.y, v[4 * q + 2] = f.z, v[4 * q + 3] = f.w;
            }
            uint32_t pk[4];
#pragma unroll
            for (int h = 0; h < 4; h++) {
                const int k = k0 + 2 * h;
                pk[h] = k < NFEAT ? pack_bf16((v[2 * h] - snorm[k]) / snorm[NIN + k],
                                              (v[2 * h + 1] - snorm[k + 1]) / snorm[NIN + k + 1])
                                  : 0u;
            }
            *reinterpret_cast<uint4 *>(act + canon_off(r, k0, W)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        }
        proxy_fence();
        group_sync(g);
#pragma unroll 1
        for (int l = 0; l < 4; l++) {
            const int K = l == 0 ? NIN : W;
            const uint32_t b_off = l == 0 ? TB_W1 : l == 1 ? TB_W2 : l == 2 ? TB_W3 : TB_W4;
            if (gt == 0 && !idle) {
                tc_fence_after();
#pragma unroll 1
                for (int s = 0; s < K / 16; s++)
                    umma_bf16(tmem, umma_desc(act_s + s * 256, W), umma_desc(sbase + b_off + s * 256, K),
                              l < 3 ? idesc_h : idesc_o, s > 0 ? 1u : 0u);
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                                 mbar)
                             : "memory");
            }
            if (!mbar_wait(mbar, phase, wait_limit)) *gflag = 1;
            group_sync(g);  // one decision for the pipeline
            if (*gflag) break;
            phase ^= 1u;
            tc_fence_after();
            if (l < 3) {  // bias + GELU -> bf16 activations of the next layer, in place
#pragma unroll 1
                for (int c0 = 0; c0 < W; c0 += 16) {
                    float v[16];
                    tmem_ld16(trow + c0, v);
                    uint32_t pk[8];
#pragma unroll
                    for (int h = 0; h < 8; h++)
                        pk[h] = pack_bf16(gelu(v[2 * h] + sb[l * W + c0 + 2 * h]),
                                          gelu(v[2 * h + 1] + sb[l * W + c0 + 2 * h + 1]));
                    *reinterpret_cast<uint4 *>(act + canon_off(gt, c0, W)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
                    *reinterpret_cast<uint4 *>(act + canon_off(gt, c0 + 8, W)) =
                        make_uint4(pk[4], pk[5], pk[6], pk[7]);
                }
            } else {  // outputs
                float v[16];
                tmem_ld16(trow, v);
                const int gr = row0 + gt;
                if (gr < n) {
                    y[(size_t)gr * NY] = v[0] + sb[3 * W];
                    y[(size_t)gr * NY + 1] = v[1] + sb[3 * W + 1];
                }
            }
            tc_fence_before();
            proxy_fence();
            group_sync(g);
        }
    }
    if (*gflag) {
        if (gt == 0) atomicExch(err, 1);
        // a wait that gave up may leave tensor-core work in flight: give it a bounded chance
        // to finish before the accumulator memory is released
        mbar_wait(mbar, phase, wait_limit);
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(*tmem_slot), "r"(TC_TMEM_COLS)
                     : "memory");
}

// Backward for MSE loss mean over (n x NY): fills grad[NPARAM] (atomic sums over CTAs) and
// adds the CTA's loss partial to *loss.
__global__ void __launch_bounds__(128) k_backward(Net net, int n, const float *__restrict__ x,
                                                  const float *__restrict__ y, const float *__restrict__ target,
                                                  const float *__restrict__ z1, const float *__restrict__ z2,
                                                  const float *__restrict__ z3, float *__restrict__ grad,
                                                  float *__restrict__ loss)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    __nv_bfloat16 *sw = reinterpret_cast<__nv_bfloat16 *>(smraw);
    float *sb = reinterpret_cast<float *>(smraw + S_TOTAL * 2);
    float *snorm = sb + 3 * W + NOUT;
    load_net(net, sw, sb, snorm);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int row0 = blockIdx.x * ROWS + warp * 16;
    __nv_bfloat16 *hb = sw + S_ACT + warp * 16 * KP;   // activation of the layer below (A^T of dW)
    __nv_bfloat16 *db = sw + S_ACT2 + warp * 16 * KP;  // upstream gradient dZ (bf16)
    const float scale = 2.0f / (float)(n * NY);
    // dY (16 x 8, 2 valid) -> db; loss partial
    float lpart = 0.f;
    for (int i = lane; i < 16 * 16; i += 32) {
        const int r = i / 16, c = i % 16, gr = row0 + r;
        float d = 0.f;
        if (gr < n && c < NY) {
            const float e = y[(size_t)gr * NY + c] - target[(size_t)gr * NY + c];
            lpart += e * e;
            d = scale * e;
        }
        db[r * KP + c] = __float2bfloat16_rn(d);
    }
    for (int o = 16; o > 0; o >>= 1) lpart += __shfl_down_sync(0xffffffffu, lpart, o);
    if (lane == 0) atomicAdd(loss, lpart / (float)(n * NY));
    // h3 = gelu(z3) -> hb
    const float *zs[3] = {z1, z2, z3};
    auto load_h = [&](int l) {  // hb = gelu(z_l) (l = 0..2), or the normalised input (l = -1)
        if (l < 0) {
            for (int i = lane; i < 16 * NIN; i += 32) {
                const int r = i / NIN, k = i % NIN, gr = row0 + r;
                float v = 0.f;
                if (gr < n && k < NFEAT) v = (x[(size_t)gr * NFEAT + k] - snorm[k]) / snorm[NIN + k];
                hb[r * KP + k] = __float2bfloat16_rn(v);
            }
        } else {
            for (int i = lane; i < 16 * W; i += 32) {
                const int r = i / W, k = i % W, gr = row0 + r;
                const float v = gr < n ? gelu(zs[l][(size_t)gr * W + k]) : 0.f;
                hb[r * KP + k] = __float2bfloat16_rn(v);
            }
        }
    };
    load_h(2);
    __syncwarp();
    // layer 4: dW4 = h3^T dY (128 x 8, 2 valid columns), db4 = sum dY
    warp_outer<W, NOUT>(grad + OFF_W4, NOUT, hb, KP, db, KP, NY);
    if (lane < NY) {
        float s = 0.f;
        for (int r = 0; r < 16; r++) s += __bfloat162float(db[r * KP + lane]);
        atomicAdd(&grad[OFF_B4 + lane], s);
    }
    // dH3 = dY W4^T  (K = 8 padded to 16: db columns 8..15 are zero)
    float acc[16][4];
    {
        // W4^T stored as WT4[NOUT][KP] (n = out, k = in): B(k = j out, n = i in) = WT4[j][i]
        const __nv_bfloat16 *WT4 = sw + S_WT4;
        const uint32_t a0 = ld32(db + g * KP + 2 * t), a1 = ld32(db + (g + 8) * KP + 2 * t);
        const uint32_t a2 = ld32(db + g * KP + 8 + 2 * t), a3 = ld32(db + (g + 8) * KP + 8 + 2 * t);
#pragma unroll
        for (int mt = 0; mt < 16; mt++) {
            acc[mt][0] = acc[mt][1] = acc[mt][2] = acc[mt][3] = 0.f;
            const int i = mt * 8 + g;
            const int j0 = 2 * t, j1 = 2 * t + 1;  // k rows 0..7 real, 8..15 zero
            const uint32_t b0 = pack2(WT4 + j0 * KP + i, WT4 + j1 * KP + i);
            mma16816(acc[mt], a0, a1, a2, a3, b0, 0u);
        }
    }
    // hidden layers 3, 2, 1
    const int offW[3] = {OFF_W1, OFF_W2, OFF_W3}, offB[3] = {OFF_B1, OFF_B2, OFF_B3};
    const __nv_bfloat16 *wts[3] = {sw + S_WT1, sw + S_WT2, sw + S_WT3};
#pragma unroll 1
    for (int l = 2; l >= 0; l--) {
        __syncwarp();
        // dZ_l = dH_l * gelu'(z_l) -> db (bf16); db_l bias gradient
#pragma unroll
        for (int mt = 0; mt < 16; mt++) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = g + 8 * h, c = mt * 8 + 2 * t, gr = row0 + r;
                float d0 = 0.f, d1 = 0.f;
                if (gr < n) {
                    d0 = acc[mt][2 * h] * gelu_grad(zs[l][(size_t)gr * W + c]);
                    d1 = acc[mt][2 * h + 1] * gelu_grad(zs[l][(size_t)gr * W + c + 1]);
                }
                *reinterpret_cast<uint32_t *>(db + r * KP + c) = pack_bf16(d0, d1);
            }
        }
        __syncwarp();
        for (int c = lane; c < W; c += 32) {
            float s = 0.f;
            for (int r = 0; r < 16; r++) s += __bfloat162float(db[r * KP + c]);
            atomicAdd(&grad[offB[l] + c], s);
        }
        // h_{l-1} (or the input) -> hb; dW_l = h_{l-1}^T dZ_l
        load_h(l - 1);
        __syncwarp();
        if (l == 0)
            warp_outer<NIN, W>(grad + offW[0], W, hb, KP, db, KP, W);
        else
            warp_outer<W, W>(grad + offW[l], W, hb, KP, db, KP, W);
        if (l > 0) {
            // dH_{l-1} = dZ_l W_l^T
            warp_gemm_wt<W, W>(acc, db, KP, wts[l], KP);
        }
    }
}

// Adam on the fp32 master weights; refreshes the bf16 transposed image and clears grad.
__global__ void k_adam(int np, float *__restrict__ p, float *__restrict__ g, float *__restrict__ m,
                       float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= np) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    g[i] = 0.f;
}

// bf16 transposed weight image WT_l[n][k] from the fp32 master W_l[k][n].
__global__ void k_pack_weights(const float *__restrict__ p, __nv_bfloat16 *__restrict__ wt)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= S_WEND) return;
    float v = 0.f;
    if (i < S_WT2) {
        const int nn = i / KP_IN, k = i % KP_IN;
        if (k < NIN) v = p[OFF_W1 + k * W + nn];
    } else if (i < S_WT3) {
        const int j = i - S_WT2, nn = j / KP, k = j % KP;
        if (k < W) v = p[OFF_W2 + k * W + nn];
    } else if (i < S_WT4) {
        const int j = i - S_WT3, nn = j / KP, k = j % KP;
        if (k < W) v = p[OFF_W3 + k * W + nn];
    } else {
        const int j = i - S_WT4, nn = j / KP, k = j % KP;
        if (k < W) v = p[OFF_W4 + k * NOUT + nn];
    }
    wt[i] = __float2bfloat16_rn(v);
}

// Features of each cell's current state (SoA cell arrays of a context).
// Features of a block of cells are formed in shared memory and written out as one
// contiguous run of the row-major feature matrix (coalesced stores).
constexpr int FEAT_BLOCK = 128, FEAT_PAD = NFEAT + 1;
__global__ void __launch_bounds__(FEAT_BLOCK) k_features(int n, int ld, const double *__restrict__ var,
                                                         const double *__restrict__ fix,
                                                         const double *__restrict__ temp,
                                                         const double *__restrict__ jv, float dt,
                                                         float *__restrict__ f)
{
    __shared__ float sf[FEAT_BLOCK * FEAT_PAD];
    const int c0 = blockIdx.x * FEAT_BLOCK, c = c0 + threadIdx.x;
    float *o = sf + threadIdx.x * FEAT_PAD;
    if (c < n) {
        for (int i = 0; i < NVAR; i++) o[i] = (float)log10(fmax(var[(size_t)i * ld + c], 1.0e-3));
        o[59] = (float)temp[c];
        o[60] = (float)log10(fmax(fix[(size_t)ld + c], 1.0));
        o[61] = (float)log10(fmax(fix[c], 1.0));
        for (int k = 0; k < RADM2_NJV_USED; k++) o[62 + k] = (float)log10(jv[(size_t)k * ld + c] + 1.0e-12);
        o[83] = dt;
    }
    __syncthreads();
    const int rows = min(FEAT_BLOCK, n - c0);
    float *dst = f + (size_t)c0 * NFEAT;
    for (int i = threadIdx.x; i < rows * NFEAT; i += FEAT_BLOCK) dst[i] = sf[(i / NFEAT) * FEAT_PAD + i % NFEAT];
}

// Predictions -> per-cell starting step (h0 = 10^(y0 * s0 + m0)) and a descending cost key.
__global__ void k_seed(int n, const float *__restrict__ y, float m0, float s0, float m1, float s1, float scale,
                       double *__restrict__ h0, unsigned int *__restrict__ key, int *__restrict__ idx)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const float lh = y[(size_t)c * NY] * s0 + m0;
    const float lc = y[(size_t)c * NY + 1] * s1 + m1;
    h0[c] = isfinite(lh) ? scale * exp10((double)lh) : -1.0;  // non-finite -> solver uses its default
    // sort ascending on the bitwise-flipped key = descending predicted cost
    unsigned int u = __float_as_uint(isfinite(lc) ? lc : 0.f);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    key[c] = ~u;
    idx[c] = c;
}

// Cost order by chunks of 32 consecutive cells: a chunk's key is its costliest cell's
// (the smallest flipped key); a partial last chunk sorts last.  Keeping 32 consecutive
// cells together keeps the solver's loads of a warp's cells coalesced.
constexpr int ORDER_CHUNK = 32;

__global__ void k_chunk_keys(int n, const unsigned int *__restrict__ key, unsigned int *__restrict__ ckey,
                             int *__restrict__ cidx)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nq = (n + ORDER_CHUNK - 1) / ORDER_CHUNK;
    if (q >= nq) return;
    const int lo = q * ORDER_CHUNK, hi = min(n, lo + ORDER_CHUNK);
    unsigned int k = 0xFFFFFFFFu;
    if (hi - lo == ORDER_CHUNK)
        for (int c = lo; c < hi; c++) k = min(k, key[c]);
    ckey[q] = k;
    cidx[q] = q;
}

__global__ void k_expand_chunks(int n, const int *__restrict__ chunk, int *__restrict__ order)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    order[p] = chunk[p / ORDER_CHUNK] * ORDER_CHUNK + p % ORDER_CHUNK;
}

}  // namespace mlp
}  // namespace radm2

// ============================================================================ host ABI
#include <cub/cub.cuh>

#include "radm2_ctx.h"

struct radm2_mlp {
    int device = 0;
    cudaStream_t st = nullptr;
    float *p = nullptr, *g = nullptr, *m = nullptr, *v = nullptr;  // master params, grads, Adam moments
    __nv_bfloat16 *wt = nullptr;                                     // bf16 transposed weight image
    float *xmean = nullptr, *xstd = nullptr;                         // [NIN] (device)
    float ymean[2] = {0.f, 0.f}, ystd[2] = {1.f, 1.f};
    float *loss = nullptr;                                           // device scalar
    float *z = nullptr, *y = nullptr, *xbuf = nullptr, *tbuf = nullptr;  // work, capacity `cap` rows
    int cap = 0, zcap = 0;
    int step = 0;
    int nsm = 148;
    float h0_scale = 1.0f;  // seeded h0 = h0_scale * predicted step
    unsigned int gen = 0;   // bumped when a value that seeding passes by value changes
    int attached = 0;       // contexts that seed every integration from this network
    bool use_tc = true;     // inference forward on tcgen05 (else mma.sync)
    int *tc_err = nullptr;  // device flag: a tcgen05 forward wait gave up
};

namespace {

using namespace radm2::mlp;

// Work buffers for n rows; the pre-activations (3 x n x 128 floats) only for training.
int mlp_ensure(radm2_mlp *m, int n, bool train)
{
    if (n > m->cap) {
        cudaFree(m->y);
        cudaFree(m->xbuf);
        cudaFree(m->tbuf);
        m->y = m->xbuf = m->tbuf = nullptr;
        m->cap = 0;
        if (cudaMalloc(&m->y, sizeof(float) * (size_t)n * NY) != cudaSuccess ||
            cudaMalloc(&m->xbuf, sizeof(float) * (size_t)n * NFEAT) != cudaSuccess ||
            cudaMalloc(&m->tbuf, sizeof(float) * (size_t)n * NY) != cudaSuccess)
            return RADM2_E_NOMEM;
        m->cap = n;
    }
    if (train && n > m->zcap) {
        cudaFree(m->z);
        m->z = nullptr;
        m->zcap = 0;
        if (cudaMalloc(&m->z, sizeof(float) * (size_t)n * W * 3) != cudaSuccess) return RADM2_E_NOMEM;
        m->zcap = n;
    }
    return RADM2_OK;
}

radm2::mlp::Net net_of(const radm2_mlp *m) { return radm2::mlp::Net{m->p, m->wt, m->xmean, m->xstd}; }

cudaError_t pack(radm2_mlp *m)
{
    k_pack_weights<<<(S_WEND + 255) / 256, 256, 0, m->st>>>(m->p, m->wt);
    return cudaGetLastError();
}

// Opt the network kernels into their dynamic shared memory, once per process (first
// call is made outside any stream capture by every entry point that launches them).
cudaError_t set_kernel_attributes()
{
    static bool done = false;
    if (done) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, FWD_SMEM_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
    if (e == cudaSuccess) e = cudaFuncSetAttribute(k_forward_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, TC_SMEM);
    done = e == cudaSuccess;
    return e;
}

cudaError_t forward(radm2_mlp *m, int n, const float *dx, float *dy, bool keep, cudaStream_t st)
{
    cudaError_t e0 = set_kernel_attributes();
    if (e0 != cudaSuccess) return e0;
    (void)cudaGetLastError();
    if (!keep && m->use_tc) {  // inference: tcgen05 pipelines of 128-row tiles, one CTA per SM
        const int groups = (n + TC_M * TC_G - 1) / (TC_M * TC_G);
        k_forward_tc<<<groups < m->nsm ? groups : m->nsm, TC_THREADS, TC_SMEM, st>>>(net_of(m), n, dx, dy,
                                                                                   m->tc_err, TC_WAIT_LIMIT, 0);
        return cudaGetLastError();
    }
    const size_t zs = (size_t)m->zcap * W;
    const int ntiles = (n + FWD_ROWS - 1) / FWD_ROWS;
    const int grid = ntiles < m->nsm ? ntiles : m->nsm;  // one CTA per SM walks the row tiles
    (void)cudaGetLastError();
    k_forward<<<grid, FWD_WARPS * 32, FWD_SMEM_BYTES, st>>>(net_of(m), n, dx, dy, keep ? m->z : nullptr,
                                                                 keep ? m->z + zs : nullptr,
                                                                 keep ? m->z + 2 * zs : nullptr);
    return cudaGetLastError();
}

cudaError_t backward(radm2_mlp *m, int n, const float *dx, const float *dt)
{
    const size_t zs = (size_t)m->zcap * W;
    cudaError_t e = cudaMemsetAsync(m->loss, 0, sizeof(float), m->st);
    if (e != cudaSuccess) return e;
    k_backward<<<(n + ROWS - 1) / ROWS, 128, SMEM_BYTES, m->st>>>(net_of(m), n, dx, m->y, dt, m->z, m->z + zs,
                                                                  m->z + 2 * zs, m->g, m->loss);
    return cudaGetLastError();
}

}  // namespace

// Allocate what seeding a context needs (h0, feature and prediction rows, sort keys, and
// the order with its sort workspace when asked).  The rows belong to the context, so a
// captured graph never reads buffers that the network may reallocate; nothing is
// allocated again while the cell count stays the same.
int radm2::mlp_prepare_seed(radm2_ctx *c, radm2_mlp *m, int order)
{
    (void)m;
    const int n = c->ncell;
    cudaError_t e = set_kernel_attributes();
    if (e == cudaSuccess && !c->h0) e = cudaMalloc((void **)&c->h0, sizeof(double) * c->ld);
    if (e == cudaSuccess && order && !c->order) e = cudaMalloc((void **)&c->order, sizeof(int) * c->ld);
    if (e == cudaSuccess && c->seed_cap < n) {
        void *old[] = {c->seed_keys, c->seed_idx, c->seed_tmp, c->seed_x, c->seed_y};
        for (void *q : old) cudaFree(q);
        c->seed_keys = nullptr;
        c->seed_idx = nullptr;
        c->seed_tmp = nullptr;
        c->seed_x = c->seed_y = nullptr;
        c->seed_tmp_bytes = 0;
        c->seed_cap = 0;
        e = cudaMalloc((void **)&c->seed_keys, sizeof(unsigned int) * (size_t)n * 2);
        // per-cell indices, then room for chunk indices in and out of the chunk sort
        if (e == cudaSuccess) e = cudaMalloc((void **)&c->seed_idx, sizeof(int) * ((size_t)n + 2 * (size_t)(n / 32 + 1)));
        if (e == cudaSuccess) e = cudaMalloc((void **)&c->seed_x, sizeof(float) * (size_t)n * NFEAT);
        if (e == cudaSuccess) e = cudaMalloc((void **)&c->seed_y, sizeof(float) * (size_t)n * NY);
        if (e == cudaSuccess) c->seed_cap = n;
    }
    if (e == cudaSuccess && order && !c->seed_tmp) {
        e = cub::DeviceRadixSort::SortPairs(nullptr, c->seed_tmp_bytes, c->seed_keys, c->seed_keys + n, c->seed_idx,
                                            c->order, n, 0, 32, c->st);
        if (e == cudaSuccess) e = cudaMalloc(&c->seed_tmp, c->seed_tmp_bytes);
    }
    if (e != cudaSuccess) {
        c->err = std::string("seeding buffers: ") + cudaGetErrorString(e);
        return RADM2_E_NOMEM;
    }
    return RADM2_OK;
}

unsigned int radm2::mlp_generation(const radm2_mlp *m) { return m ? m->gen : 0u; }
void radm2::mlp_detach(radm2_mlp *m) { m->attached--; }

// Stream-ordered seeding on the context's stream (capturable): features -> network ->
// per-cell h0 (and the descending-cost order when asked).
cudaError_t radm2::mlp_enqueue_seed(radm2_ctx *c, radm2_mlp *m, double dt, int order, int lo, int count)
{
    // cells [lo, lo + count) (count < 0: all); a sub-range gets h0 only, no order
    const int n = count < 0 ? c->ncell : count;
    if (count >= 0) order = 0;
    (void)cudaGetLastError();
    k_features<<<(n + FEAT_BLOCK - 1) / FEAT_BLOCK, FEAT_BLOCK, 0, c->st>>>(n, c->ld, c->var + lo, c->fix + lo,
                                                                         c->temp + lo, c->jv + lo, (float)dt,
                                                                         c->seed_x);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = forward(m, n, c->seed_x, c->seed_y, false, c->st);
    if (e == cudaSuccess) {
        k_seed<<<(n + 127) / 128, 128, 0, c->st>>>(n, c->seed_y, m->ymean[0], m->ystd[0], m->ymean[1], m->ystd[1],
                                                   m->h0_scale, c->h0 + lo, c->seed_keys, c->seed_idx);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess && order == 1) {
        size_t tb = c->seed_tmp_bytes;
        e = cub::DeviceRadixSort::SortPairs(c->seed_tmp, tb, c->seed_keys, c->seed_keys + n, c->seed_idx, c->order, n,
                                            0, 32, c->st);
    } else if (e == cudaSuccess && order == 2) {
        const int nq = (n + ORDER_CHUNK - 1) / ORDER_CHUNK;
        unsigned int *ckey = c->seed_keys + n;  // chunk keys in the second half, sorted into the first
        int *cin = c->seed_idx + n, *cout = c->seed_idx + n + nq;
        k_chunk_keys<<<(nq + 127) / 128, 128, 0, c->st>>>(n, c->seed_keys, ckey, cin);
        e = cudaGetLastError();
        size_t tb = c->seed_tmp_bytes;
        if (e == cudaSuccess)
            e = cub::DeviceRadixSort::SortPairs(c->seed_tmp, tb, ckey, c->seed_keys, cin, cout, nq, 0, 32, c->st);
        if (e == cudaSuccess) {
            k_expand_chunks<<<(n + 127) / 128, 128, 0, c->st>>>(n, cout, c->order);
            e = cudaGetLastError();
        }
    }
    return e;
}

extern "C" {

int radm2_mlp_nparams(void) { return NPARAM; }

int radm2_mlp_create(radm2_mlp **out, int device, unsigned int seed)
{
    if (!out) return RADM2_E_ARG;
    *out = nullptr;
    if (cudaSetDevice(device) != cudaSuccess) return RADM2_E_NODEV;
    radm2_mlp *m = new radm2_mlp();
    m->device = device;
    cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, device);
    bool ok = cudaStreamCreateWithFlags(&m->st, cudaStreamNonBlocking) == cudaSuccess &&
              cudaMalloc(&m->p, sizeof(float) * NPARAM) == cudaSuccess &&
              cudaMalloc(&m->g, sizeof(float) * NPARAM) == cudaSuccess &&
              cudaMalloc(&m->m, sizeof(float) * NPARAM) == cudaSuccess &&
              cudaMalloc(&m->v, sizeof(float) * NPARAM) == cudaSuccess &&
              cudaMalloc(&m->wt, sizeof(__nv_bfloat16) * S_WEND) == cudaSuccess &&
              cudaMalloc(&m->xmean, sizeof(float) * NIN) == cudaSuccess &&
              cudaMalloc(&m->xstd, sizeof(float) * NIN) == cudaSuccess &&
              cudaMalloc(&m->loss, sizeof(float)) == cudaSuccess &&
              cudaMalloc(&m->tc_err, sizeof(int)) == cudaSuccess;
    if (!ok) {
        radm2_mlp_destroy(m);
        return RADM2_E_NOMEM;
    }
    // He-uniform initialisation from a seeded linear congruential stream; padding stays zero.
    std::vector<float> h(NPARAM, 0.f);
    unsigned long long s = 0x9E3779B97F4A7C15ull ^ seed;
    auto unif = [&]() {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        return (float)((s >> 11) * (1.0 / 9007199254740992.0)) * 2.f - 1.f;
    };
    auto fill = [&](int off, int fan_in, int rows, int cols, int valid_rows, int valid_cols) {
        const float b = sqrtf(6.f / (float)fan_in);
        for (int r = 0; r < rows; r++)
            for (int c = 0; c < cols; c++) h[off + r * cols + c] = (r < valid_rows && c < valid_cols) ? b * unif() : 0.f;
    };
    fill(OFF_W1, NFEAT, NIN, W, NFEAT, W);
    fill(OFF_W2, W, W, W, W, W);
    fill(OFF_W3, W, W, W, W, W);
    fill(OFF_W4, W, W, NOUT, W, NY);
    std::vector<float> ones(NIN, 1.f), zeros(NIN, 0.f);
    ok = cudaMemcpy(m->p, h.data(), sizeof(float) * NPARAM, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemset(m->g, 0, sizeof(float) * NPARAM) == cudaSuccess &&
         cudaMemset(m->m, 0, sizeof(float) * NPARAM) == cudaSuccess &&
         cudaMemset(m->v, 0, sizeof(float) * NPARAM) == cudaSuccess &&
         cudaMemset(m->tc_err, 0, sizeof(int)) == cudaSuccess &&
         cudaMemcpy(m->xmean, zeros.data(), sizeof(float) * NIN, cudaMemcpyHostToDevice) == cudaSuccess &&
         cudaMemcpy(m->xstd, ones.data(), sizeof(float) * NIN, cudaMemcpyHostToDevice) == cudaSuccess &&
         pack(m) == cudaSuccess && cudaStreamSynchronize(m->st) == cudaSuccess;
    if (!ok) {
        radm2_mlp_destroy(m);
        return RADM2_E_CUDA;
    }
    *out = m;
    return RADM2_OK;
}

int radm2_mlp_destroy(radm2_mlp *m)
{
    if (!m) return RADM2_E_ARG;
    if (m->attached > 0) return RADM2_E_STATE;  // still attached to a context
    cudaSetDevice(m->device);
    if (m->st) cudaStreamSynchronize(m->st);
    void *ptrs[] = {m->p,    m->g, m->m, m->v,    m->wt,   m->xmean, m->xstd,
                    m->loss, m->z, m->y, m->xbuf, m->tbuf, m->tc_err};
    for (void *q : ptrs)
        if (q) cudaFree(q);
    if (m->st) cudaStreamDestroy(m->st);
    delete m;
    return RADM2_OK;
}

int radm2_mlp_set_params(radm2_mlp *m, const float *host)
{
    if (!m || !host) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    if (cudaMemcpyAsync(m->p, host, sizeof(float) * NPARAM, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        pack(m) != cudaSuccess || cudaStreamSynchronize(m->st) != cudaSuccess)
        return RADM2_E_CUDA;
    return RADM2_OK;
}

int radm2_mlp_get_params(radm2_mlp *m, float *host)
{
    if (!m || !host) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    if (cudaMemcpyAsync(host, m->p, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return RADM2_E_CUDA;
    return RADM2_OK;
}

int radm2_mlp_set_norm(radm2_mlp *m, const float *xmean, const float *xstd, const float *ymean, const float *ystd)
{
    if (!m || !xmean || !xstd || !ymean || !ystd) return RADM2_E_ARG;
    float mm[NIN], ss[NIN];
    for (int i = 0; i < NIN; i++) {
        mm[i] = i < NFEAT ? xmean[i] : 0.f;
        ss[i] = i < NFEAT ? (xstd[i] > 0.f ? xstd[i] : 1.f) : 1.f;
    }
    for (int k = 0; k < NY; k++) {
        m->ymean[k] = ymean[k];
        m->ystd[k] = ystd[k] > 0.f ? ystd[k] : 1.f;
    }
    m->gen++;
    cudaSetDevice(m->device);
    if (cudaMemcpy(m->xmean, mm, sizeof mm, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(m->xstd, ss, sizeof ss, cudaMemcpyHostToDevice) != cudaSuccess)
        return RADM2_E_CUDA;
    return RADM2_OK;
}

int radm2_mlp_forward(radm2_mlp *m, int n, const float *x, float *y)
{
    if (!m || n <= 0 || !x || !y) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    int rc = mlp_ensure(m, n, false);
    if (rc) return rc;
    if (cudaMemcpyAsync(m->xbuf, x, sizeof(float) * (size_t)n * NFEAT, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        forward(m, n, m->xbuf, m->y, false, m->st) != cudaSuccess ||
        cudaMemcpyAsync(y, m->y, sizeof(float) * (size_t)n * NY, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return RADM2_E_CUDA;
    return radm2_mlp_status(m);
}

int radm2_mlp_gradients(radm2_mlp *m, int n, const float *x, const float *target, float *grad, float *loss)
{
    if (!m || n <= 0 || !x || !target || !grad || !loss) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    int rc = mlp_ensure(m, n, true);
    if (rc) return rc;
    if (cudaMemcpyAsync(m->xbuf, x, sizeof(float) * (size_t)n * NFEAT, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        cudaMemcpyAsync(m->tbuf, target, sizeof(float) * (size_t)n * NY, cudaMemcpyHostToDevice, m->st) != cudaSuccess ||
        cudaMemsetAsync(m->g, 0, sizeof(float) * NPARAM, m->st) != cudaSuccess ||
        forward(m, n, m->xbuf, m->y, true, m->st) != cudaSuccess || backward(m, n, m->xbuf, m->tbuf) != cudaSuccess ||
        cudaMemcpyAsync(grad, m->g, sizeof(float) * NPARAM, cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
        cudaMemsetAsync(m->g, 0, sizeof(float) * NPARAM, m->st) != cudaSuccess ||
        cudaStreamSynchronize(m->st) != cudaSuccess)
        return RADM2_E_CUDA;
    return RADM2_OK;
}

int radm2_mlp_train_step(radm2_mlp *m, int n, const float *dx, const float *dtarget, float lr, float *loss)
{
    if (!m || n <= 0 || !dx || !dtarget) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    int rc = mlp_ensure(m, n, true);
    if (rc) return rc;
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
    if (forward(m, n, dx, m->y, true, m->st) != cudaSuccess || backward(m, n, dx, dtarget) != cudaSuccess)
        return RADM2_E_CUDA;
    k_adam<<<(NPARAM + 255) / 256, 256, 0, m->st>>>(NPARAM, m->p, m->g, m->m, m->v, lr, b1, b2, eps, c1, c2);
    if (cudaGetLastError() != cudaSuccess || pack(m) != cudaSuccess) return RADM2_E_CUDA;
    if (loss) {
        if (cudaMemcpyAsync(loss, m->loss, sizeof(float), cudaMemcpyDeviceToHost, m->st) != cudaSuccess ||
            cudaStreamSynchronize(m->st) != cudaSuccess)
            return RADM2_E_CUDA;
    }
    return RADM2_OK;
}

int radm2_mlp_set_h0_scale(radm2_mlp *m, float scale)
{
    if (!m || !(scale > 0.f)) return RADM2_E_ARG;
    m->h0_scale = scale;
    m->gen++;
    return RADM2_OK;
}

int radm2_mlp_set_tensor_path(radm2_mlp *m, int tcgen05)
{
    if (!m) return RADM2_E_ARG;
    m->use_tc = tcgen05 != 0;
    m->gen++;  // graphs that captured the other forward are rebuilt
    return RADM2_OK;
}

int radm2_mlp_status(radm2_mlp *m)
{
    if (!m) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    int flag = 0;
    if (cudaMemcpy(&flag, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) return RADM2_E_CUDA;
    return flag ? RADM2_E_CUDA : RADM2_OK;
}

int radm2_mlp_selftest_wait_limit(radm2_mlp *m)
{
    if (!m) return RADM2_E_ARG;
    cudaSetDevice(m->device);
    int rc = mlp_ensure(m, TC_M, false);
    if (rc) return rc;
    if (set_kernel_attributes() != cudaSuccess) return RADM2_E_CUDA;
    int raised = 0;
    const int zero = 0;
    // one CTA, one tile, nothing committed: every wait gives up after 4096 polls
    (void)cudaGetLastError();
    k_forward_tc<<<1, TC_THREADS, TC_SMEM, m->st>>>(net_of(m), TC_M, m->xbuf, m->y, m->tc_err, 4096L, 1);
    if (cudaGetLastError() != cudaSuccess || cudaStreamSynchronize(m->st) != cudaSuccess ||
        cudaMemcpy(&raised, m->tc_err, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess ||
        cudaMemcpy(m->tc_err, &zero, sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess)
        return RADM2_E_CUDA;
    return raised ? RADM2_OK : RADM2_E_STATE;
}

int radm2_mlp_synchronize(radm2_mlp *m)
{
    if (!m) return RADM2_E_ARG;
    return cudaStreamSynchronize(m->st) == cudaSuccess ? RADM2_OK : RADM2_E_CUDA;
}

int radm2_get_features(radm2_ctx *c, double dt, float *host_out)
{
    if (!c || !host_out || !(dt > 0.0)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    cudaSetDevice(c->o.device);
    float *d = nullptr;
    if (cudaMalloc(&d, sizeof(float) * (size_t)c->ncell * NFEAT) != cudaSuccess) return RADM2_E_NOMEM;
    k_features<<<(c->ncell + FEAT_BLOCK - 1) / FEAT_BLOCK, FEAT_BLOCK, 0, c->st>>>(c->ncell, c->ld, c->var, c->fix,
                                                                              c->temp, c->jv, (float)dt, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(host_out, d, sizeof(float) * (size_t)c->ncell * NFEAT,
                                              cudaMemcpyDeviceToHost, c->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->st);
    cudaFree(d);
    return e == cudaSuccess ? RADM2_OK : RADM2_E_CUDA;
}

int radm2_seed_cells(radm2_ctx *c, radm2_mlp *m, double dt, int set_h0, int set_order)
{
    if (!c || !m || !(dt > 0.0)) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    cudaSetDevice(c->o.device);
    if (set_order < 0 || set_order > 2) return RADM2_E_ARG;
    int rc = radm2::mlp_prepare_seed(c, m, set_order);
    if (rc) return rc;
    if (radm2::mlp_enqueue_seed(c, m, dt, set_order) != cudaSuccess || cudaStreamSynchronize(c->st) != cudaSuccess) {
        c->err = "radm2_seed_cells: CUDA error";
        return RADM2_E_CUDA;
    }
    c->use_h0 = set_h0 != 0;
    c->use_order = set_order != 0;
    return RADM2_OK;
}

int radm2_attach_mlp(radm2_ctx *c, radm2_mlp *m, int set_order)
{
    if (!c) return RADM2_E_ARG;
    if (!c->var) return RADM2_E_STATE;
    cudaSetDevice(c->o.device);
    if (set_order < 0 || set_order > 2) return RADM2_E_ARG;
    if (m && m->device != c->o.device) {
        c->err = "radm2_attach_mlp: network and context are on different devices";
        return RADM2_E_ARG;
    }
    if (m) {
        int rc = radm2::mlp_prepare_seed(c, m, set_order);
        if (rc) return rc;
    }
    radm2::ctx_drop_graph(c);
    if (c->mlp) c->mlp->attached--;
    c->mlp = m;
    c->mlp_order = m ? set_order : 0;
    if (!m) return RADM2_OK;
    m->attached++;
    // the network's stream may still be writing its weights (training)
    if (cudaStreamSynchronize(m->st) != cudaSuccess) return RADM2_E_CUDA;
    c->use_h0 = true;
    c->use_order = set_order != 0;
    return RADM2_OK;
}

}  // extern "C"
