// The fused per-cell ROS-3 solver kernel.
//
// One thread integrates one grid cell at a time through the reference's whole
// step loop -- time-loop mask and step clamp (mgpu.cu:1595-1614), Jacobian and
// matrix preparation (mgpu.cu:1672-2652, 3128-3166), pivot-free LU
// (mgpu.cu:2726-2780), the three ROS-3 stages (mgpu.cu:3595-3625, restored),
// and the error norm / step-size controller (mgpu.cu:3168-3262) -- without
// returning to the host between steps.
//
// Per-thread working set, three regions, each laid out word-major per block
// (word w of thread t at base + w*BS + t, so every access is coalesced / bank-
// conflict free and carries a compile-time offset):
//   RCY  rate constants (156) and state Y (59)             FP64
//   VEC  Fcn0, K1, K2, K3 and a temporary (5 x 59)          FP64, global scratch
//   LU   the 659 LU slots                                   LUT (double or float)
// PLACE selects shared memory for LU (bit 0) and RCY (bit 1), and tensor memory for the
// most used LU slots (bit 2: 128 slots per thread; bit 3: 256 slots per thread, one
// 128-thread CTA per SM); what is not on chip lives in the global scratch slot of the thread.
//
// Schedules:
//   static      one thread per cell, cell = global thread index (the plain method)
//   persistent  a grid sized to the machine; each lane takes its next cell from a
//               global queue (warp-aggregated atomics) as soon as its current cell
//               finishes, optionally in a caller-given order (cost-sorted cells).
//
// LU precision: double (plain FP64) or float with FP64 iterative refinement, the
// residual b - G x being formed in FP64 with a fresh Jacobian-vector product.
#pragma once

#include "radm2_device.cuh"
#include "gen/radm2_tmem.h"
#include "gen/radm2_tmem_wide.h"

namespace radm2 {

enum { SCHED_STATIC = 0, SCHED_PERSISTENT = 1 };
enum { PLACE_GLOBAL = 0, PLACE_LU_SMEM = 1, PLACE_RCY_SMEM = 2, PLACE_LU_TMEM = 4, PLACE_LU_TMEM_256 = 8 };

constexpr int RCY_WORDS = NREACT + NVAR;  // 215
constexpr int RCY_RC = 0, RCY_Y = NREACT;
constexpr int VEC_WORDS = 5 * NVAR;  // 295
constexpr int VEC_F0 = 0, VEC_K1 = NVAR, VEC_K2 = 2 * NVAR, VEC_K3 = 3 * NVAR, VEC_TMP = 4 * NVAR;

template <typename LUT>
struct LuWords {  // LU slots expressed in double words
    static constexpr int value = sizeof(LUT) == 8 ? NJVS : (NJVS + 1) / 2;
};

// Where each region of a thread's working set lives, in doubles from the block base
// of its memory (global scratch block or dynamic shared memory); a thread's word w
// of a region sits at base + (off + w) * BS + thread.
template <typename LUT, int PLACE>
struct Layout {
    static constexpr bool rcy_smem = (PLACE & PLACE_RCY_SMEM) != 0;
    static constexpr bool lu_smem = (PLACE & PLACE_LU_SMEM) != 0;
    static constexpr int vec_off = 0;  // always global
    static constexpr int rcy_off = rcy_smem ? 0 : VEC_WORDS;
    static constexpr int lu_off = lu_smem ? (rcy_smem ? RCY_WORDS : 0) : VEC_WORDS + (rcy_smem ? 0 : RCY_WORDS);
    static constexpr int global_words = VEC_WORDS + (rcy_smem ? 0 : RCY_WORDS) + (lu_smem ? 0 : LuWords<LUT>::value);
    static constexpr int smem_words = (rcy_smem ? RCY_WORDS : 0) + (lu_smem ? LuWords<LUT>::value : 0);
};

// Host-side bounds check of a layout for block size bs: every word of every region
// of every thread lands inside its block's allocation.  Returns 0 when it holds.
template <typename LUT, int PLACE>
inline int layout_check(int bs)
{
    using L = Layout<LUT, PLACE>;
    const long gcap = (long)L::global_words * bs, scap = (long)L::smem_words * bs;  // doubles per block
    // last element touched, in doubles (LU in LUT units converted to doubles)
    const long vec_last = (long)(L::vec_off + VEC_WORDS - 1) * bs + (bs - 1);
    const long rcy_last = (long)(L::rcy_off + RCY_WORDS - 1) * bs + (bs - 1);
    const long lu_last_elem = (long)L::lu_off * bs * (8 / (long)sizeof(LUT)) + (long)(NJVS - 1) * bs + (bs - 1);
    const long lu_last = lu_last_elem * (long)sizeof(LUT) / 8;
    int bad = 0;
    bad |= vec_last >= gcap;
    bad |= rcy_last >= (L::rcy_smem ? scap : gcap);
    bad |= lu_last >= (L::lu_smem ? scap : gcap);
    // regions must not overlap inside one memory
    if (!L::rcy_smem) bad |= L::rcy_off < L::vec_off + VEC_WORDS;
    if (!L::lu_smem) bad |= L::lu_off < L::vec_off + VEC_WORDS;
    if (!L::lu_smem && !L::rcy_smem) bad |= L::lu_off < L::rcy_off + RCY_WORDS;
    if (L::lu_smem && L::rcy_smem) bad |= L::lu_off < RCY_WORDS;
    return bad;
}

// LU representation inside the solver: with RADM2_LU_RECIP (default) the factorisation
// stores 1/U(k,k) in the diagonal slots, so eliminations and back substitution multiply
// instead of divide (one division per row).  Each multiply-by-reciprocal differs from the
// division by at most one rounding; the mirror kernels keep the exact divisions.
#ifndef RADM2_LU_RECIP
#define RADM2_LU_RECIP 1
#endif
#if RADM2_LU_RECIP
#define RADM2_DECOMP_TM_INC "gen/radm2_decomp_rcp_tm.inc"
#define RADM2_SOLVE_TM_INC "gen/radm2_solve_rcp_tm.inc"
#define RADM2_DECOMP_TMW_INC "gen/radm2_decomp_rcp_tm_wide.inc"
#define RADM2_SOLVE_TMW_INC "gen/radm2_solve_rcp_tm_wide.inc"
#define RADM2_DECOMP_INC "gen/radm2_decomp_rcp.inc"
#define RADM2_JACLU_INC "gen/radm2_jaclu_rcp.inc"
#define RADM2_SOLVE_INC "gen/radm2_solve_rcp.inc"
#else
#define RADM2_DECOMP_TM_INC "gen/radm2_decomp_tm.inc"
#define RADM2_SOLVE_TM_INC "gen/radm2_solve_tm.inc"
#define RADM2_DECOMP_TMW_INC "gen/radm2_decomp_tm_wide.inc"
#define RADM2_SOLVE_TMW_INC "gen/radm2_solve_tm_wide.inc"
#define RADM2_DECOMP_INC "gen/radm2_decomp.inc"
#define RADM2_JACLU_INC "gen/radm2_jaclu.inc"
#define RADM2_SOLVE_INC "gen/radm2_solve.inc"
#endif
// Jacobian and LU: RADM2_JACLU 0 (default) writes the whole Jacobian into the LU slots and
// factors it in place afterwards (ph_jac + ph_decomp).  1 forms each row of G in registers
// and factors it before storing it (ph_jaclu): the slots are stored once instead of written,
// read back and written again, but a partial that feeds several rows is formed once per row
// (1,200 partial products instead of 275).  Measured 7% slower on B200, so not the default.
// The same sums in the same order; the compiler contracts them into multiply-adds
// differently, so the fast forms of the two agree to rounding, not bit for bit.
#ifndef RADM2_JACLU
#define RADM2_JACLU 0
#endif
// Error-norm terms (mgpu.cu:3238): with RADM2_ACCEPT_RCP, yerr^2 times the correctly
// rounded reciprocal of scale^2 instead of the division (at most one rounding apart).
#ifndef RADM2_ACCEPT_RCP
#define RADM2_ACCEPT_RCP 0
#endif
// Phase functions are inlined into the kernel (measured 1.5-1.7x faster on B200 than
// separate non-inlined functions, despite a few hundred bytes of spills); build with
// -DRADM2_PHASE_INLINE=0 to compile them as separate functions.  The RHS is the exception
// (RADM2_FUN_PHASE): it runs at two sites, Fcn0 and the stage-2 right-hand side, and as one
// out-of-line copy it keeps ~1,500 instructions out of the kernel's instruction-cache
// footprint.  Measured 2.7% faster on the 4M mixed batch, with fewer spills and results
// identical to the inlined form.
#ifndef RADM2_PHASE_INLINE
#define RADM2_PHASE_INLINE 1
#endif
#if RADM2_PHASE_INLINE
#define RADM2_PHASE __forceinline__
#else
#define RADM2_PHASE __noinline__
#endif
#ifndef RADM2_FUN_INLINE
#define RADM2_FUN_INLINE 0
#endif
#if RADM2_FUN_INLINE
#define RADM2_FUN_PHASE __forceinline__
#else
#define RADM2_FUN_PHASE __noinline__
#endif

// ---------------------------------------------------------------- tensor-memory slots
// PLACE_LU_TMEM keeps the RADM2_TMEM_SLOTS most accessed LU slots of every thread in tensor
// memory instead of its global scratch: thread t of warp w owns lane 32 (w % 4) + t of its
// CTA's allocation and 256 columns of it (the upper half of a 512-column allocation for warps
// 4-7), a double in two 32-bit columns.  PLACE_LU_TMEM_256 gives one CTA of 128 threads all
// 512 columns, so each thread holds the 256 most accessed slots.  Tensor memory is separate
// from the L1 / shared memory array, so it adds on-chip storage without shrinking the cache.  Its loads and stores
// are warp-collective (.sync.aligned): every lane of the warp executes them together.

// One double from tensor memory.  The thread's earlier stores are completed first (they may
// be to the same columns), and the value is waited for inside the same statement, so it is
// never read before it has arrived.
__device__ __forceinline__ double tmem_ld_f64(uint32_t t)
{
    uint32_t lo, hi;
    asm volatile(
        "tcgen05.wait::st.sync.aligned;\n\t"
        "tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(lo), "=r"(hi)
        : "r"(t));
    return __hiloint2double((int)hi, (int)lo);
}

__device__ __forceinline__ void tmem_st_f64(uint32_t t, double v)
{
    asm volatile("tcgen05.st.sync.aligned.32x32b.x2.b32 [%0], {%1, %2};" ::"r"(t), "r"(__double2loint(v)),
                 "r"(__double2hiint(v)));
}

// An LU slot held in tensor memory: reads load it, assignment stores it.
struct TmemSlot {
    uint32_t t;  // address of the slot's first column in the thread's lane
    __device__ __forceinline__ operator double() const { return tmem_ld_f64(t); }
    __device__ __forceinline__ void operator=(double v) const { tmem_st_f64(t, v); }
};

// Slot S of the thread's LU: its global (or shared) scratch word, or with TM its
// tensor-memory columns when the slot is one of the tensor-memory slots (TM 1: the
// 128-slot map, TM 2: the 256-slot map, PLACE_LU_TMEM_256).
template <int TM, int BS, int S, typename LUT>
__device__ __forceinline__ decltype(auto) lu_slot(LUT *sg, uint32_t tb)
{
    constexpr int col = TM == 2 ? radm2_tmem_wide_col[S] : radm2_tmem_col[S];
    if constexpr (TM != 0 && col >= 0)
        return TmemSlot{tb + (uint32_t)col};
    else
        return (sg[S * BS]);
}

// ---------------------------------------------------------------- phases
// Each phase is a function of its own, inlined into the kernel (RADM2_PHASE) except the
// RHS (RADM2_FUN_PHASE), which exists once in the instruction stream although both Fcn0
// and the stage-2 right-hand side use it.

// dst = F(v): the RHS at state v (v and dst may alias; dst is written after v is read).
template <int BS>
__device__ RADM2_FUN_PHASE void ph_fun(const double *v, const double *rc, double *dst, double fix0, double fix1)
{
#define V(i) v[(i) * BS]
#define RC(r) rc[(r) * BS]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define VDOT_OUT(i, e) dst[(i) * BS] = (e)
#include "gen/radm2_fun.inc"
#undef VDOT_OUT
#undef V
#undef RC
#undef FIX
}

// G = -J(y) + ghinv I in the LU slots (mgpu.cu:3139-3142 with the diagonal of 2700 restored).
template <int BS, typename LUT, int TM = 0>
__device__ RADM2_PHASE void ph_jac(const double *y, const double *rc, LUT *sg, double fix0, double fix1, double ghinv,
                                   uint32_t tb = 0)
{
#define V(i) y[(i) * BS]
#define RC(r) rc[(r) * BS]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define G(s) lu_slot<TM, BS, (s)>(sg, tb)
#define JAC_OUT(s, e) G(s) = (LUT)(-(e))
#define JAC_OUT_DIAG(s, e) G(s) = (LUT)((-(e)) + ghinv)
#define JAC_OUT_ZERO(s, d) G(s) = (d) ? (LUT)((-0.0) + ghinv) : (LUT)(-0.0)
#include "gen/radm2_jac.inc"
    if constexpr (TM) asm volatile("tcgen05.wait::st.sync.aligned;");  // stores done before the LU reads
#undef JAC_OUT
#undef JAC_OUT_DIAG
#undef JAC_OUT_ZERO
#undef G
#undef V
#undef RC
#undef FIX
}

// In-place LU; returns 0 or the 1-based row of a zero pivot (checked before the row is
// eliminated, as mgpu.cu:2753-2757 does).
template <int BS, typename LUT, int TM = 0>
__device__ RADM2_PHASE int ph_decomp(LUT *sg, uint32_t tb = 0)
{
    int sing = 0;
#define G(s) lu_slot<TM, BS, (s)>(sg, tb)
#define LU_T LUT
// One elimination step's loads may not be hoisted above the previous step: this bounds
// the live set to one pivot row's worth of U entries and keeps the LU free of spills.
#define LU_STEP_FENCE asm volatile("" ::: "memory")
// (tensor memory: the pivot is read on every lane, as its load is warp-collective)
#define LU_PIVOT_CHECK(k, v)                                      \
    if (TM) {                                                     \
        const LUT pv_ = (v);                                      \
        sing = (sing == 0 && pv_ == (LUT)0) ? (k) + 1 : sing;     \
        __syncwarp();                                             \
    } else if (sing == 0 && (v) == (LUT)0)                        \
    sing = (k) + 1
    if constexpr (TM == 2) {  // the 256-slot map
#define TM_BASE tb
#include RADM2_DECOMP_TMW_INC
#undef TM_BASE
    } else if constexpr (TM) {  // tensor-memory slots read and written in groups
#define TM_BASE tb
#include RADM2_DECOMP_TM_INC
#undef TM_BASE
    } else {
#include RADM2_DECOMP_INC
    }
#undef LU_PIVOT_CHECK
#undef LU_STEP_FENCE
#undef LU_T
#undef G
    return sing;
}

// G = -J(y) + ghinv I and its in-place LU, row by row: each row's slots are formed in
// registers, checked, eliminated against the finished rows above it and stored once.
// Returns 0 or the 1-based row of a zero pivot, as ph_decomp.
template <int BS, typename LUT>
__device__ RADM2_PHASE int ph_jaclu(const double *y, const double *rc, LUT *sg, double fix0, double fix1,
                                    double ghinv)
{
    int sing = 0;
#define V(i) y[(i) * BS]
#define RC(r) rc[(r) * BS]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define G(s) sg[(s) * BS]
#define LU_T LUT
#define JAC_VAL(e) ((LUT)(-(e)))
#define JAC_VAL_DIAG(e) ((LUT)((-(e)) + ghinv))
#define JAC_VAL_ZERO(d) ((d) ? (LUT)((-0.0) + ghinv) : (LUT)(-0.0))
#define LU_STEP_FENCE asm volatile("" ::: "memory")
#define LU_PIVOT_CHECK(k, v) \
    if (sing == 0 && (v) == (LUT)0) sing = (k) + 1
#include RADM2_JACLU_INC
#undef LU_PIVOT_CHECK
#undef LU_STEP_FENCE
#undef JAC_VAL_ZERO
#undef JAC_VAL_DIAG
#undef JAC_VAL
#undef LU_T
#undef G
#undef V
#undef RC
#undef FIX
    return sing;
}

// One ROS-3 stage: build the right-hand side, solve with the factored G, store K[stage].
//   stage 0: Fcn0                      (mgpu.cu:3601-3602)
//   stage 1: F(Y + A21 K1) + C21/h K1  (stage 2 reuses that F, NewF = 0; its partial
//            right-hand side F + C31/h K1 is parked in K3)
//   stage 2: (F + C31/h K1) + C32/h K2
// FP64 LU: one substitution.  FP32 LU: the substitution in float, then `refine`
// sweeps of x += G32^-1 (b - G64 x), residual in FP64 (G64 x = ghinv x - J x).  IR = 0
// compiles the FP32 form without the refinement code (refine must be 0): the residual's
// Jacobian-vector product and second substitution would otherwise stay in the kernel's
// instruction footprint although they never run.
template <int BS, typename LUT, int IR, int TM = 0>
__device__ RADM2_PHASE void ph_stage(int stage, const double *y, const double *rc, double *vec, const LUT *sg,
                                      double fix0, double fix1, double hc21, double hc31, double hc32,
                                      double ghinv, int refine, uint32_t tb = 0)
{
    static_assert(TM == 0 || sizeof(LUT) == 8, "tensor-memory LU slots hold doubles");
#define VW(w) vec[(w) * BS]
#define G(s) lu_slot<TM, BS, (s)>(sg, tb)
    double x[NVAR];
    if (stage == 0) {
#pragma unroll
        for (int i = 0; i < NVAR; i++) x[i] = VW(VEC_F0 + i);
    } else if (stage == 1) {
#pragma unroll
        for (int i = 0; i < NVAR; i++) VW(VEC_TMP + i) = y[i * BS] + RADM2_ROS_A0 * VW(VEC_K1 + i);
        ph_fun<BS>(vec + VEC_TMP * BS, rc, vec + VEC_TMP * BS, fix0, fix1);
#pragma unroll
        for (int i = 0; i < NVAR; i++) {
            const double f = VW(VEC_TMP + i), k1 = VW(VEC_K1 + i);
            x[i] = f + k1 * hc21;
            VW(VEC_K3 + i) = f + k1 * hc31;
        }
    } else {
#pragma unroll
        for (int i = 0; i < NVAR; i++) x[i] = VW(VEC_K3 + i) + VW(VEC_K2 + i) * hc32;
    }
    if constexpr (TM == 2) {
#define X(i) x[i]
#define TM_BASE tb
#include RADM2_SOLVE_TMW_INC
#undef TM_BASE
#undef X
    } else if constexpr (TM) {
#define X(i) x[i]
#define TM_BASE tb
#include RADM2_SOLVE_TM_INC
#undef TM_BASE
#undef X
    } else if (sizeof(LUT) == 8) {
#define X(i) x[i]
#include RADM2_SOLVE_INC
#undef X
    } else {
        float xf[NVAR];
#pragma unroll
        for (int i = 0; i < NVAR; i++) {
            if (IR) VW(VEC_TMP + i) = x[i];  // b, for the residual
            xf[i] = (float)x[i];
        }
#define X(i) xf[i]
#include RADM2_SOLVE_INC
#undef X
#pragma unroll
        for (int i = 0; i < NVAR; i++) x[i] = (double)xf[i];
        double *kout = vec + (VEC_K1 + stage * NVAR) * BS;
#pragma unroll 1
        for (int sweep = 0; sweep < (IR ? refine : 0); sweep++) {
            // park x in the stage's output slot so the residual reads it from memory
#pragma unroll
            for (int i = 0; i < NVAR; i++) kout[i * BS] = x[i];
            {
#define V(i) y[(i) * BS]
#define RC(r) rc[(r) * BS]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define XIN(i) kout[(i) * BS]
#define JX_OUT(row, e) xf[row] = (float)(VW(VEC_TMP + (row)) - (ghinv * kout[(row) * BS] - (e)))
#include "gen/radm2_jacvec.inc"
#undef JX_OUT
#undef XIN
#undef V
#undef RC
#undef FIX
            }
#define X(i) xf[i]
#include RADM2_SOLVE_INC
#undef X
#pragma unroll
            for (int i = 0; i < NVAR; i++) x[i] = kout[i * BS] + (double)xf[i];
        }
    }
    double *kout = vec + (VEC_K1 + stage * NVAR) * BS;
#pragma unroll
    for (int i = 0; i < NVAR; i++) kout[i * BS] = x[i];
#undef VW
#undef G
}

// ARITH tags the arithmetic the including file compiles the kernel with (0 = the fast form,
// 1 = reference arithmetic: RADM2_LU_RECIP=0 and no multiply-add contraction).  The body does
// not read it; it makes the two forms distinct instantiations, so that the same (BS, LUT,
// SCHED, PLACE, MINB) built both ways in two files are two kernels, not one name with two
// definitions.
template <int BS, typename LUT, int SCHED, int PLACE, int MINB, int IR = 1, int ARITH = 0>
__global__ void __launch_bounds__(BS, MINB) k_rosenbrock(const SolveArgs a)
{
    using L = Layout<LUT, PLACE>;
    constexpr int TM = (PLACE & PLACE_LU_TMEM_256) ? 2 : (PLACE & PLACE_LU_TMEM) ? 1 : 0;
    static_assert(!TM || (sizeof(LUT) == 8 && (BS == 128 || BS == 256) && (PLACE & PLACE_LU_SMEM) == 0),
                  "tensor-memory LU slots: FP64, 128 or 256 threads per block, LU otherwise in global scratch");
    static_assert(TM != 2 || (BS == 128 && (PLACE & PLACE_LU_TMEM) == 0), "wide tensor-memory map: 128 threads");
    // Tensor memory: 256 columns per 128 threads (two CTAs of 128 or one of 256 fill an SM's
    // 512 columns), or with the wide map all 512 columns for one CTA of 128 threads; warp 0
    // allocates them and gives up the right to allocate more.
    constexpr uint32_t TCOLS = (BS == 256 || TM == 2) ? 512u : 256u;
    uint32_t talloc = 0, tb = 0;  // the allocation, and this thread's first column in it
    if constexpr (TM) {
        __shared__ uint32_t tmem_base;
        if (threadIdx.x < 32) {
            asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                             (uint32_t)__cvta_generic_to_shared(&tmem_base)),
                         "r"(TCOLS)
                         : "memory");
            asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
        }
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        talloc = tmem_base;
        const uint32_t w = threadIdx.x >> 5;
        tb = talloc + ((32u * (w & 3u)) << 16) + (w >> 2) * 256u;
    }
    extern __shared__ double smem[];
    double *const gblk = a.scratch + (size_t)blockIdx.x * (L::global_words * BS);  // block bases
    double *const sblk = smem;
    double *const vec = gblk + L::vec_off * BS + threadIdx.x;
    double *const rcy = (L::rcy_smem ? sblk : gblk) + L::rcy_off * BS + threadIdx.x;
    LUT *const sg = reinterpret_cast<LUT *>((L::lu_smem ? sblk : gblk) + L::lu_off * BS) + threadIdx.x;
#define RW(w) rcy[(w) * BS]
#define VW(w) vec[(w) * BS]
#define G(s) sg[(s) * BS]
    const SolveParams &P = a.p;
    const int ld = a.ld;
    const int dir = P.direction;

    // ---- lane state
    int cell;
    if (SCHED == SCHED_STATIC) {
        cell = blockIdx.x * BS + threadIdx.x;
    } else {
        const unsigned m = __activemask();
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(a.queue, __popc(m));
        base = __shfl_sync(m, base, leader);
        cell = base + __popc(m & ((1u << lane) - 1));
    }
    bool have = cell < a.ncell;
    bool outer = true;  // next action: time-loop test, step clamp, Fcn0
    bool done = false;  // cell finished (ok or error) and must be written back
    int cidx = 0;       // cell index after the optional permutation
    double T = 0.0, H = 0.0, fix0 = 0.0, fix1 = 0.0, hfirst = 0.0;
    int rlast = 0, rmore = 0, nacc = 0, nrej = 0, nstp = 0, status = 1;

    auto load_cell = [&](int c) {
        cidx = (SCHED == SCHED_PERSISTENT && a.order) ? a.order[c] : c;
        const double *v = a.var + cidx;
#pragma unroll
        for (int i = 0; i < NVAR; i++) RW(RCY_Y + i) = v[(size_t)i * ld];
        const double *rc = a.rconst + cidx;
#pragma unroll
        for (int r = 0; r < NREACT; r++) RW(RCY_RC + r) = rc[(size_t)r * ld];
        fix0 = a.fix[cidx];
        fix1 = a.fix[(size_t)ld + cidx];
        T = P.Tstart;
        double hs = P.Hstart;
        if (a.h0) {
            const double h = a.h0[cidx];
            if (h > 0.0 && h <= P.Hmax) hs = h;  // non-finite or out of range: default
        }
        H = mind(hs, P.Hmax);  // mgpu.cu:3475-3477
        if (absd(H) <= 10.0 * P.Roundoff) H = DELTA_MIN;
        rlast = rmore = nacc = nrej = nstp = 0;
        status = 1;
        hfirst = 0.0;
        outer = true;
        done = false;
    };
    auto store_cell = [&]() {
        double *v = a.var + cidx;
#pragma unroll
        for (int i = 0; i < NVAR; i++) v[(size_t)i * ld] = RW(RCY_Y + i);
        a.status[cidx] = status;
        a.nacc[cidx] = nacc;
        a.nrej[cidx] = nrej;
        a.hfirst[cidx] = hfirst;
        a.hexit[cidx] = H;
        a.texit[cidx] = T;
    };
    auto next_cell = [&]() {
        if (SCHED == SCHED_STATIC) {
            have = false;
            return;
        }
        const unsigned m = __activemask();
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(a.queue, __popc(m));
        base = __shfl_sync(m, base, leader);
        cell = base + __popc(m & ((1u << lane) - 1));
        have = cell < a.ncell;
        if (have) load_cell(cell);
    };

    if (have) load_cell(cell);

    for (;;) {
        // Bring every lane that still has work to the start of a step attempt.
        while (have && (outer || done)) {
            if (done) {
                store_cell();
                next_cell();
                continue;
            }
            // Time-loop mask (mgpu.cu:1608-1613).
            const bool more = (dir > 0 && (T - P.Tend) + P.Roundoff <= 0.0) ||
                              (dir < 0 && (P.Tend - T) + P.Roundoff <= 0.0);
            if (!more) {
                done = true;
                continue;
            }
            H = mind(H, absd(P.Tend - T));
            // Fcn0 = F(Y)
            ph_fun<BS>(rcy + RCY_Y * BS, rcy + RCY_RC * BS, vec + VEC_F0 * BS, fix0, fix1);
            outer = false;
        }
        if (!__any_sync(0xffffffffu, have)) break;
        if (!TM && !have) continue;

        // ---------------------------------------------------------------- one attempt
        // With tensor-memory LU slots every lane of the warp runs the Jacobian, the LU and
        // the stages together (their tensor-memory accesses are warp-collective); a lane
        // without an attempt (act false) runs them on its own scratch and drops the result.
        bool act = have;
        if (act && nstp >= P.max_steps) {
            status = -6;
            done = true;
            act = false;
        }
        if (act && ((T + 0.1 * H == T) || (H <= P.Roundoff))) {
            status = -7;
            done = true;
            act = false;
        }
        if (!TM && !act) continue;
        const double Ha = act ? H : 1.0;
        const double ghinv = 1.0 / (dir * Ha * RADM2_ROS_GAMMA0);
        if (TM) __syncwarp();
        // G = -J(Y) + ghinv I in the LU slots, factored.
        int sing;
        if constexpr (TM || !RADM2_JACLU) {
            ph_jac<BS, LUT, TM>(rcy + RCY_Y * BS, rcy + RCY_RC * BS, sg, fix0, fix1, ghinv, tb);
            sing = ph_decomp<BS, LUT, TM>(sg, tb);
        } else {
            sing = ph_jaclu<BS, LUT>(rcy + RCY_Y * BS, rcy + RCY_RC * BS, sg, fix0, fix1, ghinv);
        }
        if (act && sing) {
            status = -8;
            done = true;
            act = false;
        }
        if (!TM && !act) continue;
        const double hc21 = RADM2_ROS_C0 / (dir * Ha);
        const double hc31 = RADM2_ROS_C1 / (dir * Ha);
        const double hc32 = RADM2_ROS_C2 / (dir * Ha);

#pragma unroll 1
        for (int stage = 0; stage < 3; stage++) {
            if (TM) __syncwarp();
            ph_stage<BS, LUT, IR, TM>(stage, rcy + RCY_Y * BS, rcy + RCY_RC * BS, vec, sg, fix0, fix1, hc21, hc31, hc32,
                                      ghinv, a.refine, tb);
        }
        if (!act) continue;
        nstp++;

        // Error norm and step control (mgpu.cu:3223-3260).
        double err = 0.0;
#pragma unroll
        for (int i = 0; i < NVAR; i++) {
            const double k0 = VW(VEC_K1 + i), k1 = VW(VEC_K2 + i), k2 = VW(VEC_K3 + i);
            const double y = RW(RCY_Y + i);
            const double ynew = P.M[0] * k0 + P.M[1] * k1 + P.M[2] * k2 + y;
            const double yerr = P.E[0] * k0 + P.E[1] * k1 + P.E[2] * k2;
            const double ymax = maxd(absd(y), absd(ynew));
            const double scale = P.AbsTol[i] + P.RelTol[i] * ymax;
#if RADM2_ACCEPT_RCP
            err += (yerr * yerr) * __drcp_rn(scale * scale);
#else
            err += (yerr * yerr) / (scale * scale);
#endif
            VW(VEC_TMP + i) = ynew;
        }
        err = sqrt(err / (double)NVAR);
        const double fac = mind(P.FacMax, maxd(P.FacMin, P.FacSafe / pow(err, 1.0 / RADM2_ROS_ELO)));
        double hnew = H * fac;
        if (err != err) hnew = H * P.FacRej;  // non-finite norm: shrink hard and retry
        if ((err <= 1.0) || (H <= P.Hmin)) {
#pragma unroll
            for (int i = 0; i < NVAR; i++) RW(RCY_Y + i) = VW(VEC_TMP + i);
            T += dir * H;
            if (rlast) hnew = mind(hnew, H);
            rlast = 0;
            rmore = 0;
            if (nacc == 0) hfirst = H;
            nacc++;
            H = hnew;
            outer = true;
        } else {
            if (rmore) hnew = H * P.FacRej;
            rmore = rlast;
            rlast = 1;
            nrej++;
            H = hnew;
        }
    }
    if constexpr (TM) {  // every warp is done with its tensor memory: warp 0 frees it
        asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
        asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
        __syncthreads();
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        if (threadIdx.x < 32)
            asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(talloc), "r"(TCOLS)
                         : "memory");
    }
#undef RW
#undef VW
#undef G
}

}  // namespace radm2
