// The cooperative per-cell ROS-3 solver kernel: a cell's working set on chip.
//
// A thread block holds 32 cells, one per lane, and G warps ("roles").  Every warp runs
// lane-per-cell SIMT code over the block's 32 cells, but each phase of a step attempt is
// split between the G roles (the split is generated by mech/emit_coop.py):
//   RHS                  each role sums the right-hand side of the species it owns
//   Jacobian             each role forms its share of the 659 slots, G = -J + I/(h gamma)
//   LU                   each role eliminates its rows (row-Doolittle, mgpu.cu:2746-2779);
//                        a row that needs another role's pivot row waits on that row's flag
//   solves               forward rows, a block barrier, backward rows, likewise with flags
//   stage vectors        each role keeps Fcn0, K1, K2, K3 of its own species in registers
//   error norm           each role writes the terms of its species; every role then sums
//                        all 59 in species order (the sequential sum of mgpu.cu:3223-3238),
//                        so every role takes the same step-control decision
// So one cell is served by G lanes (one in each warp), and its LU (5.3 KB), state, stage
// right-hand side and RHS values live in shared memory: 32 cells x 836 words = 214 KB per
// block, one block per SM.  The rate constants of the block's cells are copied once per cell
// into a small per-block slot array in global memory, [156][32] per block (40 KB, L1/L2
// resident), so that every read is a fixed offset from the lane's base address; per step
// attempt nothing else of a cell touches global memory.
//
// Cells come from the same work queue as the persistent schedule: lanes whose cell
// finished take the next queue entries (warp-aggregated atomic in role 0) between
// attempts, so lanes never wait for the slowest cell of the block.
//
// Waits on another role's row flag are bounded (COOP_WAIT_CYCLES of the SM clock, about
// one second); a wait that runs out marks the block's cells with status RADM2_E_CUDA and
// the block returns, so a fault in the schedule ends the launch with an error instead of
// hanging the GPU.
//
// This header is included by one instantiation file per kernel, which defines
//   RADM2_COOP_G       roles (warps) per block: 4 or 8
//   RADM2_COOP_RECIP   1 = reciprocal pivots (the fast form), 0 = the reference's divisions
//                      (that file is compiled without multiply-add contraction)
//   RADM2_COOP_KERNEL  the kernel's name
//   RADM2_COOP_TABLES  0 (default): the unrolled per-role LU and solve code; 1: the LU and
//                      the triangular solves run from per-role operation tables
//                      (gen/radm2_coop_g<G>_ops.h) through a small interpreter.  The
//                      tables end the instruction-fetch stalls but execute 2.4x the
//                      instructions; measured 27% slower on B200, so not the default.
#pragma once

#include "radm2_device.cuh"

#ifndef RADM2_COOP_TABLES
#define RADM2_COOP_TABLES 0
#endif

#if RADM2_COOP_G == 4
#include "gen/radm2_coop_g4.h"
#if RADM2_COOP_TABLES
#include "gen/radm2_coop_g4_ops.h"
#endif
#define RADM2_COOP_NS RADM2_COOP_G4_NS
#define RADM2_COOP_OWN_INC "gen/radm2_coop_g4_own.inc"
#define RADM2_COOP_FUN_INC "gen/radm2_coop_g4_fun.inc"
#define RADM2_COOP_JAC_INC "gen/radm2_coop_g4_jac.inc"
#define RADM2_COOP_FWD_INC "gen/radm2_coop_g4_fwd.inc"
#if RADM2_COOP_RECIP
#define RADM2_COOP_LU_INC "gen/radm2_coop_g4_lu.inc"
#define RADM2_COOP_BWD_INC "gen/radm2_coop_g4_bwd.inc"
#else
#define RADM2_COOP_LU_INC "gen/radm2_coop_g4_lu_div.inc"
#define RADM2_COOP_BWD_INC "gen/radm2_coop_g4_bwd_div.inc"
#endif
#elif RADM2_COOP_G == 8
#include "gen/radm2_coop_g8.h"
#if RADM2_COOP_TABLES
#include "gen/radm2_coop_g8_ops.h"
#endif
#define RADM2_COOP_NS RADM2_COOP_G8_NS
#define RADM2_COOP_OWN_INC "gen/radm2_coop_g8_own.inc"
#define RADM2_COOP_FUN_INC "gen/radm2_coop_g8_fun.inc"
#define RADM2_COOP_JAC_INC "gen/radm2_coop_g8_jac.inc"
#define RADM2_COOP_FWD_INC "gen/radm2_coop_g8_fwd.inc"
#if RADM2_COOP_RECIP
#define RADM2_COOP_LU_INC "gen/radm2_coop_g8_lu.inc"
#define RADM2_COOP_BWD_INC "gen/radm2_coop_g8_bwd.inc"
#else
#define RADM2_COOP_LU_INC "gen/radm2_coop_g8_lu_div.inc"
#define RADM2_COOP_BWD_INC "gen/radm2_coop_g8_bwd_div.inc"
#endif
#else
#error "RADM2_COOP_G must be 4 or 8"
#endif

namespace radm2 {

// Shared-memory layout of a block, in doubles: word w of lane l at w * 32 + l.
constexpr int COOP_LU = 0;                     // the 659 LU slots
constexpr int COOP_Y = NJVS;                   // state Y
constexpr int COOP_X = NJVS + NVAR;            // stage right-hand side / solution, error terms
constexpr int COOP_F = NJVS + 2 * NVAR;        // RHS values, each role its own species
constexpr int COOP_DWORDS = NJVS + 3 * NVAR;   // 836
// then ints
constexpr int COOP_FLAG_LU = 0;                // [64] LU row flags
constexpr int COOP_FLAG_SV = 64;               // [64] solve row flags
constexpr int COOP_FLAG_NEVER = 127;           // a flag no row sets (wait-limit self-test)
constexpr int COOP_CELL = 128;                 // [32] cell taken by each lane (-1: none)
constexpr int COOP_SING = 160;                 // [32] zero pivot seen in this attempt
constexpr int COOP_ERR = 192;                  // block error flag (a wait ran out)
constexpr int COOP_IWORDS = 224;
constexpr size_t COOP_SMEM_BYTES = (size_t)COOP_DWORDS * 32 * sizeof(double) + COOP_IWORDS * sizeof(int);
static_assert(COOP_SMEM_BYTES <= 227 * 1024, "cooperative block does not fit shared memory");

constexpr long long COOP_WAIT_CYCLES = 1ll << 31;  // ~1 s at 2 GHz
constexpr int COOP_STATUS_WAIT_LIMIT = -101;        // RADM2_E_CUDA: a wait ran out
constexpr long long COOP_SELFTEST_WAIT_CYCLES = 1ll << 20;

// Publish a finished row: every lane's stores are ordered before the flag, which one lane
// sets once the whole warp has stored.  Out of line, like coop_wait: the hundreds of call
// sites would otherwise each carry a copy, and instruction fetch limits this kernel.
static __device__ __noinline__ void coop_signal(volatile int *flag, int seq)
{
    __threadfence_block();
    __syncwarp();
    if ((threadIdx.x & 31) == 0) {
        __threadfence_block();
        *flag = seq;
    }
}

// Wait until another role published the row (flag >= seq), at most `limit` SM cycles;
// returns 1 if the wait ran out.  Callers skip later waits once one has run out (the block
// then only runs on to its error exit at the end of the attempt).
static __device__ __noinline__ int coop_wait(volatile int *flag, int seq, long long limit)
{
    int out = 0;
    if (*flag < seq) {
        const long long t0 = clock64();
        while (*flag < seq) {
            if (clock64() - t0 > limit) {
                out = 1;
                break;
            }
        }
    }
    __threadfence_block();  // the row's loads stay after the flag
    return out;
}
#define COOP_WAIT_ON(flag, seq, limit) \
    do {                               \
        if (!werr) werr = coop_wait((flag), (seq), (limit)); \
    } while (0)

// RHS of the role's own species at state vb (shared memory, word-major), written to fs
// (the same layout, the role's species only).  Out of line: the step loop needs it at two
// places (Fcn0 and the stage-2 right-hand side) and one copy of the code is enough.
static __device__ __noinline__ void coop_fun(int role, const double *vb, const double *rcs, double fix0, double fix1,
                                     double *fs)
{
    const int lane = threadIdx.x & 31;
#define COOP_ROLE role
#define RC(r) rcs[(r) * 32]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define V(i) vb[(i) * 32 + lane]
#define COOP_FENCE asm volatile("" ::: "memory")
#define FUN_OUT(k, s, e) fs[(s) * 32 + lane] = (e)
#include RADM2_COOP_FUN_INC
#undef FUN_OUT
#undef COOP_FENCE
#undef V
#undef FIX
#undef RC
#undef COOP_ROLE
}

#if RADM2_COOP_TABLES
// ---- table-driven LU and triangular solves
// Every role runs the same few loops over its own operation words, so the instruction cache
// holds one small interpreter instead of every role's unrolled rows.  A word is
// opcode << 28 | A << 18 | B << 8 | C; the streams (mech/emit_coop.py) keep each slot's
// operations in the order of the unrolled row blocks, so results are the same.
enum : unsigned {
    COOP_OP_END = 0, COOP_OP_CHECK = 1, COOP_OP_WAIT = 2, COOP_OP_PIVOT = 3, COOP_OP_UPD = 4, COOP_OP_RCP = 5,
    COOP_OP_DONE = 6, COOP_OP_ROW = 7, COOP_OP_TERM = 8, COOP_OP_STORE = 9, COOP_OP_STORE_DIAG = 10
};
#define COOP_FA(w) (((w) >> 18) & 1023u)
#define COOP_FB(w) (((w) >> 8) & 1023u)
#define COOP_FC(w) ((w)&255u)

// LU: CHECK(diag) records a zero pivot; WAIT(row) waits for another role's finished row;
// PIVOT(slot i,j; diag j; n) forms the multiplier and is followed by n UPD(slot i,k; slot
// j,k) updates, four at a time (distinct targets, sources in the pivot row); RCP(diag) stores
// the reciprocal pivot; DONE(row) publishes the row.
static __device__ __forceinline__ int coop_lu_run(const unsigned *p, double *lu, int lane, volatile int *flags,
                                                 int seq, int werr, int *sing)
{
    double *const L = lu + lane;  // slot s of this lane's cell at L[s * 32]
    for (;;) {
        const unsigned w = __ldg(p);
        const unsigned op = w >> 28;
        if (op == COOP_OP_PIVOT) {
            const unsigned n = COOP_FC(w);
#if RADM2_COOP_RECIP
            const double a = -L[COOP_FA(w) * 32] * L[COOP_FB(w) * 32];
#else
            const double a = -L[COOP_FA(w) * 32] / L[COOP_FB(w) * 32];
#endif
            L[COOP_FA(w) * 32] = -a;
            p++;
            unsigned q = 0;
            for (; q + 4 <= n; q += 4, p += 4) {
                const unsigned w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
                const double u0 = L[COOP_FB(w0) * 32], u1 = L[COOP_FB(w1) * 32], u2 = L[COOP_FB(w2) * 32],
                             u3 = L[COOP_FB(w3) * 32];
                const double v0 = L[COOP_FA(w0) * 32], v1 = L[COOP_FA(w1) * 32], v2 = L[COOP_FA(w2) * 32],
                             v3 = L[COOP_FA(w3) * 32];
                L[COOP_FA(w0) * 32] = v0 + a * u0;
                L[COOP_FA(w1) * 32] = v1 + a * u1;
                L[COOP_FA(w2) * 32] = v2 + a * u2;
                L[COOP_FA(w3) * 32] = v3 + a * u3;
            }
            for (; q < n; q++, p++) {
                const unsigned w0 = __ldg(p);
                L[COOP_FA(w0) * 32] = L[COOP_FA(w0) * 32] + a * L[COOP_FB(w0) * 32];
            }
            continue;
        }
        p++;
        if (op == COOP_OP_END) break;
        if (op == COOP_OP_CHECK) {
            if (L[COOP_FA(w) * 32] == 0.0) sing[lane] = 1;
        } else if (op == COOP_OP_WAIT) {
            if (!werr) werr = coop_wait(flags + COOP_FC(w), seq, COOP_WAIT_CYCLES);
        } else if (op == COOP_OP_RCP) {
            L[COOP_FA(w) * 32] = 1.0 / L[COOP_FA(w) * 32];
        } else if (op == COOP_OP_DONE) {
            coop_signal(flags + COOP_FC(w), seq);
        }
    }
    return werr;
}

// Triangular solve rows: ROW(k; n) starts x_k's sum, n TERM(slot; j) subtract G(slot) x_j in
// the row's order, STORE(k) or STORE_DIAG(k; diag) ends it (the backward rows times the
// reciprocal pivot, or divided by the pivot); WAIT and DONE as for the LU.
static __device__ __forceinline__ int coop_solve_run(const unsigned *p, const double *lu, double *xs, int lane,
                                                    volatile int *flags, int seq, int werr)
{
    const double *const L = lu + lane;
    double *const X = xs + lane;
    for (;;) {
        const unsigned w = __ldg(p++);
        const unsigned op = w >> 28;
        if (op == COOP_OP_ROW) {
            const unsigned n = COOP_FC(w);
            double acc = X[COOP_FA(w) * 32];
            unsigned q = 0;
            for (; q + 4 <= n; q += 4, p += 4) {
                const unsigned w0 = __ldg(p), w1 = __ldg(p + 1), w2 = __ldg(p + 2), w3 = __ldg(p + 3);
                const double g0 = L[COOP_FA(w0) * 32], g1 = L[COOP_FA(w1) * 32], g2 = L[COOP_FA(w2) * 32],
                             g3 = L[COOP_FA(w3) * 32];
                const double x0 = X[COOP_FB(w0) * 32], x1 = X[COOP_FB(w1) * 32], x2 = X[COOP_FB(w2) * 32],
                             x3 = X[COOP_FB(w3) * 32];
                acc = acc - g0 * x0;
                acc = acc - g1 * x1;
                acc = acc - g2 * x2;
                acc = acc - g3 * x3;
            }
            for (; q < n; q++, p++) {
                const unsigned w0 = __ldg(p);
                acc = acc - L[COOP_FA(w0) * 32] * X[COOP_FB(w0) * 32];
            }
            const unsigned we = __ldg(p++);
            if ((we >> 28) == COOP_OP_STORE) {
                X[COOP_FA(we) * 32] = acc;
            } else {
#if RADM2_COOP_RECIP
                X[COOP_FA(we) * 32] = acc * L[COOP_FB(we) * 32];
#else
                X[COOP_FA(we) * 32] = acc / L[COOP_FB(we) * 32];
#endif
            }
        } else if (op == COOP_OP_END) {
            break;
        } else if (op == COOP_OP_WAIT) {
            if (!werr) werr = coop_wait(flags + COOP_FC(w), seq, COOP_WAIT_CYCLES);
        } else if (op == COOP_OP_DONE) {
            coop_signal(flags + COOP_FC(w), seq);
        }
    }
    return werr;
}
#if RADM2_COOP_RECIP
#define COOP_LU_OPS coop_lu_ops
#define COOP_LU_START coop_lu_start
#define COOP_BWD_OPS coop_bwd_ops
#define COOP_BWD_START coop_bwd_start
#else
#define COOP_LU_OPS coop_lu_div_ops
#define COOP_LU_START coop_lu_div_start
#define COOP_BWD_OPS coop_bwd_div_ops
#define COOP_BWD_START coop_bwd_div_start
#endif
#endif

__global__ void __launch_bounds__(32 * RADM2_COOP_G, 1) RADM2_COOP_KERNEL(const SolveArgs a)
{
    constexpr int NS = RADM2_COOP_NS;
    extern __shared__ double smem[];
    double *const lu = smem + COOP_LU * 32;
    double *const ys = smem + COOP_Y * 32;
    double *const xs = smem + COOP_X * 32;
    double *const fs = smem + COOP_F * 32;
    int *const ism = reinterpret_cast<int *>(smem + COOP_DWORDS * 32);
    volatile int *const vflag = ism;
    const int lane = threadIdx.x & 31;
    const int role = threadIdx.x >> 5;
    const SolveParams &P = a.p;
    const int ld = a.ld;
    const int dir = P.direction;

    for (int i = threadIdx.x; i < COOP_IWORDS; i += blockDim.x) ism[i] = (i >= COOP_CELL && i < COOP_CELL + 32) ? -1 : 0;
    __syncthreads();

    // ---- lane state, the same in every role
    bool have = false;   // the lane holds a cell
    bool fetch = true;   // the lane's cell finished (or none yet): results out, next cell in
    bool outer = false;  // the next attempt starts a step: Fcn0 first
    int cidx = 0;
    double T = 0.0, H = 0.0, fix0 = 0.0, fix1 = 0.0, hfirst = 0.0;
    int rlast = 0, rmore = 0, nacc = 0, nrej = 0, nstp = 0, status = 1;
    double *const rcs = a.scratch + (size_t)blockIdx.x * NREACT * 32 + lane;  // [156][32] per block
    // ---- the role's own species: stage vectors in registers
    double f0[NS], k1[NS], k2[NS], k3[NS];
#pragma unroll
    for (int k = 0; k < NS; k++) f0[k] = k1[k] = k2[k] = k3[k] = 0.0;
    int lu_seq = 0, sv_seq = 0, werr = 0;

#define COOP_ROLE role
#define RC(r) rcs[(r) * 32]
#define FIX(k) ((k) == 0 ? fix0 : fix1)
#define SW(base, w) (base)[(w) * 32 + lane]
#define COOP_FENCE asm volatile("" ::: "memory")

    for (;;) {
        // ================================================================ cells out / in
        if (fetch && have) {
            double *v = a.var + cidx;
#define OWN(k, s) v[(size_t)(s) * ld] = SW(ys, s);
#include RADM2_COOP_OWN_INC
#undef OWN
            if (role == 0) {
                a.status[cidx] = status;
                a.nacc[cidx] = nacc;
                a.nrej[cidx] = nrej;
                a.hfirst[cidx] = hfirst;
                a.hexit[cidx] = H;
                a.texit[cidx] = T;
            }
            have = false;
        }
        if (role == 0) {
            const unsigned m = __ballot_sync(0xffffffffu, fetch);
            if (m) {
                const int leader = __ffs(m) - 1;
                int base = 0;
                if (lane == leader) base = atomicAdd(a.queue, __popc(m));
                base = __shfl_sync(0xffffffffu, base, leader);
                if (fetch) {
                    const int c = base + __popc(m & ((1u << lane) - 1));
                    ism[COOP_CELL + lane] = c < a.ncell ? c : -1;
                }
            }
        }
        __syncthreads();
        if (fetch) {
            const int c = ism[COOP_CELL + lane];
            fetch = false;
            if (c >= 0) {
                have = true;
                cidx = a.order ? a.order[c] : c;
                const double *v = a.var + cidx;
                const double *rc = a.rconst + cidx;
                for (int r = role; r < NREACT; r += RADM2_COOP_G) rcs[r * 32] = rc[(size_t)r * ld];
#define OWN(k, s) SW(ys, s) = v[(size_t)(s) * ld];
#include RADM2_COOP_OWN_INC
#undef OWN
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
                // time-loop mask (mgpu.cu:1608-1613) and the clamp to the remaining interval
                const bool more = (dir > 0 && (T - P.Tend) + P.Roundoff <= 0.0) ||
                                  (dir < 0 && (P.Tend - T) + P.Roundoff <= 0.0);
                if (more) {
                    H = mind(H, absd(P.Tend - T));
                    outer = true;
                } else {
                    fetch = true;  // nothing to integrate: out again at the next turn
                }
            }
        }
        if (!__syncthreads_or(have)) break;  // also orders the state loads before the RHS

        // ================================================================ Fcn0 = F(Y)
        if (__syncthreads_or(outer)) {
            coop_fun(role, ys, rcs, fix0, fix1, fs);
#define OWN(k, s) \
    if (outer) f0[k] = SW(fs, s);
#include RADM2_COOP_OWN_INC
#undef OWN
        }
        outer = false;

        // ================================================================ one attempt
        bool active = have && !fetch;
        if (active && nstp >= P.max_steps) {
            status = -6;
            fetch = true;
            active = false;
        }
        if (active && ((T + 0.1 * H == T) || (H <= P.Roundoff))) {
            status = -7;
            fetch = true;
            active = false;
        }
        const double ghinv = 1.0 / (dir * H * RADM2_ROS_GAMMA0);
        // G = -J(Y) + ghinv I into the LU slots; the stage-1 right-hand side Fcn0
        {
#define V(i) SW(ys, i)
#define JAC_OUT(s, e) SW(lu, s) = -(e)
#define JAC_OUT_DIAG(s, e) SW(lu, s) = (-(e)) + ghinv
#define JAC_OUT_ZERO(s, d) SW(lu, s) = (d) ? ((-0.0) + ghinv) : (-0.0)
#include RADM2_COOP_JAC_INC
#undef JAC_OUT
#undef JAC_OUT_DIAG
#undef JAC_OUT_ZERO
#undef V
        }
#define OWN(k, s) SW(xs, s) = f0[k];
#include RADM2_COOP_OWN_INC
#undef OWN
        if (role == 0) ism[COOP_SING + lane] = 0;
        __syncthreads();

        // LU, rows split between the roles
        lu_seq++;
        if (a.coop_selftest && role == 1)  // a flag nothing sets: the bounded wait runs out
            COOP_WAIT_ON(vflag + COOP_FLAG_NEVER, lu_seq, COOP_SELFTEST_WAIT_CYCLES);
#if RADM2_COOP_TABLES
        werr = coop_lu_run(COOP_LU_OPS + __ldg(COOP_LU_START + role), lu, lane, vflag + COOP_FLAG_LU, lu_seq, werr,
                           ism + COOP_SING);
#else
        {
#define G(s) SW(lu, s)
#define LU_T double
#define LU_PIVOT_CHECK(k, v) \
    if ((v) == 0.0) ism[COOP_SING + lane] = 1
#define LU_WAIT(j) COOP_WAIT_ON(vflag + COOP_FLAG_LU + (j), lu_seq, COOP_WAIT_CYCLES)
#define LU_DONE(i) coop_signal(vflag + COOP_FLAG_LU + (i), lu_seq)
#include RADM2_COOP_LU_INC
#undef LU_WAIT
#undef LU_DONE
#undef LU_PIVOT_CHECK
#undef LU_T
#undef G
        }
#endif
        __syncthreads();
        if (active && ism[COOP_SING + lane]) {
            status = -8;
            fetch = true;
            active = false;
        }
        const double hc21 = RADM2_ROS_C0 / (dir * H);
        const double hc31 = RADM2_ROS_C1 / (dir * H);
        const double hc32 = RADM2_ROS_C2 / (dir * H);

        // ---- the three stages, one solve each: stage 1 K1 = G^-1 Fcn0; stage 2 the RHS
        // F(Y + A21 K1) + C21/h K1; stage 3 reuses that F (NewF = 0) with C31/h K1 + C32/h K2
#pragma unroll 1
        for (int stage = 0; stage < 3; stage++) {
            if (stage == 1) {
#define OWN(k, s)                                     \
    {                                                 \
        k1[k] = SW(xs, s);                            \
        SW(xs, s) = SW(ys, s) + RADM2_ROS_A0 * k1[k]; \
    }
#include RADM2_COOP_OWN_INC
#undef OWN
                __syncthreads();
                coop_fun(role, xs, rcs, fix0, fix1, fs);
                __syncthreads();  // every role has read Y + A21 K1
#define OWN(k, s)                              \
    {                                          \
        const double f = SW(fs, s);            \
        SW(xs, s) = f + k1[k] * hc21;          \
        k3[k] = f + k1[k] * hc31;              \
    }
#include RADM2_COOP_OWN_INC
#undef OWN
                __syncthreads();
            } else if (stage == 2) {
#define OWN(k, s)                          \
    {                                      \
        k2[k] = SW(xs, s);                 \
        SW(xs, s) = k3[k] + k2[k] * hc32;  \
    }
#include RADM2_COOP_OWN_INC
#undef OWN
                __syncthreads();
            }
            // forward rows (flags), barrier, backward rows (flags), barrier
#define G(s) SW(lu, s)
#define X(i) SW(xs, i)
#define SOLVE_WAIT(j) COOP_WAIT_ON(vflag + COOP_FLAG_SV + (j), sv_seq, COOP_WAIT_CYCLES)
#define SOLVE_DONE(i) coop_signal(vflag + COOP_FLAG_SV + (i), sv_seq)
            sv_seq++;
#if RADM2_COOP_TABLES
            werr = coop_solve_run(coop_fwd_ops + __ldg(coop_fwd_start + role), lu, xs, lane, vflag + COOP_FLAG_SV,
                                  sv_seq, werr);
#else
#include RADM2_COOP_FWD_INC
#endif
            __syncthreads();
            sv_seq++;
#if RADM2_COOP_TABLES
            werr = coop_solve_run(COOP_BWD_OPS + __ldg(COOP_BWD_START + role), lu, xs, lane, vflag + COOP_FLAG_SV,
                                  sv_seq, werr);
#else
#include RADM2_COOP_BWD_INC
#endif
            __syncthreads();
#undef SOLVE_WAIT
#undef SOLVE_DONE
#undef X
#undef G
        }

        // ================================================================ error norm, step control
        // (mgpu.cu:3223-3260): each role its species' terms, then every role the ordered sum
        double yn[NS];
#define OWN(k, s)                                                                   \
    {                                                                               \
        k3[k] = SW(xs, s);                                                          \
        const double y = SW(ys, s);                                                 \
        yn[k] = P.M[0] * k1[k] + P.M[1] * k2[k] + P.M[2] * k3[k] + y;              \
        const double yerr = P.E[0] * k1[k] + P.E[1] * k2[k] + P.E[2] * k3[k];      \
        const double ymax = maxd(absd(y), absd(yn[k]));                             \
        const double scale = P.AbsTol[s] + P.RelTol[s] * ymax;                      \
        SW(xs, s) = (yerr * yerr) / (scale * scale);                                \
    }
#include RADM2_COOP_OWN_INC
#undef OWN
        if (werr) ism[COOP_ERR] = 1;
        __syncthreads();
        if (ism[COOP_ERR]) {
            // a bounded wait ran out: this block's cells end with an error status
            if (role == 0 && have) a.status[cidx] = COOP_STATUS_WAIT_LIMIT;
            break;
        }
        double err = 0.0;
#pragma unroll
        for (int i = 0; i < NVAR; i++) err += SW(xs, i);
        err = sqrt(err / (double)NVAR);
        const double fac = mind(P.FacMax, maxd(P.FacMin, P.FacSafe / pow(err, 1.0 / RADM2_ROS_ELO)));
        double hnew = H * fac;
        if (err != err) hnew = H * P.FacRej;  // non-finite norm: shrink hard and retry
        if (active) {
            nstp++;
            if ((err <= 1.0) || (H <= P.Hmin)) {
#define OWN(k, s) SW(ys, s) = yn[k];
#include RADM2_COOP_OWN_INC
#undef OWN
                T += dir * H;
                if (rlast) hnew = mind(hnew, H);
                rlast = 0;
                rmore = 0;
                if (nacc == 0) hfirst = H;
                nacc++;
                H = hnew;
                const bool more = (dir > 0 && (T - P.Tend) + P.Roundoff <= 0.0) ||
                                  (dir < 0 && (P.Tend - T) + P.Roundoff <= 0.0);
                if (more) {
                    H = mind(H, absd(P.Tend - T));
                    outer = true;
                } else {
                    fetch = true;
                }
            } else {
                if (rmore) hnew = H * P.FacRej;
                rmore = rlast;
                rlast = 1;
                nrej++;
                H = hnew;
            }
        }
    }
#undef COOP_FENCE
#undef SW
#undef FIX
#undef RC
#undef COOP_ROLE
}

}  // namespace radm2
