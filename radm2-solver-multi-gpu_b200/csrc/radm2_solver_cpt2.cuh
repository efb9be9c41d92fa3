// Two cells per thread: the thread-per-cell solver (radm2_solver.cuh) with every thread
// integrating two cells side by side.
//
// A block of BS threads holds 2 x BS cells.  Thread t owns virtual lanes t and t + BS,
// each a full cell with its own step-size loop, and runs each phase of a step attempt for
// both of them back to back, so the two cells' independent instruction streams can
// overlap in the scheduler where register pressure allows.  The working set of a virtual
// lane is the global-placement layout of the thread-per-cell kernel with a word stride of
// 2 x BS.  Cells come from the static index (cell = 2 x BS x block + virtual lane) or the
// persistent work queue, one queue entry per virtual lane.  Arithmetic is that of the
// thread-per-cell fast solver, so both give the same results.
#pragma once

#include "radm2_solver.cuh"

namespace radm2 {

template <int BS, int SCHED>
__global__ void __launch_bounds__(BS, 1) k_rosenbrock_cpt2(const SolveArgs a)
{
    constexpr int VB = 2 * BS;  // virtual lanes per block = word stride of the layout
    using L = Layout<double, PLACE_GLOBAL>;
    double *const gblk = a.scratch + (size_t)blockIdx.x * (L::global_words * VB);
    const SolveParams &P = a.p;
    const int ld = a.ld;
    const int dir = P.direction;

    int cell[2], cidx[2] = {0, 0};
    bool have[2], outer[2] = {true, true}, done[2] = {false, false};
    double T[2] = {0, 0}, H[2] = {0, 0}, fix0[2] = {0, 0}, fix1[2] = {0, 0}, hfirst[2] = {0, 0};
    int rlast[2] = {0, 0}, rmore[2] = {0, 0}, nacc[2] = {0, 0}, nrej[2] = {0, 0}, nstp[2] = {0, 0};
    int status[2] = {1, 1};

    auto vec = [&](int v) { return gblk + L::vec_off * VB + threadIdx.x + v * BS; };
    auto rcy = [&](int v) { return gblk + L::rcy_off * VB + threadIdx.x + v * BS; };
    auto lu = [&](int v) { return gblk + L::lu_off * VB + threadIdx.x + v * BS; };

    auto take = [&]() {  // next queue entry for a virtual lane (persistent schedule)
        if (SCHED == SCHED_STATIC) return a.ncell;
        const unsigned m = __activemask();
        const int lane = threadIdx.x & 31;
        const int leader = __ffs(m) - 1;
        int base = 0;
        if (lane == leader) base = atomicAdd(a.queue, __popc(m));
        base = __shfl_sync(m, base, leader);
        return base + __popc(m & ((1u << lane) - 1));
    };
    auto load_cell = [&](int v, int c) {
        cidx[v] = (SCHED == SCHED_PERSISTENT && a.order) ? a.order[c] : c;
        double *rw = rcy(v);
        const double *y = a.var + cidx[v];
#pragma unroll
        for (int i = 0; i < NVAR; i++) rw[(RCY_Y + i) * VB] = y[(size_t)i * ld];
        const double *rc = a.rconst + cidx[v];
#pragma unroll
        for (int r = 0; r < NREACT; r++) rw[(RCY_RC + r) * VB] = rc[(size_t)r * ld];
        fix0[v] = a.fix[cidx[v]];
        fix1[v] = a.fix[(size_t)ld + cidx[v]];
        T[v] = P.Tstart;
        double hs = P.Hstart;
        if (a.h0) {
            const double h = a.h0[cidx[v]];
            if (h > 0.0 && h <= P.Hmax) hs = h;  // non-finite or out of range: default
        }
        H[v] = mind(hs, P.Hmax);  // mgpu.cu:3475-3477
        if (absd(H[v]) <= 10.0 * P.Roundoff) H[v] = DELTA_MIN;
        rlast[v] = rmore[v] = nacc[v] = nrej[v] = nstp[v] = 0;
        status[v] = 1;
        hfirst[v] = 0.0;
        outer[v] = true;
        done[v] = false;
    };
    auto store_cell = [&](int v) {
        const double *rw = rcy(v);
        double *y = a.var + cidx[v];
#pragma unroll
        for (int i = 0; i < NVAR; i++) y[(size_t)i * ld] = rw[(RCY_Y + i) * VB];
        a.status[cidx[v]] = status[v];
        a.nacc[cidx[v]] = nacc[v];
        a.nrej[cidx[v]] = nrej[v];
        a.hfirst[cidx[v]] = hfirst[v];
        a.hexit[cidx[v]] = H[v];
        a.texit[cidx[v]] = T[v];
    };

#pragma unroll
    for (int v = 0; v < 2; v++) {
        cell[v] = SCHED == SCHED_STATIC ? (int)(blockIdx.x * VB + v * BS + threadIdx.x) : take();
        have[v] = cell[v] < a.ncell;
        if (have[v]) load_cell(v, cell[v]);
    }

    for (;;) {
        // Bring each virtual lane that still has work to the start of a step attempt.
#pragma unroll 1
        for (int v = 0; v < 2; v++) {
            while (have[v] && (outer[v] || done[v])) {
                if (done[v]) {
                    store_cell(v);
                    if (SCHED == SCHED_STATIC) {
                        have[v] = false;
                        break;
                    }
                    cell[v] = take();
                    have[v] = cell[v] < a.ncell;
                    if (have[v]) load_cell(v, cell[v]);
                    continue;
                }
                // time-loop mask (mgpu.cu:1608-1613)
                const bool more = (dir > 0 && (T[v] - P.Tend) + P.Roundoff <= 0.0) ||
                                  (dir < 0 && (P.Tend - T[v]) + P.Roundoff <= 0.0);
                if (!more) {
                    done[v] = true;
                    continue;
                }
                H[v] = mind(H[v], absd(P.Tend - T[v]));
                ph_fun<VB>(rcy(v) + RCY_Y * VB, rcy(v) + RCY_RC * VB, vec(v) + VEC_F0 * VB, fix0[v], fix1[v]);
                outer[v] = false;
            }
        }
        if (!__any_sync(0xffffffffu, have[0] || have[1])) break;

        // ---- one attempt of each virtual lane that has a cell, phase by phase
        bool go[2];
        double ghinv[2];
#pragma unroll
        for (int v = 0; v < 2; v++) {
            go[v] = have[v];
            if (go[v] && nstp[v] >= P.max_steps) {
                status[v] = -6;
                done[v] = true;
                go[v] = false;
            }
            if (go[v] && ((T[v] + 0.1 * H[v] == T[v]) || (H[v] <= P.Roundoff))) {
                status[v] = -7;
                done[v] = true;
                go[v] = false;
            }
            ghinv[v] = 1.0 / (dir * H[v] * RADM2_ROS_GAMMA0);
        }
#if RADM2_JACLU
#pragma unroll
        for (int v = 0; v < 2; v++)
            if (go[v] && ph_jaclu<VB, double>(rcy(v) + RCY_Y * VB, rcy(v) + RCY_RC * VB, lu(v), fix0[v], fix1[v],
                                              ghinv[v])) {
                status[v] = -8;
                done[v] = true;
                go[v] = false;
            }
#else
#pragma unroll
        for (int v = 0; v < 2; v++)
            if (go[v]) ph_jac<VB, double>(rcy(v) + RCY_Y * VB, rcy(v) + RCY_RC * VB, lu(v), fix0[v], fix1[v], ghinv[v]);
#pragma unroll
        for (int v = 0; v < 2; v++)
            if (go[v] && ph_decomp<VB, double>(lu(v))) {
                status[v] = -8;
                done[v] = true;
                go[v] = false;
            }
#endif
#pragma unroll 1
        for (int stage = 0; stage < 3; stage++) {
#pragma unroll
            for (int v = 0; v < 2; v++)
                if (go[v])
                    ph_stage<VB, double, 1>(stage, rcy(v) + RCY_Y * VB, rcy(v) + RCY_RC * VB, vec(v), lu(v), fix0[v],
                                            fix1[v], RADM2_ROS_C0 / (dir * H[v]), RADM2_ROS_C1 / (dir * H[v]),
                                            RADM2_ROS_C2 / (dir * H[v]), ghinv[v], 0);
        }
#pragma unroll
        for (int v = 0; v < 2; v++) {
            if (!go[v]) continue;
            nstp[v]++;
            double *vw = vec(v), *rw = rcy(v);
            // error norm and step control (mgpu.cu:3223-3260)
            double err = 0.0;
#pragma unroll
            for (int i = 0; i < NVAR; i++) {
                const double k0 = vw[(VEC_K1 + i) * VB], k1 = vw[(VEC_K2 + i) * VB], k2 = vw[(VEC_K3 + i) * VB];
                const double y = rw[(RCY_Y + i) * VB];
                const double ynew = P.M[0] * k0 + P.M[1] * k1 + P.M[2] * k2 + y;
                const double yerr = P.E[0] * k0 + P.E[1] * k1 + P.E[2] * k2;
                const double ymax = maxd(absd(y), absd(ynew));
                const double scale = P.AbsTol[i] + P.RelTol[i] * ymax;
                err += (yerr * yerr) / (scale * scale);
                vw[(VEC_TMP + i) * VB] = ynew;
            }
            err = sqrt(err / (double)NVAR);
            const double fac = mind(P.FacMax, maxd(P.FacMin, P.FacSafe / pow(err, 1.0 / RADM2_ROS_ELO)));
            double hnew = H[v] * fac;
            if (err != err) hnew = H[v] * P.FacRej;  // non-finite norm: shrink hard and retry
            if ((err <= 1.0) || (H[v] <= P.Hmin)) {
#pragma unroll
                for (int i = 0; i < NVAR; i++) rw[(RCY_Y + i) * VB] = vw[(VEC_TMP + i) * VB];
                T[v] += dir * H[v];
                if (rlast[v]) hnew = mind(hnew, H[v]);
                rlast[v] = 0;
                rmore[v] = 0;
                if (nacc[v] == 0) hfirst[v] = H[v];
                nacc[v]++;
                H[v] = hnew;
                outer[v] = true;
            } else {
                if (rmore[v]) hnew = H[v] * P.FacRej;
                rmore[v] = rlast[v];
                rlast[v] = 1;
                nrej[v]++;
                H[v] = hnew;
            }
        }
    }
}

}  // namespace radm2
