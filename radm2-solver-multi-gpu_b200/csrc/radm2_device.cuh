// Device-side building blocks shared by every RADM2 kernel: rate laws, the
// solver's parameter block and the per-thread scratch layout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "gen/radm2_gen.h"

namespace radm2 {

constexpr int NVAR = RADM2_NVAR;
constexpr int NFIX = RADM2_NFIX;
constexpr int NREACT = RADM2_NREACT;
constexpr int NJVS = RADM2_LU_NONZERO;
constexpr int NPH = RADM2_NPH;
constexpr double DELTA_MIN = 1.0e-6;  // mgpu.cu:15

// ---------------------------------------------------------------- rate laws (mgpu.cu:708-750)
// Written out in the same evaluation order as the reference so CPU and GPU round alike
// apart from the math library's exp/pow/log10.

__device__ __forceinline__ double rk_arr2(double a0, double b0, double temp) { return a0 * exp(-b0 / temp); }

__device__ __forceinline__ double rk_troe(double k0_300, double n, double kinf_300, double m, double temp,
                                          double cair)
{
    const double zt = 300.0 / temp;
    const double k0 = k0_300 * pow(zt, n) * cair;
    const double kinf = kinf_300 * pow(zt, m);
    const double ratio = k0 / kinf;
    const double lg = log10(ratio);
    return k0 / (1.0 + ratio) * pow(0.6, 1.0 / (1.0 + pow(lg, 2.0)));
}

__device__ __forceinline__ double rk_troee(double a, double b, double k0_300, double n, double kinf_300,
                                           double m, double temp, double cair)
{
    const double zt = 300.0 / temp;
    const double k0 = k0_300 * pow(zt, n) * cair;
    const double kinf = kinf_300 * pow(zt, m);
    const double ratio = k0 / kinf;
    const double lg = log10(ratio);
    const double troe = k0 / (1.0 + ratio) * pow(0.6, 1.0 / (1.0 + pow(lg, 2.0)));
    return a * exp(-b / temp) * troe;
}

__device__ __forceinline__ double rk_thermal_t2(double c, double d, double temp)
{
    return pow(temp, 2.0) * c * exp(-d / temp);
}

__device__ __forceinline__ double rk_k46(double cair, double temp)
{
    const double k0 = 7.2e-15 * exp(785.0 / temp);
    const double k2 = 4.1e-16 * exp(1440.0 / temp);
    const double k3 = 1.9e-33 * exp(725.0 / temp) * cair;
    return k0 + k3 / (1.0 + k3 / k2);
}

// ---------------------------------------------------------------- solver parameters

// Integration parameters after IPAR/RPAR parsing (mgpu.cu:3684-3800), passed by value
// so the tolerance vectors sit in the constant bank.
struct SolveParams {
    double Tstart, Tend;
    double Hmin, Hmax, Hstart;
    double FacMin, FacMax, FacRej, FacSafe;
    double Roundoff;
    double M[3], E[3];  // ROS-3 M and E (float-rounded in reference-parity mode)
    double AbsTol[NVAR], RelTol[NVAR];
    int max_steps;      // per-cell attempt cap (>0)
    int direction;      // +1 / -1
};

struct SolveArgs {
    SolveParams p;
    int ncell;
    int ld;                  // leading dimension of the struct-of-arrays cell arrays
    double *var;             // [NVAR][ld] species, in/out
    const double *fix;       // [NFIX][ld] H2O, M
    const double *rconst;    // [NREACT][ld]
    const double *h0;        // optional per-cell starting step
    const int *order;        // optional cell permutation (persistent schedule)
    int *queue;              // work counter (persistent schedule)
    double *scratch;         // per-block slot arrays, SCR_WORDS * blockDim doubles per block
    int *status;             // per-cell outcome
    int *nacc, *nrej;
    double *hfirst, *hexit, *texit;
    int refine;              // FP32 LU: FP64 refinement sweeps per stage solve
    int coop_selftest;       // cooperative kernel: one role waits on a flag nothing sets
};

// Per-thread scratch, in double words.  Laid out word-major inside each block
// (word w of thread t at block_base + w*BS + t) so every access is coalesced and
// carries a compile-time offset.
constexpr int SCR_RC = 0;
constexpr int SCR_Y = SCR_RC + NREACT;
constexpr int SCR_F0 = SCR_Y + NVAR;
constexpr int SCR_K1 = SCR_F0 + NVAR;
constexpr int SCR_K2 = SCR_K1 + NVAR;
constexpr int SCR_K3 = SCR_K2 + NVAR;
constexpr int SCR_TMP = SCR_K3 + NVAR;
constexpr int SCR_G = SCR_TMP + NVAR;                 // LU slots start here
constexpr int SCR_WORDS_FP64 = SCR_G + NJVS;          // 1110 doubles = 8880 B per thread
constexpr int SCR_WORDS_FP32 = SCR_G + (NJVS + 1) / 2;  // LU stored as float

template <typename LUT>
struct ScratchWords {
    static constexpr int value = sizeof(LUT) == 8 ? SCR_WORDS_FP64 : SCR_WORDS_FP32;
};

// Reference comparison macros (mgpu.cu:191-195) as ternaries, to keep NaN behaviour.
__device__ __forceinline__ double maxd(double a, double b) { return (a >= b) ? a : b; }
__device__ __forceinline__ double mind(double b, double c) { return (b < c) ? b : c; }
__device__ __forceinline__ double absd(double x) { return (x >= 0) ? x : -x; }

}  // namespace radm2
