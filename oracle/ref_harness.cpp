// Host shim around the reference's own per-cell mechanism functions (cut from
// mgpu.cu by oracle/build_ref.py into oracle/_ref/ref_extract.inc).
//
// TEST INFRASTRUCTURE ONLY: it exists to pin the CPU oracle against the
// reference's code.  Each wrapper runs one kernel body for one cell (p == 0):
// CUDA qualifiers become no-ops, blockIdx/threadIdx/blockDim/gridDim are host
// variables, and the LU_DIAG/CROW/ICOL texture fetches (mgpu.cu:201-206)
// read the CSR tables recovered from dev_KppSolve, which the reference
// declares but never fills (mgpu.cu:197-207).
#include <math.h>
#include <string.h>

#include "../radm2-solver-multi-gpu_b200/csrc/gen/radm2_gen.h"

struct shim_dim3 {
    unsigned x, y, z;
};
static shim_dim3 blockIdx = {0, 0, 0}, threadIdx = {0, 0, 0}, blockDim = {1, 1, 1}, gridDim = {1, 1, 1};

static const int ref_lu_crow[] = RADM2_LU_CROW_INIT;
static const int ref_lu_diag[] = RADM2_LU_DIAG_INIT;
static const int ref_lu_icol[] = RADM2_LU_ICOL_INIT;
#define LU_DIAG(k) ref_lu_diag[k]
#define LU_CROW(k) ref_lu_crow[k]
#define LU_ICOL(k) ref_lu_icol[k]

// Dynamic shared memory of dev_KppDecomp / dev_KppSolve: one cell's worth.
double share_W[64];
double shared_X[64];

#define __global__ static
#define __device__ static inline
#define __host__
#define __shared__

#include "ref_extract.inc"

extern "C" {

void ref_rconst(const double *jv, const double *fix, const double *rc_n2o5, const double *temp, double *rconst)
{
    dev_Update_RCONST(rconst, (double *)jv, (double *)fix, (double *)rc_n2o5, (double *)temp);
}

void ref_fun(const double *v, const double *f, const double *rct, double *vdot)
{
    dev_Fun(1, (double *)v, (double *)f, (double *)rct, vdot);
}

void ref_jac(const double *v, const double *f, const double *rct, double *jvs)
{
    dev_Jac_SP(1, (double *)v, (double *)f, (double *)rct, jvs);
}

int ref_decomp(double *jvs)
{
    int m1 = 1, m2 = 1, ret = 0;
    dev_KppDecomp(&m1, &m2, 1, jvs, &ret);
    return ret;
}

void ref_solve(const double *jvs, double *x)
{
    int m1 = 1, m2 = 1;
    dev_KppSolve(&m1, &m2, 1, (double *)jvs, x);
}

// dev_convert over the reference's launch (mgpu.cu:682-706): gridDim (19, 39), blockDim 39.
// The kernel writes *TEMP and *RC_N2O5 without a cell offset; the wrapper hands it the
// cell's own element so every cell's value is kept.
void ref_convert_wrf(const double *ph, const double *chem, const double *rad, const double *phy, const double *moist,
                     double *VAR, double *FIX, double *TEMP, double *RC_N2O5, double *JV)
{
    gridDim = {19, 39, 1};
    blockDim = {39, 1, 1};
    for (unsigned by = 0; by < 39; by++)
        for (unsigned bx = 0; bx < 19; bx++)
            for (unsigned tx = 0; tx < 39; tx++) {
                blockIdx = {bx, by, 0};
                threadIdx = {tx, 0, 0};
                const size_t p = (size_t)by * 19 * 39 + bx * 39 + tx;
                dev_convert(VAR, FIX, TEMP + p, nullptr, RC_N2O5 + p, JV, (double *)ph, (double *)chem, (double *)rad,
                            (double *)phy, (double *)moist);
            }
    gridDim = {1, 1, 1};
    blockDim = {1, 1, 1};
    blockIdx = {0, 0, 0};
    threadIdx = {0, 0, 0};
}

}  // extern "C"
