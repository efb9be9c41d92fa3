// Support kernels: rate constants, layout transposes, the batched mechanism
// kernels behind radm2_fun / radm2_jac / radm2_decomp_solve, and the reduction of
// per-cell outcomes into the IPAR/RPAR aggregates.
#include "radm2_device.cuh"
#include "radm2_internal.h"
#include "gen/radm2_wrf.h"

namespace radm2 {

// ---------------------------------------------------------------- rate constants
// dev_Update_RCONST (mgpu.cu:752-919) with a per-cell index: one thread per cell,
// struct-of-arrays in and out.
__global__ void __launch_bounds__(128) k_rconst(int n, int ld, const double *__restrict__ jv,
                                                const double *__restrict__ temp, const double *__restrict__ fix,
                                                const double *__restrict__ rcn2o5, double *__restrict__ rconst)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const double TEMP = temp[c];
    const double C_M = fix[(size_t)ld + c];
    const double RC_N2O5 = rcn2o5 ? rcn2o5[c] : 0.0;
#define JV(k) jv[(size_t)(k) * ld + c]
#define RC_OUT(r, e) rconst[(size_t)(r) * ld + c] = (e)
#include "gen/radm2_rconst.inc"
#undef RC_OUT
#undef JV
}

// ---------------------------------------------------------------- transposes
// aos[n][m] <-> soa[m][ld] through a 32x33 shared tile (coalesced both ways).
__global__ void k_aos_to_soa(int n, int m, int ld, const double *__restrict__ aos, double *__restrict__ soa)
{
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, f0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r, f = f0 + threadIdx.x;
        if (c < n && f < m) tile[r][threadIdx.x] = aos[(size_t)c * m + f];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int f = f0 + r, c = c0 + threadIdx.x;
        if (c < n && f < m) soa[(size_t)f * ld + c] = tile[threadIdx.x][r];
    }
}

__global__ void k_soa_to_aos(int n, int m, int ld, const double *__restrict__ soa, double *__restrict__ aos)
{
    __shared__ double tile[32][33];
    const int c0 = blockIdx.x * 32, f0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int f = f0 + r, c = c0 + threadIdx.x;
        if (c < n && f < m) tile[r][threadIdx.x] = soa[(size_t)f * ld + c];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int c = c0 + r, f = f0 + threadIdx.x;
        if (c < n && f < m) aos[(size_t)c * m + f] = tile[threadIdx.x][r];
    }
}

// ---------------------------------------------------------------- mechanism kernels
// dev_Fun (mgpu.cu:1084-1386): vdot[59][ld] = F(var).
__global__ void __launch_bounds__(128) k_fun(int n, int ld, const double *__restrict__ var,
                                             const double *__restrict__ fix, const double *__restrict__ rconst,
                                             double *__restrict__ vdot)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
#define V(i) var[(size_t)(i) * ld + c]
#define FIX(k) fix[(size_t)(k) * ld + c]
#define RC(r) rconst[(size_t)(r) * ld + c]
#define VDOT_OUT(i, e) vdot[(size_t)(i) * ld + c] = (e)
#include "gen/radm2_fun.inc"
#undef VDOT_OUT
}

// dev_Jac_SP (mgpu.cu:1672-2652): jvs[659][ld] = J(var) in LU slot order.
__global__ void __launch_bounds__(128) k_jac(int n, int ld, const double *__restrict__ var,
                                             const double *__restrict__ fix, const double *__restrict__ rconst,
                                             double *__restrict__ jvs)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
#define JAC_OUT(s, e) jvs[(size_t)(s) * ld + c] = (e)
#define JAC_OUT_DIAG(s, e) jvs[(size_t)(s) * ld + c] = (e)
#define JAC_OUT_ZERO(s, d) jvs[(size_t)(s) * ld + c] = 0.0
#include "gen/radm2_jac.inc"
#undef JAC_OUT
#undef JAC_OUT_DIAG
#undef JAC_OUT_ZERO
#undef V
#undef FIX
#undef RC
}

// KppDecomp + KppSolve (mgpu.cu:2726-2780, 2854-3096) on caller matrices: g[659][ld]
// is factored in place (in LUT precision, stored back as double) and x[59][ld] is
// overwritten with the solution.  sing[c] = first zero-pivot row + 1, or 0.
template <typename LUT>
__global__ void __launch_bounds__(128) k_decomp_solve(int n, int ld, double *__restrict__ g,
                                                      double *__restrict__ x, int *__restrict__ sing_out)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    LUT gl[NJVS];
#pragma unroll
    for (int s = 0; s < NJVS; s++) gl[s] = (LUT)g[(size_t)s * ld + c];
    int sing = 0;
#define G(s) gl[s]
#define LU_T LUT
#define LU_PIVOT_CHECK(k, v) \
    if (sing == 0 && (v) == (LUT)0) sing = (k) + 1
#include "gen/radm2_decomp.inc"
#undef LU_PIVOT_CHECK
#undef LU_T
    LUT xl[NVAR];
#pragma unroll
    for (int i = 0; i < NVAR; i++) xl[i] = (LUT)x[(size_t)i * ld + c];
#define X(i) xl[i]
#include "gen/radm2_solve.inc"
#undef X
#undef G
#pragma unroll
    for (int i = 0; i < NVAR; i++) x[(size_t)i * ld + c] = (double)xl[i];
#pragma unroll
    for (int s = 0; s < NJVS; s++) g[(size_t)s * ld + c] = (double)gl[s];
    sing_out[c] = sing;
}

// ---------------------------------------------------------------- outcome reduction
// Stage 1: per-block partials; stage 2: one block folds the partials into out[].
struct Partial {
    unsigned long long nacc, nrej, nfail;
    int worst, max_att;
    double tmin, tmax, hmin;
};

__device__ __forceinline__ void fold(Partial &a, const Partial &b)
{
    a.nacc += b.nacc;
    a.nrej += b.nrej;
    a.nfail += b.nfail;
    a.worst = min(a.worst, b.worst);
    a.max_att = max(a.max_att, b.max_att);
    a.tmin = fmin(a.tmin, b.tmin);
    a.tmax = fmax(a.tmax, b.tmax);
    a.hmin = fmin(a.hmin, b.hmin);
}

__device__ void block_fold(Partial &p)
{
    __shared__ Partial sh[32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) {
        Partial q;
        q.nacc = __shfl_down_sync(0xffffffffu, p.nacc, o);
        q.nrej = __shfl_down_sync(0xffffffffu, p.nrej, o);
        q.nfail = __shfl_down_sync(0xffffffffu, p.nfail, o);
        q.worst = __shfl_down_sync(0xffffffffu, p.worst, o);
        q.max_att = __shfl_down_sync(0xffffffffu, p.max_att, o);
        q.tmin = __shfl_down_sync(0xffffffffu, p.tmin, o);
        q.tmax = __shfl_down_sync(0xffffffffu, p.tmax, o);
        q.hmin = __shfl_down_sync(0xffffffffu, p.hmin, o);
        fold(p, q);
    }
    if (lane == 0) sh[w] = p;
    __syncthreads();
    if (w == 0) {
        const int nw = blockDim.x >> 5;
        p = sh[lane < nw ? lane : 0];
        for (int o = 16; o > 0; o >>= 1) {
            Partial q;
            q.nacc = __shfl_down_sync(0xffffffffu, p.nacc, o);
            q.nrej = __shfl_down_sync(0xffffffffu, p.nrej, o);
            q.nfail = __shfl_down_sync(0xffffffffu, p.nfail, o);
            q.worst = __shfl_down_sync(0xffffffffu, p.worst, o);
            q.max_att = __shfl_down_sync(0xffffffffu, p.max_att, o);
            q.tmin = __shfl_down_sync(0xffffffffu, p.tmin, o);
            q.tmax = __shfl_down_sync(0xffffffffu, p.tmax, o);
            q.hmin = __shfl_down_sync(0xffffffffu, p.hmin, o);
            if (lane + o < nw) fold(p, q);
        }
    }
}

__device__ __forceinline__ Partial empty_partial()
{
    Partial p;
    p.nacc = p.nrej = p.nfail = 0;
    p.worst = 1;
    p.max_att = 0;
    p.tmin = __longlong_as_double(0x7ff0000000000000ULL);   // +inf
    p.tmax = -__longlong_as_double(0x7ff0000000000000ULL);  // -inf
    p.hmin = __longlong_as_double(0x7ff0000000000000ULL);
    return p;
}

__global__ void __launch_bounds__(256) k_reduce_partial(int n, const int *__restrict__ status,
                                                        const int *__restrict__ nacc, const int *__restrict__ nrej,
                                                        const double *__restrict__ texit,
                                                        const double *__restrict__ hexit, Partial *__restrict__ out)
{
    Partial p = empty_partial();
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < n; c += gridDim.x * blockDim.x) {
        const int s = status[c], a = nacc[c], r = nrej[c];
        p.nacc += a;
        p.nrej += r;
        p.nfail += (s != 1);
        p.worst = min(p.worst, s);
        p.max_att = max(p.max_att, a + r);
        p.tmin = fmin(p.tmin, texit[c]);
        p.tmax = fmax(p.tmax, texit[c]);
        p.hmin = fmin(p.hmin, hexit[c]);
    }
    block_fold(p);
    if (threadIdx.x == 0) out[blockIdx.x] = p;
}

__global__ void __launch_bounds__(256) k_reduce_final(int nparts, const Partial *__restrict__ parts,
                                                      RunResult *__restrict__ out)
{
    Partial p = empty_partial();
    for (int i = threadIdx.x; i < nparts; i += blockDim.x) fold(p, parts[i]);
    block_fold(p);
    if (threadIdx.x == 0) {
        out->nacc = (long long)p.nacc;
        out->nrej = (long long)p.nrej;
        out->nfail = (long long)p.nfail;
        out->worst = p.worst;
        out->max_att = p.max_att;
        out->tmin = p.tmin;
        out->tmax = p.tmax;
        out->hmin = p.hmin;
    }
}

// ---------------------------------------------------------------- host launchers

cudaError_t launch_rconst(int n, int ld, const double *jv, const double *temp, const double *fix,
                          const double *rcn2o5, double *rconst, cudaStream_t st)
{
    (void)cudaGetLastError();
    k_rconst<<<(n + 127) / 128, 128, 0, st>>>(n, ld, jv, temp, fix, rcn2o5, rconst);
    return cudaGetLastError();
}

cudaError_t launch_aos_to_soa(int n, int m, int ld, const double *aos, double *soa, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    dim3 grid((n + 31) / 32, (m + 31) / 32), block(32, 8);
    (void)cudaGetLastError();
    k_aos_to_soa<<<grid, block, 0, st>>>(n, m, ld, aos, soa);
    return cudaGetLastError();
}

cudaError_t launch_soa_to_aos(int n, int m, int ld, const double *soa, double *aos, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    dim3 grid((n + 31) / 32, (m + 31) / 32), block(32, 8);
    (void)cudaGetLastError();
    k_soa_to_aos<<<grid, block, 0, st>>>(n, m, ld, soa, aos);
    return cudaGetLastError();
}

// ---------------------------------------------------------------- WRF -> KPP conversion
// mgpu.cu:513-646 (dev_convert), one thread per cell of the window, writing the context's
// struct-of-arrays inputs directly.  Expressions as the reference writes them (this file
// is built without FMA contraction); TEMP and RC_N2O5 per cell.
#define RADM2_NAVGDRO (6.022e23)
#define RADM2_MWAIR (28.97)
#define RADM2_MWH2O (2 * (1.0079) + (15.9994))
#define RADM2_DENS2CON_A (1.0e-3 * (1.0 / RADM2_MWAIR) * RADM2_NAVGDRO)
#define RADM2_DENS2CON_W (1.0e-3 * (1.0 / RADM2_MWH2O) * RADM2_NAVGDRO)

__global__ void k_convert_wrf(const WrfGrid g, const double *__restrict__ ph, const double *__restrict__ chem,
                              const double *__restrict__ rad, const double *__restrict__ phy,
                              const double *__restrict__ moist, int ld, double *__restrict__ var,
                              double *__restrict__ fix, double *__restrict__ temp, double *__restrict__ rcn,
                              double *__restrict__ jv)
{
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= g.wi * g.wk * g.wj) return;
    const size_t fs = (size_t)g.nj * g.nk * g.ni;
    const int ii = p % g.wi, kk = (p / g.wi) % g.wk, jj = p / (g.wi * g.wk);
    const size_t o = ((size_t)(g.j0 + jj) * g.nk + (g.k0 + kk)) * g.ni + (g.i0 + ii);
    const double pres = phy[o], t = phy[fs + o], rho = phy[2 * fs + o], qv = moist[fs + o];
    fix[(size_t)ld + p] = RADM2_DENS2CON_A * rho;
    fix[p] = RADM2_DENS2CON_W * qv * rho;
    temp[p] = t;
    const double es = 1000. * 0.6112 * exp(17.67 * (t - 273.15) / (t - 29.65));
    const double qvs = es / (pres - es);
    double rh = qv / qvs;
    rh = rh >= 0.0f ? rh : 0.0f;
    rh = rh < 1.0f ? rh : 1.0f;
    rcn[p] = 1.0 / (3.6e4 * exp(-pow((rh / 0.28), 2.8) + 300.0));
    const double conv = 1.0E-6 * RADM2_DENS2CON_A * rho;
#define RADM2_JV_OUT(k, f) jv[(size_t)(k) * ld + p] = ph[(size_t)(f) * fs + o] / 60.0;
    RADM2_WRF_JV_SRC(RADM2_JV_OUT)
#undef RADM2_JV_OUT
#define RADM2_VAR_OUT(v, src, f)                                             \
    {                                                                        \
        const double x_ = ((src) == 0 ? chem : rad)[(size_t)(f) * fs + o];   \
        var[(size_t)(v) * ld + p] = conv * (x_ >= 0.0 ? x_ : 0.0);          \
    }
    RADM2_WRF_VAR_SRC(RADM2_VAR_OUT)
#undef RADM2_VAR_OUT
}

cudaError_t launch_convert_wrf(const WrfGrid &g, const double *ph, const double *chem, const double *rad,
                               const double *phy, const double *moist, int ld, double *var, double *fix,
                               double *temp, double *rcn, double *jv, cudaStream_t st)
{
    const int n = g.wi * g.wk * g.wj;
    if (n <= 0) return cudaSuccess;
    (void)cudaGetLastError();
    k_convert_wrf<<<(n + 127) / 128, 128, 0, st>>>(g, ph, chem, rad, phy, moist, ld, var, fix, temp, rcn, jv);
    return cudaGetLastError();
}

// dst[r][i] = src[r][i * stride] for r < m, i < n (struct-of-arrays rows, leading
// dimensions lds / ldd): a strided sample of cells.
__global__ void k_gather_rows(int n, int m, int lds, int stride, const double *__restrict__ src, int ldd,
                              double *__restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int r = blockIdx.y;
    if (i < n && r < m) dst[(size_t)r * ldd + i] = src[(size_t)r * lds + (size_t)i * stride];
}

cudaError_t launch_gather_rows(int n, int m, int lds, int stride, const double *src, int ldd, double *dst,
                               cudaStream_t st)
{
    if (n <= 0 || m <= 0) return cudaSuccess;
    dim3 grid((n + 255) / 256, m);
    (void)cudaGetLastError();
    k_gather_rows<<<grid, 256, 0, st>>>(n, m, lds, stride, src, ldd, dst);
    return cudaGetLastError();
}

cudaError_t launch_fun(int n, int ld, const double *var, const double *fix, const double *rconst, double *vdot,
                       cudaStream_t st)
{
    (void)cudaGetLastError();
    k_fun<<<(n + 127) / 128, 128, 0, st>>>(n, ld, var, fix, rconst, vdot);
    return cudaGetLastError();
}

cudaError_t launch_jac(int n, int ld, const double *var, const double *fix, const double *rconst, double *jvs,
                       cudaStream_t st)
{
    (void)cudaGetLastError();
    k_jac<<<(n + 127) / 128, 128, 0, st>>>(n, ld, var, fix, rconst, jvs);
    return cudaGetLastError();
}

cudaError_t launch_decomp_solve(int n, int ld, int fp32, double *g, double *x, int *sing, cudaStream_t st)
{
    (void)cudaGetLastError();
    if (fp32)
        k_decomp_solve<float><<<(n + 127) / 128, 128, 0, st>>>(n, ld, g, x, sing);
    else
        k_decomp_solve<double><<<(n + 127) / 128, 128, 0, st>>>(n, ld, g, x, sing);
    return cudaGetLastError();
}

size_t reduce_partials_bytes() { return sizeof(Partial) * REDUCE_BLOCKS; }

cudaError_t launch_reduce(int n, const int *status, const int *nacc, const int *nrej, const double *texit,
                          const double *hexit, void *partials, RunResult *out, cudaStream_t st)
{
    Partial *parts = static_cast<Partial *>(partials);
    (void)cudaGetLastError();
    k_reduce_partial<<<REDUCE_BLOCKS, 256, 0, st>>>(n, status, nacc, nrej, texit, hexit, parts);
    k_reduce_final<<<1, 256, 0, st>>>(REDUCE_BLOCKS, parts, out);
    return cudaGetLastError();
}

}  // namespace radm2
