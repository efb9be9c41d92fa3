// Internal interfaces between the C ABI (radm2_capi.cu) and the kernel files.
#pragma once

#include <cuda_runtime.h>

#include "radm2_device.cuh"

namespace radm2 {

constexpr int REDUCE_BLOCKS = 296;  // 2 x 148 SMs

// Aggregated outcome of one integration, produced on the device.
struct RunResult {
    long long nacc, nrej, nfail;
    int worst, max_att;
    double tmin, tmax, hmin;
};

// IPAR/RPAR parsing with the reference's checks and codes (mgpu.cu:3684-3811): returns 1
// or a negative IERR; fills p and the autonomous flag.
int parse_params(double Tstart, double Tend, const double *AbsTol, const double *RelTol, const double *RPAR,
                 const int *IPAR, int float_coeffs, SolveParams *p, int *autonomous);

// Add one integration's 64-bit step totals to IPAR[10..16], saturating at INT_MAX.
void add_step_counters(int *IPAR, long long nacc, long long nrej, long long nfail, int autonomous);

cudaError_t launch_rconst(int n, int ld, const double *jv, const double *temp, const double *fix,
                          const double *rcn2o5, double *rconst, cudaStream_t st);
cudaError_t launch_aos_to_soa(int n, int m, int ld, const double *aos, double *soa, cudaStream_t st);
cudaError_t launch_soa_to_aos(int n, int m, int ld, const double *soa, double *aos, cudaStream_t st);
// WRF field dimensions (i fastest) and the converted window; mirrors radm2_wrf_grid.
struct WrfGrid {
    int ni, nk, nj;
    int i0, k0, j0;
    int wi, wk, wj;
};
cudaError_t launch_convert_wrf(const WrfGrid &g, const double *ph, const double *chem, const double *rad,
                               const double *phy, const double *moist, int ld, double *var, double *fix,
                               double *temp, double *rcn, double *jv, cudaStream_t st);
cudaError_t launch_gather_rows(int n, int m, int lds, int stride, const double *src, int ldd, double *dst,
                               cudaStream_t st);
cudaError_t launch_fun(int n, int ld, const double *var, const double *fix, const double *rconst, double *vdot,
                       cudaStream_t st);
cudaError_t launch_jac(int n, int ld, const double *var, const double *fix, const double *rconst, double *jvs,
                       cudaStream_t st);
cudaError_t launch_decomp_solve(int n, int ld, int fp32, double *g, double *x, int *sing, cudaStream_t st);
size_t reduce_partials_bytes();
cudaError_t launch_reduce(int n, const int *status, const int *nacc, const int *nrej, const double *texit,
                          const double *hexit, void *partials, RunResult *out, cudaStream_t st);

// (block size, placement, min resident blocks per SM) lists of the built solver variants,
// per precision (each built for both schedules).  A min-blocks value above 1 caps the
// registers per thread (65536 / (bs * minb)) for occupancy.
#define RADM2_VARIANTS_FP64(X) X(32, 0, 1) X(64, 0, 1) X(128, 0, 1) X(256, 0, 1) X(128, 0, 3) X(128, 0, 4) X(32, 1, 1) X(32, 3, 1) \
    X(128, 4, 1) X(256, 4, 1)
// Persistent schedule only: one 128-thread CTA per SM owning all of its tensor memory
// (256 LU slots per thread), rate constants and state in shared memory (RADM2_PLACE_LU_TMEM_WIDE).
#define RADM2_VARIANTS_FP64_PERS(X) RADM2_VARIANTS_FP64(X) X(128, 10, 1)
#define RADM2_VARIANTS_FP32(X) X(64, 0, 1) X(128, 0, 1) X(256, 0, 1) X(128, 0, 3) X(128, 0, 4) X(32, 1, 1) X(64, 1, 1) X(32, 3, 1)
// Reference-arithmetic FP64 solver (radm2_opts.parity): global placement only.
#define RADM2_VARIANTS_FP64X(X) X(32, 0, 1) X(64, 0, 1) X(128, 0, 1) X(256, 0, 1) X(256, 4, 1)
#define RADM2_VARIANTS_FP64X_PERS(X) RADM2_VARIANTS_FP64X(X) X(128, 10, 1)

// Cooperative kernels (radm2_coop.cuh): 32 cells per block, G roles (warps) per block,
// one block per SM; the "x" kernel keeps the reference's arithmetic.
cudaError_t launch_solver_coop_g4(const SolveArgs &a, int grid, cudaStream_t st);
cudaError_t launch_solver_coop_g8(const SolveArgs &a, int grid, cudaStream_t st);
cudaError_t launch_solver_coopx_g8(const SolveArgs &a, int grid, cudaStream_t st);

// Two cells per thread (radm2_solver_cpt2.cuh): FP64, global placement, bs 64 or 128,
// sched 0 static / 1 persistent.
cudaError_t launch_solver_cpt2(const SolveArgs &a, int bs, int sched, int grid, cudaStream_t st);

// Static properties of one solver variant on the current device.
struct SolverInfo {
    int regs;           // registers per thread
    int local_bytes;    // local (spill) bytes per thread
    int blocks_per_sm;  // resident blocks per SM (registers and shared memory)
    int global_words;   // global-scratch doubles per thread
    int smem_bytes;     // dynamic shared memory per block
};

// Solver kernels: one launcher per (precision, schedule) file, variant key
// bs * 256 + min_blocks * 16 + place (place: bit 0 = LU in shared memory, bit 1 = rate
// constants and state in shared memory, bit 2 = LU slots in tensor memory, bit 3 = the wide
// tensor-memory map; min_blocks <= 4).
inline int variant_key(int bs, int place, int min_blocks) { return bs * 256 + min_blocks * 16 + place; }
cudaError_t launch_solver_fp64_static(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t launch_solver_fp64_persistent(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t launch_solver_fp32_static(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t launch_solver_fp32_persistent(const SolveArgs &a, int key, int grid, cudaStream_t st);
// FP32 LU without the refinement code (refine_sweeps = 0); same variant keys as fp32.
cudaError_t launch_solver_fp32d_static(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t launch_solver_fp32d_persistent(const SolveArgs &a, int key, int grid, cudaStream_t st);
// Reference-arithmetic FP64 (divisions kept, no multiply-add contraction); FP64 variant keys.
cudaError_t launch_solver_fp64x_static(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t launch_solver_fp64x_persistent(const SolveArgs &a, int key, int grid, cudaStream_t st);
cudaError_t solver_info_fp64_static(int key, SolverInfo *out);
cudaError_t solver_info_fp64_persistent(int key, SolverInfo *out);
cudaError_t solver_info_fp32_static(int key, SolverInfo *out);
cudaError_t solver_info_fp32_persistent(int key, SolverInfo *out);
cudaError_t solver_info_fp32d_static(int key, SolverInfo *out);
cudaError_t solver_info_fp32d_persistent(int key, SolverInfo *out);
cudaError_t solver_info_fp64x_static(int key, SolverInfo *out);
cudaError_t solver_info_fp64x_persistent(int key, SolverInfo *out);
cudaError_t solver_info_cpt2(int bs, int sched, SolverInfo *out);
int solver_layout_check_cpt2();
cudaError_t solver_info_coop_g4(SolverInfo *out);
cudaError_t solver_info_coop_g8(SolverInfo *out);
cudaError_t solver_info_coopx_g8(SolverInfo *out);
// Host-side bounds check of every built variant's working-set layout (0 = all in bounds).
int solver_layout_check_fp64_static();
int solver_layout_check_fp64_persistent();
int solver_layout_check_fp32_static();
int solver_layout_check_fp32_persistent();
int solver_layout_check_fp32d_static();
int solver_layout_check_fp32d_persistent();
int solver_layout_check_fp64x_static();
int solver_layout_check_fp64x_persistent();

}  // namespace radm2
