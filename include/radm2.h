/*
 * radm2.h -- C ABI of the B200 batched RADM2 Rosenbrock (ROS-3) chemistry solver.
 *
 * Drop-in for the reference's host path (Rizkyanno/RADM2-Solver-Multi-GPU, mgpu.cu):
 * the reference keeps its per-cell arrays in library-owned device globals, fills
 * them with dev_convert, computes rate constants with updatingCoefficientWRFChemData()
 * and integrates every cell with Rosenbrock(Tstart, Tend, AbsTol, RelTol, RPAR, IPAR).
 * Here the device arrays live in a context; the same three steps are
 * radm2_set_inputs, radm2_update_rconst and radm2_rosenbrock, with the reference's
 * argument meaning, IPAR/RPAR conventions and IERR codes.
 *
 * Conventions: every function returns RADM2_OK (0) or a negative RADM2_E* code,
 * except radm2_rosenbrock / radm2_run_split, which return the reference's IERR
 * (1 = success, -1..-8 = Rosenbrock error, see radm2_error_string) or a RADM2_E*
 * code (<= -100) for API/CUDA failures.  No function prints or exits.  A context
 * is used by one host thread at a time; different contexts are independent.
 * Host arrays are in the reference's per-cell (array-of-structs) layout; the
 * library keeps struct-of-arrays copies in device memory.
 */
#ifndef RADM2_H
#define RADM2_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RADM2_NVAR 59        /* variable species (mgpu.cu:18) */
#define RADM2_NFIX 2         /* fixed species: [0] H2O, [1] M (mgpu.cu:20, 191-192) */
#define RADM2_NREACT 156     /* reactions / rate constants (mgpu.cu:21) */
#define RADM2_NPH 28         /* photolysis rates per cell (mgpu.cu:48) */
#define RADM2_LU_NONZERO 659 /* LU slots (mgpu.cu:25) */

/* API / runtime error codes (Rosenbrock's own IERR codes are -1..-8). */
#define RADM2_OK 0
#define RADM2_E_ARG (-100)      /* bad argument (null pointer, size, option) */
#define RADM2_E_CUDA (-101)     /* CUDA runtime error; radm2_last_error has the text */
#define RADM2_E_NOMEM (-102)    /* device allocation failed */
#define RADM2_E_STATE (-103)    /* call out of order (e.g. rosenbrock before set_inputs) */
#define RADM2_E_NODEV (-104)    /* no usable sm_100 device */
#define RADM2_E_TOOBIG (-105)   /* size exceeds a documented maximum */

/* Solver variants. */
#define RADM2_PREC_FP64 0    /* plain FP64 method (reference parity) */
#define RADM2_PREC_FP32LU 1  /* FP32 Jacobian/LU + FP64 iterative refinement; FP64 state */

#define RADM2_SCHED_STATIC 0     /* one thread per cell, cells in order (plain) */
#define RADM2_SCHED_PERSISTENT 1 /* persistent grid, per-lane work stealing */
#define RADM2_SCHED_COOP 2       /* cooperative: 32 cells per block with the whole working set
                                    (LU, state, stage vectors) on chip; the block's warps split
                                    every phase of a step between them, so each cell is served
                                    by one lane in each warp; block_threads 128 (4 warps per cell
                                    group) or 256 (8, default); FP64; cells from a work queue */

typedef struct radm2_opts {
    int device;         /* CUDA device ordinal (default 0) */
    int precision;      /* RADM2_PREC_* (default FP64) */
    int refine_sweeps;  /* FP32LU: FP64 refinement sweeps per stage solve, 0..2 (default 1) */
    int schedule;       /* RADM2_SCHED_* (default STATIC) */
    int block_threads;  /* threads per block: 0 = default (128; 256 for RADM2_SCHED_COOP);
                           32, 64, 128 or 256 (the built variants) */
    int blocks_per_sm;  /* persistent grid blocks per SM: 0 = default */
    int float_coeffs;   /* 1 (default): M/E rounded through float as mgpu.cu:3300-3304 */
    int placement;      /* working-set placement: RADM2_PLACE_* (default GLOBAL) */
    int min_blocks;     /* register cap for occupancy: build variant with at least this many
                           resident blocks per SM (0/1 = no cap; 3 or 4 with 128 threads) */
    int parity;         /* 1: reference-arithmetic FP64 solver -- the pivot divisions of
                           dev_KppDecomp / dev_KppSolve (mgpu.cu:2766, 3086-3090) kept as
                           divisions and no multiply-add contraction anywhere in the step, so
                           every operation rounds as the reference's C expressions do
                           (FP64 only; global placement; default 0 = the fast solver, which
                           multiplies by reciprocal pivots and contracts multiply-adds) */
    int cells_per_thread; /* 1 (default) or 2: with 2, every thread of the thread-per-cell
                           solver integrates two cells side by side (FP64, global placement,
                           64 or 128 threads per block, static or persistent schedule) */
} radm2_opts;

/* Placement of each thread's working set (rate constants + state, and the LU). */
#define RADM2_PLACE_GLOBAL 0   /* all in the thread's global scratch slot */
#define RADM2_PLACE_LU_SMEM 1  /* LU in shared memory (32 or 64 threads per block) */
#define RADM2_PLACE_ALL_SMEM 3 /* LU, rate constants and state in shared memory (32 threads) */
#define RADM2_PLACE_LU_TMEM 4  /* the 128 most used LU slots in tensor memory, the rest global
                                  (FP64, 128 or 256 threads per block; with parity, 256) */
#define RADM2_PLACE_LU_TMEM_WIDE 10 /* the 256 most used LU slots in tensor memory, rate constants
                                       and state in shared memory, the rest global: one CTA of 128
                                       threads per SM owns all 512 columns (FP64, persistent;
                                       fast or reference arithmetic) */

typedef struct radm2_ctx radm2_ctx;

/* Aggregates of the last integration (also folded into IPAR/RPAR). */
typedef struct radm2_stats {
    long long n_accepted;  /* accepted steps, summed over cells */
    long long n_rejected;  /* rejected steps, summed over cells */
    long long n_failed;    /* cells that ended with a negative status */
    int worst_status;      /* minimum per-cell status (1 = all ok) */
    int max_steps_cell;    /* largest per-cell accepted+rejected count */
    double texit_min;      /* least advanced exit time */
    double hexit_min;      /* smallest step proposed at exit */
} radm2_stats;

/* Fill opts with the defaults above. */
int radm2_opts_default(radm2_opts *opts);

/* Create a context on opts->device (opts may be NULL for defaults). */
int radm2_create(radm2_ctx **ctx, const radm2_opts *opts);
int radm2_destroy(radm2_ctx *ctx);

/* Human-readable text for an IERR (-1..-8, the messages of ros_ErrorMsg,
 * mgpu.cu:976-1005) or a RADM2_E* code. */
const char *radm2_error_string(int code);
/* Text of the last CUDA/API failure on this context. */
const char *radm2_last_error(const radm2_ctx *ctx);

/* Use the caller's cudaStream_t for all work of this context (NULL = the context's own). */
int radm2_set_stream(radm2_ctx *ctx, void *cuda_stream);
int radm2_synchronize(radm2_ctx *ctx);

/*
 * Per-cell inputs, host pointers, reference layout.  Replaces the device arrays
 * dev_convert writes (mgpu.cu:513-646): VAR[ncell][59] species (molec/cm^3),
 * FIX[ncell][2] = {H2O, M}, TEMP[ncell] (K), RC_N2O5[ncell] (N2O5 + H2O rate; NULL
 * = zero, which is what mgpu.cu:552's formula evaluates to), JV[ncell][28]
 * photolysis rates (1/s).  Copies to the device (stream-ordered; host buffers
 * may be reused once the call returns).
 */
int radm2_set_inputs(radm2_ctx *ctx, int ncell, const double *VAR, const double *FIX, const double *TEMP,
                     const double *RC_N2O5, const double *JV);

/* Species state only (VAR[ncell][59]); the cell count must match set_inputs. */
int radm2_set_state(radm2_ctx *ctx, const double *VAR);
int radm2_get_state(radm2_ctx *ctx, double *VAR);
/* Copy the current per-cell inputs back to host arrays in the reference layout (any
 * pointer may be NULL to skip that array). */
int radm2_get_inputs(radm2_ctx *ctx, double *VAR, double *FIX, double *TEMP, double *RC_N2O5, double *JV);

/* Same inputs, already in device memory in struct-of-arrays layout:
 * var[59][ld], fix[2][ld], temp[ld], rc_n2o5[ld] (NULL = zero), jv[28][ld], with
 * ld >= ncell the leading dimension.  Device-to-device copy. */
int radm2_set_inputs_device(radm2_ctx *ctx, int ncell, int ld, const double *var, const double *fix,
                            const double *temp, const double *rc_n2o5, const double *jv);
int radm2_get_state_device(radm2_ctx *ctx, double *var, int ld);
/* Species state only, from device memory var[59][ld] (device-to-device). */
int radm2_set_state_device(radm2_ctx *ctx, const double *var, int ld);

/* Rate constants for every cell, replaces updatingCoefficientWRFChemData()
 * (mgpu.cu:921-947; kernel dev_Update_RCONST, mgpu.cu:752-919). */
int radm2_update_rconst(radm2_ctx *ctx);
/* Copy the rate constants out, RCONST[ncell][156] (host). */
int radm2_get_rconst(radm2_ctx *ctx, double *RCONST);
/* Override the rate constants with caller values, RCONST[ncell][156] (host). */
int radm2_set_rconst(radm2_ctx *ctx, const double *RCONST);

/*
 * Integrate every cell from Tstart to Tend.  Replaces Rosenbrock() (mgpu.cu:3664-3848):
 * same IPAR/RPAR meaning and validation (IPAR[0] autonomous, IPAR[1] scalar tol,
 * IPAR[2] max steps, IPAR[3]=2 ROS-3; RPAR[0..6] Hmin, Hmax, Hstart, FacMin, FacMax,
 * FacRej, FacSafe), same return codes.  Counters are accumulated into IPAR[10..16]
 * (Nfun, Njac, Nstp, Nacc, Nrej, Ndec, Nsol), summed over cells; each slot saturates at
 * INT_MAX instead of wrapping (large batches exceed the int range: radm2_get_stats has
 * the exact 64-bit totals); IPAR[17] (Nsng) is left as passed in.
 * RPAR[10] = Texit of the least advanced cell, RPAR[11] = smallest exit step.
 * Each cell runs its own step-size loop on the device; the call blocks until done.
 */
int radm2_rosenbrock(radm2_ctx *ctx, double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                     double *RPAR, int *IPAR);

/* Operator-split loop: nsplit back-to-back integrations of [0, dt], the state
 * carried over, replayed as one CUDA graph when use_graph != 0.  IPAR/RPAR as
 * for radm2_rosenbrock (RPAR[2] = 0 means Hstart = 0.01*dt, the reference
 * driver's ratio, mgpu.cu:3873).  Returns IERR of the worst split. */
int radm2_run_split(radm2_ctx *ctx, int nsplit, double dt, const double *AbsTol, const double *RelTol,
                    double *RPAR, int *IPAR, int use_graph);

/* Per-cell outcome of the last integration (any pointer may be NULL):
 * status (1 ok, -6 step cap, -7 step too small, -8 singular), accepted and
 * rejected step counts, first accepted step size and exit step size. */
int radm2_get_cell_stats(radm2_ctx *ctx, int *status, int *nacc, int *nrej, double *hfirst, double *hexit);
int radm2_get_stats(radm2_ctx *ctx, radm2_stats *out);
/* The IPAR statistics update every integration applies (the counter block of
 * mgpu.cu:3835-3845): IPAR[10..16] += Nfun, Njac, Nstp, Nacc, Nrej, Ndec, Nsol of an
 * integration with these 64-bit totals (Njac = accepted + failed cells' outer steps, Nfun
 * adds one more per outer step when non-autonomous, Nsol = 3 per attempt), each slot
 * saturating at INT_MAX.  Host only (no device needed), for callers that merge shards'
 * totals into one IPAR. */
int radm2_add_step_counters(int *IPAR, long long n_accepted, long long n_rejected, long long n_failed,
                            int autonomous);

/* Per-cell starting step override (device order = cell order), NULL clears it.
 * Values outside (0, Hmax] or non-finite fall back to the default Hstart. */
int radm2_set_cell_hstart(radm2_ctx *ctx, const double *h0);
/* Cell visiting order for the persistent schedule (a permutation of 0..ncell-1),
 * NULL restores natural order. */
int radm2_set_cell_order(radm2_ctx *ctx, const int *order);

/*
 * Batched mechanism kernels on caller arrays (host pointers, per-cell layout), the
 * counterparts of the reference's Fun(), Jac(), Decomp() and Solve() host wrappers
 * (mgpu.cu:1391-1424, 2654-2683, 2849-2852, 3123-3126):
 *   radm2_fun          VDOT[n][59] = F(V)        with FIX[n][2], RCT[n][156]
 *   radm2_jac          JVS[n][659] = J(V)        in LU slot order
 *   radm2_decomp_solve G[n][659] factored in place (pivot-free, fixed pattern) and
 *                      X[n][59] overwritten with G^-1 X; sing[n] = zero-pivot row + 1
 *                      or 0.  precision RADM2_PREC_FP32LU factors in float.
 * They allocate temporary device buffers per call (not for hot loops).
 */
int radm2_fun(radm2_ctx *ctx, int n, const double *V, const double *FIX, const double *RCT, double *VDOT);
int radm2_jac(radm2_ctx *ctx, int n, const double *V, const double *FIX, const double *RCT, double *JVS);
int radm2_decomp_solve(radm2_ctx *ctx, int n, int precision, double *G, double *X, int *sing);

/* Solver-kernel timing: when enabled, CUDA events bracket every solver-kernel launch
 * on the context's stream (graph replays included).  radm2_get_kernel_time returns
 * the summed device time (ms) and launch count since the previous call. */
int radm2_set_kernel_timing(radm2_ctx *ctx, int enable);
int radm2_get_kernel_time(radm2_ctx *ctx, double *ms, int *launches);
/* Kernels one replay of the context's cached split graph launches (counted from the
 * captured graph's kernel nodes; 0 when no graph is cached).  Every one is this library's
 * own kernel.  No counterpart in the reference. */
int radm2_get_graph_kernels(const radm2_ctx *ctx, int *kernels);

/* Measured CUDA-core FMA throughput of a device (TFLOP/s, 2 flops per FMA): the
 * denominators of the solver's roofline.  Runs ~0.2 s of microbenchmark. */
int radm2_fma_peak(int device, double *fp64_tflops, double *fp32_tflops);

/* Number of cells and device bytes held by the context. */
int radm2_get_ncell(const radm2_ctx *ctx);
size_t radm2_device_bytes(const radm2_ctx *ctx);

/* One integration straight from host arrays in the reference's per-cell layout -- the
 * whole radm2_set_inputs + radm2_rosenbrock + radm2_get_state sequence (mgpu.cu:648-680,
 * 921-947, 3664-3848) in one call -- with the transfers overlapped with the solve: the
 * batch is cut into nchunk consecutive chunks (at least 1,024 cells each), chunk k's
 * inputs upload while chunk k-1 integrates and chunk k-2's states download.  VAR is read
 * and overwritten with the result; RC_N2O5 may be NULL (zero, as for radm2_set_inputs).  Rate
 * constants and, with a network attached, the seeded starting steps are formed per chunk;
 * a cost order is not applied.  Host arrays should be page-locked (cudaHostRegister /
 * cudaMallocHost): pageable memory is correct but serialises the copies.  Returns IERR and
 * fills IPAR/RPAR as radm2_rosenbrock. */
int radm2_rosenbrock_host(radm2_ctx *ctx, int ncell, double *VAR, const double *FIX, const double *TEMP,
                          const double *RC_N2O5, const double *JV, double Tstart, double Tend, const double *AbsTol,
                          const double *RelTol, double *RPAR, int *IPAR, int nchunk);

/* WRF -> KPP conversion, replacing dev_convert + convertWRFChemData (mgpu.cu:513-706).
 * WRF fields are field-major with i fastest, field[f][nj][nk][ni]; the window
 * [i0, i0+wi) x [k0, k0+wk) x [j0, j0+wj) becomes the context's cells, cell
 * p = (j'*wk + k')*wi + i' (the reference launch order).  Fields read: ph 0..27 (J per
 * minute), chem and rad (the species map of mgpu.cu:586-644, chem 0..43, rad 0..27),
 * phy 0 pressure (Pa), 1 temperature (K), 2 air density (kg/m3), moist 1 water vapour
 * (kg/kg).  Sets VAR (ppmV -> molec/cm3, negatives clamped to 0), FIX {H2O, M}, TEMP,
 * RC_N2O5 (per cell) and JV (per second); the rate constants are recomputed on the next
 * integration.  radm2_wrf_grid_default gives the reference's 48 x 20 x 48 domain with its
 * 39 x 19 x 39 window (28,899 cells). */
typedef struct radm2_wrf_grid {
    int ni, nk, nj; /* field dimensions */
    int i0, k0, j0; /* window origin */
    int wi, wk, wj; /* window extent */
} radm2_wrf_grid;
int radm2_wrf_grid_default(radm2_wrf_grid *grid);
int radm2_convert_wrf(radm2_ctx *ctx, const radm2_wrf_grid *grid, const double *ph, const double *chem,
                      const double *rad, const double *phy, const double *moist);        /* host fields */
int radm2_convert_wrf_device(radm2_ctx *ctx, const radm2_wrf_grid *grid, const double *ph, const double *chem,
                             const double *rad, const double *phy, const double *moist); /* device fields */
int radm2_get_opts(const radm2_ctx *ctx, radm2_opts *out);  /* options in force (after autotune) */

/* Autotuner (no counterpart in the reference, which has one fixed launch shape).  Times
 * every built solver variant of the context's precision -- static and persistent
 * schedules x block size x placement of the working set (global scratch / shared memory)
 * x register cap, two cells per thread, and the cooperative blocks of 4 or 8 warps per 32
 * cells (FP64) -- on a strided sample of the context's current cells (sample_cells;
 * 0 = 262,144) for one split of length dt with the given tolerances and parameters, and
 * keeps the fastest in the context's options (radm2_get_opts reads them).  Candidates
 * within 2x of the best first-pass time are timed a second time and keep the faster of
 * their two times, so a one-off slow measurement does not decide the choice.  The context's
 * cells and state are not changed.  table (may be NULL) receives up to table_len
 * entries, n_entries the number of candidates. */
typedef struct radm2_tune_entry {
    int schedule, block_threads, placement, min_blocks; /* the candidate */
    double ms;                                          /* solver-kernel time, -1 = did not run */
    long long attempts;                                 /* step attempts of the sample split */
    int cells_per_thread;                               /* 1 or 2 */
} radm2_tune_entry;
int radm2_autotune(radm2_ctx *ctx, double dt, const double *AbsTol, const double *RelTol, const double *RPAR,
                   const int *IPAR, int sample_cells, radm2_tune_entry *table, int table_len, int *n_entries);

/*
 * Learned step seeding.  A small network (84 state features -> 3 x 128 GELU -> 2, BF16
 * weights on the tensor cores with FP32 accumulation, FP32 master weights, Adam) predicts
 * each cell's starting step h0 and accepted-step count from its state.  The predictions
 * seed radm2_set_cell_hstart-style starting steps (the Rosenbrock error controller still
 * accepts or rejects every step; non-finite or out-of-range predictions fall back to the
 * default Hstart) and a descending-cost visiting order for the persistent schedule.
 * Features per cell: log10 of the 59 species (floor 1e-3), T, log10 M, log10 H2O,
 * log10(J_k + 1e-12) for the 21 photolysis rates in use, and dt.  Outputs are
 * standardised log10 h0 and log10(accepted steps + 1).
 */
typedef struct radm2_mlp radm2_mlp;
int radm2_mlp_nparams(void);
int radm2_mlp_create(radm2_mlp **mlp, int device, unsigned int seed);
int radm2_mlp_destroy(radm2_mlp *mlp);
int radm2_mlp_set_params(radm2_mlp *mlp, const float *params);   /* host, radm2_mlp_nparams() floats */
int radm2_mlp_get_params(radm2_mlp *mlp, float *params);
/* Feature (84) and output (2) standardisation. */
int radm2_mlp_set_norm(radm2_mlp *mlp, const float *xmean, const float *xstd, const float *ymean, const float *ystd);
/* Standardised outputs y[n][2] for features x[n][84] (host arrays). */
int radm2_mlp_forward(radm2_mlp *mlp, int n, const float *x, float *y);
/* Gradient of the mean squared error over n samples (host arrays), without an update. */
int radm2_mlp_gradients(radm2_mlp *mlp, int n, const float *x, const float *target, float *grad, float *loss);
/* One Adam step on a batch in device memory: x[n][84], target[n][2] (standardised). */
int radm2_mlp_train_step(radm2_mlp *mlp, int n, const float *x, const float *target, float lr, float *loss);
int radm2_mlp_synchronize(radm2_mlp *mlp);
/* Safety factor on seeded starting steps: h0 = scale * predicted step (default 1). */
int radm2_mlp_set_h0_scale(radm2_mlp *mlp, float scale);
/* Inference forward (radm2_mlp_forward and the seeding of attached contexts) on the
 * tcgen05 tensor cores with the accumulator in tensor memory (tcgen05 != 0, the default)
 * or on mma.sync tiles (0).  Training always uses the mma.sync kernels, which keep the
 * pre-activations for the backward pass.  No counterpart in the reference (its solver
 * has no learned seeding). */
int radm2_mlp_set_tensor_path(radm2_mlp *mlp, int tcgen05);
/* RADM2_OK, or RADM2_E_CUDA once a tcgen05 forward gave up waiting on its tensor-core
 * work (its predictions are then not to be used; the flag stays set).  Read it after the
 * work has completed: radm2_mlp_forward checks it itself; for attached contexts call it
 * after the integration returned. */
int radm2_mlp_status(radm2_mlp *mlp);
/* Self-test of the tcgen05 forward's bounded waits: one launch that issues no tensor-core
 * work, so its mbarrier waits run out after a short limit.  RADM2_OK when the kernel
 * returned and raised the status flag (cleared again before returning), RADM2_E_STATE if
 * it did not raise it.  The network stays usable.  No counterpart in the reference. */
int radm2_mlp_selftest_wait_limit(radm2_mlp *mlp);
/* Features of the context's current cell states, host out[ncell][84]. */
int radm2_get_features(radm2_ctx *ctx, double dt, float *out);
/* Seed the context from the network: per-cell starting steps (set_h0) and, for the
 * persistent schedule, the cell order (set_order: 0 none, 1 cells by descending
 * predicted cost, 2 chunks of 32 consecutive cells by their costliest cell, which keeps
 * each warp's loads coalesced). */
int radm2_seed_cells(radm2_ctx *ctx, radm2_mlp *mlp, double dt, int set_h0, int set_order);
/* Attach a network to the context (NULL detaches): every following integration --
 * radm2_rosenbrock and each split of radm2_run_split -- is seeded from the current
 * state on the device first, inside the same CUDA graph for radm2_run_split.
 * set_order as for radm2_seed_cells. */
int radm2_attach_mlp(radm2_ctx *ctx, radm2_mlp *mlp, int set_order);

/* Self-test of the cooperative kernel's bounded waits (a context with schedule
 * RADM2_SCHED_COOP and cells set): one integration in which a warp of every block waits on
 * a flag that nothing sets, with a short limit (~1 ms).  The wait must run out, the blocks
 * must return and the integration must report RADM2_E_CUDA.  RADM2_OK when it did,
 * RADM2_E_STATE if not.  The cells' states are not changed; the context stays usable.  No
 * counterpart in the reference. */
int radm2_coop_selftest_wait_limit(radm2_ctx *ctx);

/* Host-only consistency check of the library's kernel layouts (every thread's
 * working-set offsets inside its allocation, for every built variant). */
int radm2_selfcheck(void);

/*
 * Integration without any device allocation, for callers that may not call cudaMalloc
 * while they run: host frameworks that reserved all of the GPU's memory for their own pool
 * at start-up (a later cudaMalloc fails or takes memory the pool counts on), and real-time
 * or certified model couplings whose device memory budget is fixed at initialisation.  No
 * counterpart in the reference (which allocates inside Rosenbrock(), mgpu.cu:3444-3468).
 *
 * Same method, IPAR/RPAR meaning and return codes as radm2_rosenbrock, but without a
 * context: inputs and outputs are the caller's device arrays in struct-of-arrays layout
 * with leading dimension ld (var[59][ld] species in/out, fix[2][ld], temp[ld],
 * rc_n2o5[ld] or NULL, jv[28][ld]), on the current device and the given cudaStream_t
 * (NULL = default stream); status[ncell] (device, or NULL) receives each cell's outcome.
 * Everything else -- rate constants, the solver's scratch, per-cell bookkeeping -- lives
 * in one statically sized device array of RADM2_NOALLOC_BYTES (64 MiB) that every GPU
 * which loads the library holds until the process exits.  Limits: ncell <= ld <=
 * RADM2_NOALLOC_MAX_CELLS; larger sizes return RADM2_E_TOOBIG (split the batch).
 * Set-up: the first call on a device (and CUDA context) looks up the array's device
 * address and loads the library's device code there.  All calls share the array, which
 * keeps the previous call's contents (the call clears what must start at zero), so calls
 * that overlap on the GPU (other streams, other host threads) race: serialise them.  The
 * call waits for its stream before returning, as it reads the statistics back into
 * IPAR/RPAR.  It calls no allocating routine.
 */
#define RADM2_NOALLOC_MAX_CELLS 32768
#define RADM2_NOALLOC_BYTES (64u << 20)
int radm2_rosenbrock_noalloc(int ncell, int ld, double *var, const double *fix, const double *temp,
                             const double *rc_n2o5, const double *jv, double Tstart, double Tend,
                             const double *AbsTol, const double *RelTol, double *RPAR, int *IPAR, int *status,
                             void *stream);

/* Library build string (arch, variants). */
const char *radm2_version(void);

#ifdef __cplusplus
}
#endif
#endif
