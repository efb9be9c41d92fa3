/*
 * CPU oracle for the batched RADM2 Rosenbrock (ROS-3) solve.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker, never the product: only the
 * test-suite, the smoke check and the CPU-baseline leg of the benchmark load it.
 * The product path is the CUDA library and fails loudly without it.
 *
 * It restates, per grid cell and in plain C (FP64), the reference's path:
 *   rate constants   mgpu.cu:708-919   (rk_* below, orc_rconst generated)
 *   RHS              mgpu.cu:1084-1386 (orc_fun, generated)
 *   sparse Jacobian  mgpu.cu:1672-2652 (orc_jac, generated)
 *   prepare          mgpu.cu:3128-3166, 2685-2703 (G = -J + I/(Dir*h*gamma1))
 *   LU               mgpu.cu:2726-2780 (orc_decomp, table driven)
 *   solve            mgpu.cu:2854-3096 (orc_solve, table driven)
 *   stages           mgpu.cu:3595-3625 (commented out in the reference; restored
 *                                       with KPP's Rosenbrock semantics)
 *   step control     mgpu.cu:3168-3262, time loop mgpu.cu:1595-1614
 *   driver params    mgpu.cu:3664-3848 (orc_rosenbrock: IPAR/RPAR parsing, codes)
 *   WRF -> KPP       mgpu.cu:513-646   (orc_convert_wrf, tables generated)
 *
 * The mechanism functions are pinned bit-for-bit against the reference's own
 * dev_Update_RCONST / dev_Fun / dev_Jac_SP / dev_KppDecomp / dev_KppSolve,
 * compiled for the CPU from mgpu.cu by oracle/build_ref.py.
 */
#ifndef RADM2_ORACLE_H
#define RADM2_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_NVAR 59
#define ORC_NFIX 2
#define ORC_NREACT 156
#define ORC_NJVS 659
#define ORC_NPH 28

extern const int orc_lu_crow[ORC_NVAR + 1];
extern const int orc_lu_diag[ORC_NVAR];
extern const int orc_lu_icol[ORC_NJVS];

/* Integration parameters after IPAR/RPAR parsing (mgpu.cu:3684-3800). */
typedef struct {
    double Tstart, Tend;
    double AbsTol[ORC_NVAR], RelTol[ORC_NVAR];
    double Hmin, Hmax, Hstart;
    double FacMin, FacMax, FacRej, FacSafe;
    double Roundoff;
    int max_steps;      /* per-cell bound on step attempts (IPAR[2]); 0 = unbounded */
    int autonomous;     /* IPAR[0] != 0 */
    int float_coeffs;   /* 1: M/E rounded through float as mgpu.cu:3300-3304 does */
} orc_params;

/* Per-cell outcome.  status: 1 ok, -6 step cap, -7 step too small, -8 singular. */
typedef struct {
    int status;
    int nacc, nrej;
    double texit;       /* time reached */
    double hexit;       /* step size proposed after the last accepted step */
    double hfirst;      /* size of the first accepted step */
} orc_cell_stats;

/* Rate-law helpers (mgpu.cu:708-750). */
double rk_arr2(double a0, double b0, double temp);
double rk_troe(double k0_300, double n, double kinf_300, double m, double temp, double cair);
double rk_troee(double a, double b, double k0_300, double n, double kinf_300, double m,
                double temp, double cair);
double rk_thermal_t2(double c, double d, double temp);
double rk_k46(double cair, double temp);

/* Generated mechanism functions (oracle/gen/radm2_oracle_gen.c). */
void orc_rconst(const double *jv, double TEMP, double C_M, double rc_n2o5, double *RCT);
void orc_fun(const double *V, const double *F, const double *RCT, double *Vdot);
void orc_jac(const double *V, const double *F, const double *RCT, double *JVS);

/* Table-driven LU (returns 0 or the 1-based row of a zero pivot) and solve. */
int orc_decomp(double *JVS);
void orc_solve(const double *JVS, double *X);

/* Unit roundoff as computed by mgpu.cu:949-973. */
double orc_wlamch(void);

/* One cell: integrate Y[59] in place from Tstart to Tend. */
int orc_integrate_cell(double *Y, const double *FIX, const double *RCT, const orc_params *p,
                       orc_cell_stats *st);

/* Batch over cells with OpenMP (nthreads <= 0: OpenMP default).  Arrays are in the
 * reference's per-cell (AoS) layout: VAR[ncell][59], FIX[ncell][2], RCT[ncell][156]. */
void orc_integrate_batch(int ncell, double *VAR, const double *FIX, const double *RCT,
                         const orc_params *p, orc_cell_stats *stats, int nthreads);

/* Rate constants for a batch: JV[ncell][28], TEMP[ncell], FIX[ncell][2], RC_N2O5[ncell]. */
void orc_rconst_batch(int ncell, const double *JV, const double *TEMP, const double *FIX,
                      const double *RC_N2O5, double *RCT, int nthreads);

/* Mirror of Rosenbrock() (mgpu.cu:3664-3848): parses IPAR/RPAR with the same checks
 * and error codes (-1..-5), integrates every cell, accumulates IPAR[10..17] and
 * writes RPAR[10]=Texit, RPAR[11]=Hexit.  Returns 1 or the most negative cell code.
 * float_coeffs selects the reference's float-rounded M/E. */
int orc_rosenbrock(double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                   double *RPAR, int *IPAR, int ncell, double *VAR, const double *FIX,
                   const double *RCT, int float_coeffs, orc_cell_stats *stats, int nthreads);

/* Parameter parsing only (returns 1 or a negative code). */
int orc_parse_params(double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                     const double *RPAR, const int *IPAR, int float_coeffs, orc_params *p);

/* WRF -> KPP conversion (mgpu.cu:513-646).  WRF fields are field-major with i fastest,
 * field[f][nj][nk][ni]; the window [i0, i0+wi) x [k0, k0+wk) x [j0, j0+wj) becomes cells
 * p = (j'*wk + k')*wi + i' (the order of the reference's launch, mgpu.cu:682-706).
 * Fields read: ph 0..27 (J per minute), chem and rad (orc_wrf_var_src), phy 0 pressure
 * (Pa), 1 temperature (K), 2 air density (kg/m3), moist 1 water vapour (kg/kg).
 * Outputs in the per-cell layout: VAR[p][59], FIX[p][2] = {H2O, M}, TEMP[p], RC_N2O5[p],
 * JV[p][28].  TEMP and RC_N2O5 are per cell (the reference writes element 0 for every
 * cell, mgpu.cu:545, 552: a defect, not the intent). */
typedef struct orc_wrf_grid {
    int ni, nk, nj;
    int i0, k0, j0;
    int wi, wk, wj;
} orc_wrf_grid;
extern const int orc_wrf_var_src[ORC_NVAR][2];
extern const int orc_wrf_jv_src[ORC_NPH];
void orc_convert_wrf(const orc_wrf_grid *g, const double *ph, const double *chem, const double *rad,
                     const double *phy, const double *moist, double *VAR, double *FIX, double *TEMP,
                     double *RC_N2O5, double *JV);

#ifdef __cplusplus
}
#endif
#endif
