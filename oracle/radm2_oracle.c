/*
 * CPU oracle for the batched RADM2 ROS-3 solve -- TEST INFRASTRUCTURE ONLY.
 * See radm2_oracle.h for what is restated from where.  Compiled with
 * -ffp-contract=off so every expression rounds exactly as written.
 */
#include "radm2_oracle.h"

#include <math.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ZERO 0.0
#define ONE 1.0
#define DELTA_MIN 1.0e-6

/* The reference's comparison macros (mgpu.cu:191-195): ternaries, kept as such. */
#define MAXD(a, b) (((a) >= (b)) ? (a) : (b))
#define MIND(b, c) (((b) < (c)) ? (b) : (c))
#define ABSD(x) (((x) >= 0) ? (x) : (-(x)))

/* ROS-3 method (mgpu.cu:1007-1062). */
static const double ros_A[3] = {1.0, 1.0, 0.0};
static const double ros_C[3] = {-1.0156171083877702091975600115545, 4.0759956452537699824805835358067,
                                9.2076794298330791242156818474003};
static const double ros_M[3] = {1.0, 6.1697947043828245592553615689730, -0.4277225654321857332623837380651};
static const double ros_E[3] = {0.5, -2.9079558716805469821718236208017, 0.2235406989781156962736090927619};
static const double ros_Gamma[3] = {0.43586652150845899941601945119356, 0.24291996454816804366592249683314,
                                    2.1851380027664058511513169485832};
static const int ros_NewF[3] = {1, 1, 0};
static const double ros_ELO = 3.0;

/* ---------------------------------------------------------------- rate laws (mgpu.cu:708-750) */

/* Arrhenius k = A0 exp(-B0/T). */
double rk_arr2(double a0, double b0, double temp) { return a0 * exp(-b0 / temp); }

/* Troe fall-off (Stockwell et al. 1997), broadening factor 0.6. */
double rk_troe(double k0_300, double n, double kinf_300, double m, double temp, double cair)
{
    double zt = 300.0 / temp;
    double k0 = k0_300 * pow(zt, n) * cair;
    double kinf = kinf_300 * pow(zt, m);
    double ratio = k0 / kinf;
    return k0 / (1.0 + ratio) * pow(0.6, 1.0 / (1.0 + pow(log10(ratio), 2.0)));
}

/* Troe equilibrium: A exp(-B/T) times the fall-off rate. */
double rk_troee(double a, double b, double k0_300, double n, double kinf_300, double m,
                double temp, double cair)
{
    double zt = 300.0 / temp;
    double k0 = k0_300 * pow(zt, n) * cair;
    double kinf = kinf_300 * pow(zt, m);
    double ratio = k0 / kinf;
    double troe = k0 / (1.0 + ratio) * pow(0.6, 1.0 / (1.0 + pow(log10(ratio), 2.0)));
    return a * exp(-b / temp) * troe;
}

/* k = T^2 c exp(-d/T). */
double rk_thermal_t2(double c, double d, double temp) { return pow(temp, 2.0) * c * exp(-d / temp); }

/* HNO3 + OH, pressure dependent. */
double rk_k46(double cair, double temp)
{
    double k0 = 7.2e-15 * exp(785.0 / temp);
    double k2 = 4.1e-16 * exp(1440.0 / temp);
    double k3 = 1.9e-33 * exp(725.0 / temp) * cair;
    return k0 + k3 / (1.0 + k3 / k2);
}

/* ---------------------------------------------------------------- LU and solve */

/* Row-by-row pivot-free LU on the fixed pattern, mgpu.cu:2746-2779.  The zero-pivot
 * check looks at row k's diagonal before that row is eliminated, as the reference does. */
int orc_decomp(double *JVS)
{
    double W[ORC_NVAR];
    for (int k = 0; k < ORC_NVAR; k++) {
        if (JVS[orc_lu_diag[k]] == 0.0) return k + 1;
        for (int kk = orc_lu_crow[k]; kk < orc_lu_crow[k + 1]; kk++) W[orc_lu_icol[kk]] = JVS[kk];
        for (int kk = orc_lu_crow[k]; kk < orc_lu_diag[k]; kk++) {
            int j = orc_lu_icol[kk];
            double a = -W[j] / JVS[orc_lu_diag[j]];
            W[j] = -a;
            for (int jj = orc_lu_diag[j] + 1; jj < orc_lu_crow[j + 1]; jj++) W[orc_lu_icol[jj]] += a * JVS[jj];
        }
        for (int kk = orc_lu_crow[k]; kk < orc_lu_crow[k + 1]; kk++) JVS[kk] = W[orc_lu_icol[kk]];
    }
    return 0;
}

/* Forward (unit lower) then backward (upper / diagonal) substitution, summing each
 * row left to right as the unrolled mgpu.cu:2873-3090 expressions do. */
void orc_solve(const double *JVS, double *X)
{
    for (int k = 0; k < ORC_NVAR; k++) {
        double x = X[k];
        for (int s = orc_lu_crow[k]; s < orc_lu_diag[k]; s++) x = x - JVS[s] * X[orc_lu_icol[s]];
        X[k] = x;
    }
    for (int k = ORC_NVAR - 1; k >= 0; k--) {
        double x = X[k];
        for (int s = orc_lu_diag[k] + 1; s < orc_lu_crow[k + 1]; s++) x = x - JVS[s] * X[orc_lu_icol[s]];
        X[k] = x / JVS[orc_lu_diag[k]];
    }
}

/* Unit roundoff by halving until 1 + eps == 1 (mgpu.cu:949-973); gives 2^-52. */
double orc_wlamch(void)
{
    double eps = pow(0.5, 16);
    int i;
    for (i = 17; i <= 80; i++) {
        eps = eps * 0.5;
        volatile double suma = 1.0 + eps;
        if (suma <= 1.0) break;
    }
    if (i == 80) return 2.2e-16;
    return eps * 2.0;
}

/* ---------------------------------------------------------------- one cell */

int orc_integrate_cell(double *Y, const double *FIX, const double *RCT, const orc_params *p,
                       orc_cell_stats *st)
{
    double F0[ORC_NVAR], F[ORC_NVAR], K[3][ORC_NVAR], Ynew[ORC_NVAR], dFdT[ORC_NVAR];
    double J[ORC_NJVS], G[ORC_NJVS];
    double M[3], E[3];
    for (int i = 0; i < 3; i++) {
        /* mgpu.cu:3300-3304 uploads M and E through a float array. */
        M[i] = p->float_coeffs ? (double)(float)ros_M[i] : ros_M[i];
        E[i] = p->float_coeffs ? (double)(float)ros_E[i] : ros_E[i];
    }
    const double Roundoff = p->Roundoff;
    const double Tend = p->Tend;
    double T = p->Tstart;
    double H = MIND(p->Hstart, p->Hmax); /* mgpu.cu:3475-3477 */
    if (ABSD(H) <= 10.0 * Roundoff) H = DELTA_MIN;
    const int Direction = (Tend >= p->Tstart) ? +1 : -1;
    int RejectLastH = 0, RejectMoreH = 0;
    int nstp = 0;
    st->status = 1;
    st->nacc = st->nrej = 0;
    st->hfirst = 0.0;

    /* Outer loop: mgpu.cu:1608-1613 (mask and clamp of H to the remaining interval). */
    while ((Direction > 0 && (T - Tend) + Roundoff <= 0.0) || (Direction < 0 && (Tend - T) + Roundoff <= 0.0)) {
        H = MIND(H, ABSD(Tend - T));
        orc_fun(Y, FIX, RCT, F0);
        if (!p->autonomous) {
            /* ros_FunTimeDerivative (mgpu.cu:1566-1593): this mechanism's RHS has no explicit
             * time dependence, so the finite difference is exactly zero; kept literal here. */
            double Delta = pow(Roundoff, 0.5) * MAXD(DELTA_MIN, ABSD(T));
            orc_fun(Y, FIX, RCT, dFdT);
            for (int i = 0; i < ORC_NVAR; i++) dFdT[i] = dFdT[i] + (-ONE) * F0[i];
            for (int i = 0; i < ORC_NVAR; i++) dFdT[i] = dFdT[i] * (ONE / Delta);
        }
        orc_jac(Y, FIX, RCT, J);

        for (;;) { /* reject loop, mgpu.cu:3584-3642 */
            if (p->max_steps > 0 && nstp >= p->max_steps) {
                st->status = -6;
                goto done;
            }
            if ((T + 0.1 * H == T) || (H <= Roundoff)) {
                st->status = -7;
                goto done;
            }
            /* ros_PrepareMatrix: G = -J, diagonal += 1/(Direction*H*gamma1). */
            const double ghinv = ONE / (Direction * H * ros_Gamma[0]);
            for (int s = 0; s < ORC_NJVS; s++) G[s] = -J[s];
            for (int i = 0; i < ORC_NVAR; i++) G[orc_lu_diag[i]] += ghinv;
            if (orc_decomp(G) != 0) {
                st->status = -8;
                goto done;
            }
            /* Stages (restored KPP semantics of mgpu.cu:3595-3625). */
            for (int istage = 0; istage < 3; istage++) {
                double *Ks = K[istage];
                if (istage == 0) {
                    memcpy(F, F0, sizeof F);
                } else if (ros_NewF[istage]) {
                    memcpy(Ynew, Y, sizeof Ynew);
                    for (int j = 0; j < istage; j++) {
                        const double a = ros_A[istage * (istage - 1) / 2 + j];
                        if (a != 0.0)
                            for (int i = 0; i < ORC_NVAR; i++) Ynew[i] = Ynew[i] + a * K[j][i];
                    }
                    orc_fun(Ynew, FIX, RCT, F);
                }
                memcpy(Ks, F, sizeof F);
                for (int j = 0; j < istage; j++) {
                    const double hc = ros_C[istage * (istage - 1) / 2 + j] / (Direction * H);
                    for (int i = 0; i < ORC_NVAR; i++) Ks[i] = Ks[i] + K[j][i] * hc;
                }
                if (!p->autonomous && ros_Gamma[istage] != 0.0) {
                    const double HG = Direction * H * ros_Gamma[istage];
                    for (int i = 0; i < ORC_NVAR; i++) Ks[i] = Ks[i] + HG * dFdT[i];
                }
                orc_solve(G, Ks);
            }
            nstp++;

            /* acceptStep: mgpu.cu:3223-3260 */
            double Err = 0.0;
            for (int i = 0; i < ORC_NVAR; i++) {
                Ynew[i] = M[0] * K[0][i] + M[1] * K[1][i] + M[2] * K[2][i] + Y[i];
                const double Yerr = E[0] * K[0][i] + E[1] * K[1][i] + E[2] * K[2][i];
                const double Ymax = MAXD(ABSD(Y[i]), ABSD(Ynew[i]));
                const double Scale = p->AbsTol[i] + p->RelTol[i] * Ymax;
                Err += (Yerr * Yerr) / (Scale * Scale);
            }
            Err = sqrt(Err / (double)ORC_NVAR);
            double Fac = MIND(p->FacMax, MAXD(p->FacMin, p->FacSafe / pow(Err, ONE / ros_ELO)));
            double Hnew = H * Fac;
            if (Err != Err) Hnew = H * p->FacRej; /* non-finite norm: shrink hard and retry */
            if ((Err <= ONE) || (H <= p->Hmin)) {
                memcpy(Y, Ynew, sizeof Ynew);
                T += Direction * H;
                if (RejectLastH) Hnew = MIND(Hnew, H);
                RejectLastH = 0;
                RejectMoreH = 0;
                if (st->nacc == 0) st->hfirst = H;
                st->nacc++;
                H = Hnew;
                break;
            } else {
                if (RejectMoreH) Hnew = H * p->FacRej;
                RejectMoreH = RejectLastH;
                RejectLastH = 1;
                st->nrej++;
                H = Hnew;
            }
        }
    }
done:
    st->texit = T;
    st->hexit = H;
    return st->status;
}

void orc_integrate_batch(int ncell, double *VAR, const double *FIX, const double *RCT,
                         const orc_params *p, orc_cell_stats *stats, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 8)
#endif
    for (int c = 0; c < ncell; c++)
        orc_integrate_cell(VAR + (size_t)c * ORC_NVAR, FIX + (size_t)c * ORC_NFIX, RCT + (size_t)c * ORC_NREACT,
                           p, &stats[c]);
}

void orc_rconst_batch(int ncell, const double *JV, const double *TEMP, const double *FIX,
                      const double *RC_N2O5, double *RCT, int nthreads)
{
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(static)
#endif
    for (int c = 0; c < ncell; c++)
        orc_rconst(JV + (size_t)c * ORC_NPH, TEMP[c], FIX[(size_t)c * ORC_NFIX + 1], RC_N2O5[c],
                   RCT + (size_t)c * ORC_NREACT);
}

/* ---------------------------------------------------------------- WRF -> KPP */

/* mgpu.cu:29-44: molecules per mole, molecular weights, density -> concentration. */
#define ORC_NAVGDRO (6.022e23)
#define ORC_MWAIR (28.97)
#define ORC_MWH2O (2 * (1.0079) + (15.9994))
#define ORC_DENS2CON_A (1.0e-3 * (1.0 / ORC_MWAIR) * ORC_NAVGDRO)
#define ORC_DENS2CON_W (1.0e-3 * (1.0 / ORC_MWH2O) * ORC_NAVGDRO)

void orc_convert_wrf(const orc_wrf_grid *g, const double *ph, const double *chem, const double *rad,
                     const double *phy, const double *moist, double *VAR, double *FIX, double *TEMP,
                     double *RC_N2O5, double *JV)
{
    const size_t fs = (size_t)g->nj * g->nk * g->ni; /* one field */
    const int n = g->wi * g->wk * g->wj;
    for (int p = 0; p < n; p++) {
        const int ii = p % g->wi, kk = (p / g->wi) % g->wk, jj = p / (g->wi * g->wk);
        const size_t o = ((size_t)(g->j0 + jj) * g->nk + (g->k0 + kk)) * g->ni + (g->i0 + ii);
        const double pres = phy[o], t = phy[fs + o], rho = phy[2 * fs + o], qv = moist[fs + o];
        double *v = VAR + (size_t)p * ORC_NVAR;
        /* mgpu.cu:539-552 */
        FIX[(size_t)p * ORC_NFIX + 1] = ORC_DENS2CON_A * rho;
        FIX[(size_t)p * ORC_NFIX + 0] = ORC_DENS2CON_W * qv * rho;
        TEMP[p] = t;
        const double es = 1000. * 0.6112 * exp(17.67 * (t - 273.15) / (t - 29.65));
        const double qvs = es / (pres - es);
        double rh = qv / qvs;
        rh = rh >= 0.0f ? rh : 0.0f;
        rh = rh < 1.0f ? rh : 1.0f;
        RC_N2O5[p] = 1.0 / (3.6e4 * exp(-pow((rh / 0.28), 2.8) + 300.0));
        /* mgpu.cu:555-583: ppmV -> molec/cm3, J per minute -> per second */
        const double conv = 1.0E-6 * ORC_DENS2CON_A * rho;
        for (int k = 0; k < ORC_NPH; k++) JV[(size_t)p * ORC_NPH + k] = ph[orc_wrf_jv_src[k] * fs + o] / 60.0;
        /* mgpu.cu:586-644 */
        for (int i = 0; i < ORC_NVAR; i++) {
            const double *src = orc_wrf_var_src[i][0] == 0 ? chem : rad;
            const double x = src[(size_t)orc_wrf_var_src[i][1] * fs + o];
            v[i] = conv * (x >= 0.0 ? x : 0.0);
        }
    }
}

/* ---------------------------------------------------------------- Rosenbrock() mirror */

int orc_parse_params(double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                     const double *RPAR, const int *IPAR, int float_coeffs, orc_params *p)
{
    memset(p, 0, sizeof *p);
    p->Tstart = Tstart;
    p->Tend = Tend;
    p->autonomous = !(IPAR[0] == 0);
    const int vector_tol = (IPAR[1] == 0);
    const int uplim = vector_tol ? ORC_NVAR : 1;
    p->max_steps = (IPAR[2] == 0) ? 100000 : IPAR[2];
    if (p->max_steps < 0) return -1;
    if ((IPAR[3] < 1) || (IPAR[3] > 5)) return -2;
    p->Roundoff = orc_wlamch();
    p->Hmin = RPAR[0];
    if (RPAR[0] < ZERO) return -3;
    p->Hmax = (RPAR[1] == ZERO) ? ABSD(Tend - Tstart) : MIND(ABSD(RPAR[1]), ABSD(Tend - Tstart));
    if (RPAR[1] < ZERO) return -3;
    p->Hstart = (RPAR[2] == ZERO) ? MAXD(p->Hmin, DELTA_MIN) : MIND(ABSD(RPAR[2]), ABSD(Tend - Tstart));
    if (RPAR[2] < ZERO) return -3;
    p->FacMin = (RPAR[3] == ZERO) ? 0.2 : RPAR[3];
    if (RPAR[3] < ZERO) return -4;
    p->FacMax = (RPAR[4] == ZERO) ? 6.0 : RPAR[4];
    if (RPAR[4] < ZERO) return -4;
    p->FacRej = (RPAR[5] == ZERO) ? 0.1 : RPAR[5];
    if (RPAR[5] < ZERO) return -4;
    p->FacSafe = (RPAR[6] == ZERO) ? 0.9 : RPAR[6];
    if (RPAR[6] < ZERO) return -4;
    for (int i = 0; i < uplim; i++)
        if ((AbsTol[i] <= ZERO) || (RelTol[i] <= 10.0 * p->Roundoff) || (RelTol[i] >= ONE)) return -5;
    if (IPAR[3] != 2) return -2; /* only Ros3 is wired (mgpu.cu:3803-3811) */
    for (int i = 0; i < ORC_NVAR; i++) {
        p->AbsTol[i] = vector_tol ? AbsTol[i] : AbsTol[0];
        p->RelTol[i] = vector_tol ? RelTol[i] : RelTol[0];
    }
    p->float_coeffs = float_coeffs;
    return 1;
}

int orc_rosenbrock(double Tstart, double Tend, const double *AbsTol, const double *RelTol,
                   double *RPAR, int *IPAR, int ncell, double *VAR, const double *FIX,
                   const double *RCT, int float_coeffs, orc_cell_stats *stats, int nthreads)
{
    orc_params p;
    int rc = orc_parse_params(Tstart, Tend, AbsTol, RelTol, RPAR, IPAR, float_coeffs, &p);
    if (rc != 1) return rc;
    orc_integrate_batch(ncell, VAR, FIX, RCT, &p, stats, nthreads);
    long nacc = 0, nrej = 0, nouter = 0;
    int ierr = 1;
    double texit = Tend, hexit = 0.0;
    for (int c = 0; c < ncell; c++) {
        nacc += stats[c].nacc;
        nrej += stats[c].nrej;
        nouter += stats[c].nacc + (stats[c].status != 1);
        if (stats[c].status < ierr) ierr = stats[c].status;
        /* Texit: the least advanced cell (Tend when every cell finished). */
        if (c == 0 || (Tend >= Tstart ? stats[c].texit < texit : stats[c].texit > texit)) texit = stats[c].texit;
        if (c == 0 || stats[c].hexit < hexit) hexit = stats[c].hexit;
    }
    const long natt = nacc + nrej;
    IPAR[10] += (int)(nouter * (p.autonomous ? 1 : 2) + natt); /* Nfun */
    IPAR[11] += (int)nouter;                                  /* Njac */
    IPAR[12] += (int)natt;                                    /* Nstp */
    IPAR[13] += (int)nacc;                                    /* Nacc */
    IPAR[14] += (int)nrej;                                    /* Nrej */
    IPAR[15] += (int)natt;                                    /* Ndec */
    IPAR[16] += (int)(3 * natt);                              /* Nsol */
    RPAR[10] = texit;
    RPAR[11] = hexit;
    return ierr;
}
