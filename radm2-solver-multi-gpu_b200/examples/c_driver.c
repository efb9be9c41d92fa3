/*
 * A C caller of the library, shaped like the reference's host flow (mgpu.cu:3891-3911):
 * inputs in, rate constants, one Rosenbrock integration, state out.  Plain C99 against
 * include/radm2.h and libradm2_b200.so: the drop-in boundary with no C++ or Python.
 *
 *   c_driver IN OUT     IN:  int32 ncell, then VAR[n][59], FIX[n][2], TEMP[n], RC_N2O5[n],
 *                            JV[n][28] (float64, the reference's per-cell layout)
 *                       OUT: VAR[n][59] after one 600 s step, then int32 IPAR[20]
 * Exit status 0 on success; the IERR text on stderr otherwise.
 */
#include <stdio.h>
#include <stdlib.h>

#include "radm2.h"

static int read_all(FILE *f, void *p, size_t size, size_t n) { return fread(p, size, n, f) == n; }

int main(int argc, char **argv)
{
    if (argc != 3) {
        fprintf(stderr, "usage: %s IN OUT\n", argv[0]);
        return 2;
    }
    FILE *in = fopen(argv[1], "rb");
    if (!in) return 2;
    int n = 0;
    if (!read_all(in, &n, sizeof n, 1) || n <= 0) return 2;
    double *var = malloc(sizeof(double) * n * RADM2_NVAR), *fix = malloc(sizeof(double) * n * RADM2_NFIX);
    double *temp = malloc(sizeof(double) * n), *rcn = malloc(sizeof(double) * n);
    double *jv = malloc(sizeof(double) * n * RADM2_NPH);
    if (!var || !fix || !temp || !rcn || !jv) return 2;
    if (!read_all(in, var, sizeof(double), (size_t)n * RADM2_NVAR) ||
        !read_all(in, fix, sizeof(double), (size_t)n * RADM2_NFIX) || !read_all(in, temp, sizeof(double), n) ||
        !read_all(in, rcn, sizeof(double), n) || !read_all(in, jv, sizeof(double), (size_t)n * RADM2_NPH))
        return 2;
    fclose(in);

    radm2_opts o;
    radm2_opts_default(&o);
    o.schedule = RADM2_SCHED_PERSISTENT;
    radm2_ctx *chem = NULL;
    int rc = radm2_create(&chem, &o);
    if (rc != RADM2_OK) {
        fprintf(stderr, "radm2_create: %s\n", radm2_error_string(rc));
        return 1;
    }
    /* convertWRFChemData / updatingCoefficientWRFChemData / INTEGRATE (mgpu.cu:3856-3873) */
    double atol[RADM2_NVAR], rtol[RADM2_NVAR], rpar[20] = {0};
    int ipar[20] = {0};
    for (int i = 0; i < RADM2_NVAR; i++) {
        atol[i] = 1.0;
        rtol[i] = 1.0e-3;
    }
    ipar[0] = 1;
    ipar[3] = 2;
    rpar[2] = 0.01 * 600.0;
    rc = radm2_set_inputs(chem, n, var, fix, temp, rcn, jv);
    if (rc == RADM2_OK) rc = radm2_update_rconst(chem);
    int ierr = rc == RADM2_OK ? radm2_rosenbrock(chem, 0.0, 600.0, atol, rtol, rpar, ipar) : rc;
    if (ierr != 1) {
        fprintf(stderr, "Rosenbrock: %s (%s)\n", radm2_error_string(ierr), radm2_last_error(chem));
        return 1;
    }
    radm2_get_state(chem, var);
    radm2_destroy(chem);

    FILE *out = fopen(argv[2], "wb");
    if (!out || fwrite(var, sizeof(double), (size_t)n * RADM2_NVAR, out) != (size_t)n * RADM2_NVAR ||
        fwrite(ipar, sizeof(int), 20, out) != 20)
        return 2;
    fclose(out);
    printf("c_driver: %d cells, Nacc %d Nrej %d\n", n, ipar[13], ipar[14]);
    free(var);
    free(fix);
    free(temp);
    free(rcn);
    free(jv);
    return 0;
}
