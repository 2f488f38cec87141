/*
 * ref_harness.c - drives the UNMODIFIED reference library code.
 *
 * TEST INFRASTRUCTURE ONLY.  Compiled together with the reference's own
 * src/lib/{solv,matgen,matvec,io}.c (read in place, never copied) into
 * oracle/_ref/libtasep_ref.so by oracle/Makefile.  The loop below restates
 * the driver loop of src/masterEquation.c so that runs can start from the
 * empty lattice and use any exit tolerance; the arithmetic (gencrs,
 * rk4_step, gen_meq_row, rk4_step_reduced, timeVariantProbs) is the
 * reference's compiled code.
 */
#include <fcntl.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>

#include "matgen.h"
#include "matvec.h"
#include "solv.h"

#define RH_POW2(b) (UINT64_C(1) << (b))

/* gencrs prints one progress line per row (src/lib/matgen.c:18); route it
 * to /dev/null while it runs. */
static void build_csr(int n, uint64_t rows, double *rates, uint64_t *rowPtr, double *valArr,
                      uint64_t *colInd)
{
    int bit[64];
    fflush(stdout);
    int saved = dup(1);
    int devnull = open("/dev/null", O_WRONLY);
    if (devnull >= 0) dup2(devnull, 1);
    gencrs(rowPtr, valArr, colInd, rates, bit, rows, n);
    fflush(stdout);
    if (saved >= 0) {
        dup2(saved, 1);
        close(saved);
    }
    if (devnull >= 0) close(devnull);
}

typedef struct {
    uint64_t steps_done, steps_at_stop;
    int early_stop;
    double last_checksum, t_end;
} refh_result;

/*
 * Constant-rate run through the -f path (use_csr=1: gencrs + rk4_step,
 * src/masterEquation.c:586-682) or the per-row path (use_csr=0:
 * gen_meq_row + rk4_step_reduced, src/masterEquation.c:926-981).
 * Time-variant run (timevar=1): src/masterEquation.c:883-921, per-row path,
 * rates from timeVariantProbs at the step start, no exit test.
 * init: 0 uniform (as coded at src/masterEquation.c:402-409), 1 empty lattice.
 */
int refh_run(int n, const double *rates_in, double t, double h, uint64_t steps,
             double stop_tol, int stop_count, int init, int use_csr, int timevar,
             const int *tv_type, const double *tv_amp, const double *tv_period,
             const double *tv_offset, const double *tv_const, int nthreads, double *x,
             refh_result *res)
{
    const uint64_t dim = RH_POW2(n);
    double *rates = (double *)malloc((size_t)(n + 1) * sizeof(double));
    memcpy(rates, rates_in, (size_t)(n + 1) * sizeof(double));
    if (nthreads > 0) omp_set_num_threads(nthreads);
    if (init == 1) {
        memset(x, 0, dim * sizeof(double));
        x[0] = 1.0;
    } else {
        double d = (double)RH_POW2(n);
        for (uint64_t i = 0; i < dim; i++) x[i] = 1. / d;
    }
    double *x1 = malloc(dim * sizeof(double)), *k1 = malloc(dim * sizeof(double));
    double *k2 = malloc(dim * sizeof(double)), *k3 = malloc(dim * sizeof(double));
    double *k4 = malloc(dim * sizeof(double));
    double checksum = 0;
    int early_stop = 0;
    uint64_t steps_at_stop = 0, i = 0;
    if (use_csr && !timevar) {
        uint64_t size = 2 * RH_POW2(n) + RH_POW2(n - 2) * (n - 1);
        if (n < 2) size = 2 * RH_POW2(n) + 1;
        uint64_t *rowPtr = malloc((dim + 1) * sizeof(uint64_t));
        double *valArr = malloc(size * sizeof(double));
        uint64_t *colInd = malloc(size * sizeof(uint64_t));
        build_csr(n, dim, rates, rowPtr, valArr, colInd);
        for (i = 0; i < steps; i++) {
            checksum = 0;
            rk4_step(1, dim, k1, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(2, dim, k2, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(3, dim, k3, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(4, dim, k4, x, x1, rowPtr, colInd, valArr, h);
            for (uint64_t k = 0; k < dim; k++) {
                x[k] += (k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.;
                checksum += fabs((k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.);
            }
            t += h;
            if (checksum < stop_tol * h) {
                early_stop++;
                steps_at_stop = i;
            } else {
                early_stop = 0;
            }
            if (early_stop > stop_count) {
                i++;
                break;
            }
        }
        free(rowPtr);
        free(valArr);
        free(colInd);
    } else {
        double valArr[72];
        uint64_t colInd[72];
        for (i = 0; i < steps; i++) {
            if (timevar)
                timeVariantProbs(rates, n + 1, (double *)tv_period, (double *)tv_offset,
                                 (double *)tv_amp, t, (int *)tv_type, (double *)tv_const);
            for (uint64_t k = 0; k < dim; k++) {
                uint64_t c = gen_meq_row(n, k, rates, valArr, (uint_fast64_t *)colInd);
                rk4_step_reduced(1, c, k, &k1[k], x, x1, colInd, valArr, h);
                rk4_step_reduced(2, c, k, &k2[k], x, x1, colInd, valArr, h);
                rk4_step_reduced(3, c, k, &k3[k], x, x1, colInd, valArr, h);
                rk4_step_reduced(4, c, k, &k4[k], x, x1, colInd, valArr, h);
            }
            checksum = 0;
            for (uint64_t k = 0; k < dim; k++) {
                x[k] += (k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.;
                checksum += fabs((k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.);
            }
            t += h;
            if (timevar) continue;
            if (checksum < stop_tol * h) {
                early_stop++;
                steps_at_stop = i;
            } else {
                early_stop = 0;
            }
            if (early_stop > stop_count) {
                i++;
                break;
            }
        }
    }
    free(x1);
    free(k1);
    free(k2);
    free(k3);
    free(k4);
    free(rates);
    res->steps_done = i;
    res->steps_at_stop = steps_at_stop;
    res->early_stop = early_stop;
    res->last_checksum = checksum;
    res->t_end = t;
    return 0;
}

/* The reference generator as CSR (gencrs, src/lib/matgen.c:7-74) for the
 * first `rows` rows; returns nnz.  Arrays sized by the caller. */
uint64_t refh_gencrs(int n, uint64_t rows, const double *rates, uint64_t *rowPtr,
                     double *valArr, uint64_t *colInd)
{
    double r[72];
    memcpy(r, rates, (size_t)(n + 1) * sizeof(double));
    build_csr(n, rows, r, rowPtr, valArr, colInd);
    return rowPtr[rows];
}

static double now_s(void)
{
    struct timeval tv;
    gettimeofday(&tv, NULL);
    return (double)tv.tv_sec + 1e-6 * (double)tv.tv_usec;
}

/*
 * Times the reference -f step (four rk4_step calls with OpenMP over rows and
 * the serial update, src/masterEquation.c:628-642) on the first `rows` rows of
 * the 2^n-state generator: `reps` timed steps after one untimed one.  Returns
 * seconds per step for that row sample, or a negative value when memory runs
 * out.
 */
double refh_time_sample(int n, uint64_t rows, const double *rates, double h, int reps,
                        int nthreads, uint64_t *nnz_out)
{
    const uint64_t dim = RH_POW2(n);
    if (rows > dim) rows = dim;
    if (nthreads > 0) omp_set_num_threads(nthreads);
    /* a row has at most n+2 entries */
    uint64_t cap = rows * (uint64_t)(n / 2 + 4);
    uint64_t *rowPtr = malloc((rows + 1) * sizeof(uint64_t));
    double *valArr = malloc(cap * sizeof(double));
    uint64_t *colInd = malloc(cap * sizeof(uint64_t));
    double *x = malloc(dim * sizeof(double));
    double *x1 = malloc(rows * sizeof(double)), *k1 = malloc(rows * sizeof(double));
    double *k2 = malloc(rows * sizeof(double)), *k3 = malloc(rows * sizeof(double));
    double *k4 = malloc(rows * sizeof(double));
    if (!rowPtr || !valArr || !colInd || !x || !x1 || !k1 || !k2 || !k3 || !k4) return -1.0;
    double r[72];
    memcpy(r, rates, (size_t)(n + 1) * sizeof(double));
    build_csr(n, rows, r, rowPtr, valArr, colInd);
    if (nnz_out) *nnz_out = rowPtr[rows];
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < dim; i++) x[i] = 1.0 / (double)dim;
    double t0 = 0, checksum = 0;
    for (int rep = -1; rep < reps; rep++) {
        if (rep == 0) t0 = now_s();
        checksum = 0;
        rk4_step(1, rows, k1, x, x1, rowPtr, colInd, valArr, h);
        rk4_step(2, rows, k2, x, x1, rowPtr, colInd, valArr, h);
        rk4_step(3, rows, k3, x, x1, rowPtr, colInd, valArr, h);
        rk4_step(4, rows, k4, x, x1, rowPtr, colInd, valArr, h);
        for (uint64_t k = 0; k < rows; k++) {
            x[k] += (k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.;
            checksum += fabs((k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.);
        }
    }
    double secs = (now_s() - t0) / (reps > 0 ? reps : 1);
    free(rowPtr);
    free(valArr);
    free(colInd);
    free(x);
    free(x1);
    free(k1);
    free(k2);
    free(k3);
    free(k4);
    if (!(checksum >= 0)) return -2.0;
    return secs;
}

/* The -f generator built row by row in parallel with the reference's own
 * gen_meq_row (src/lib/solv.c:81-135), which yields the rows gencrs writes
 * (src/lib/matgen.c:29-67; refh_csr_matches_gencrs checks it).  The serial
 * gencrs, with its progress line per row, takes minutes at n = 28. */
static void build_csr_parallel(int n, uint64_t rows, double *rates, uint64_t *rowPtr, double *valArr,
                               uint64_t *colInd)
{
    const uint64_t hopmask = RH_POW2(n - 1) - 1;
    uint64_t acc = 0;
    for (uint64_t i = 0; i < rows; i++) {
        rowPtr[i] = acc;
        acc += 1 + ((i >> (n - 1)) & 1) + !(i & 1) + (uint64_t)__builtin_popcountll(i & ~(i >> 1) & hopmask);
    }
    rowPtr[rows] = acc;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)rows; i++)
        gen_meq_row(n, (uint_fast64_t)i, rates, valArr + rowPtr[i], (uint_fast64_t *)(colInd + rowPtr[i]));
}

/* 1 if the parallel builder reproduces gencrs's CSR exactly (n <= 20). */
int refh_csr_matches_gencrs(int n, const double *rates_in)
{
    if (n < 2 || n > 20) return -1;
    const uint64_t dim = RH_POW2(n), size = 2 * RH_POW2(n) + RH_POW2(n - 2) * (n - 1);
    double r[72];
    memcpy(r, rates_in, (size_t)(n + 1) * sizeof(double));
    uint64_t *p1 = malloc((dim + 1) * sizeof(uint64_t)), *p2 = malloc((dim + 1) * sizeof(uint64_t));
    uint64_t *c1 = malloc(size * sizeof(uint64_t)), *c2 = malloc(size * sizeof(uint64_t));
    double *v1 = malloc(size * sizeof(double)), *v2 = malloc(size * sizeof(double));
    int ok = p1 && p2 && c1 && c2 && v1 && v2;
    if (ok) {
        build_csr(n, dim, r, p1, v1, c1);
        build_csr_parallel(n, dim, r, p2, v2, c2);
        ok = !memcmp(p1, p2, (dim + 1) * sizeof(uint64_t)) && p1[dim] == size &&
             !memcmp(c1, c2, size * sizeof(uint64_t)) && !memcmp(v1, v2, size * sizeof(double));
    }
    free(p1); free(p2); free(c1); free(c2); free(v1); free(v2);
    return ok;
}

/*
 * The reference's -f step on the WHOLE 2^n-state generator (the bench's
 * reference arm): CSR of all rows (built in parallel, above), x uniform, then
 * `warm` untimed and `reps` timed steps of rk4_step x4 + the serial update and
 * L1 norm (src/masterEquation.c:628-642).  Returns seconds per step, or a
 * negative value when memory runs out; *build_secs gets the set-up time.
 */
double refh_time_full(int n, const double *rates, double h, int warm, int reps, int nthreads,
                      double *build_secs, uint64_t *nnz_out)
{
    if (nthreads > 0) omp_set_num_threads(nthreads);
    const uint64_t dim = RH_POW2(n);
    const uint64_t size = 2 * RH_POW2(n) + RH_POW2(n - 2) * (n - 1);
    const double tb = now_s();
    uint64_t *rowPtr = malloc((dim + 1) * sizeof(uint64_t));
    double *valArr = malloc(size * sizeof(double));
    uint64_t *colInd = malloc(size * sizeof(uint64_t));
    double *x = malloc(dim * sizeof(double)), *x1 = malloc(dim * sizeof(double));
    double *k1 = malloc(dim * sizeof(double)), *k2 = malloc(dim * sizeof(double));
    double *k3 = malloc(dim * sizeof(double)), *k4 = malloc(dim * sizeof(double));
    double secs = -1.0;
    if (rowPtr && valArr && colInd && x && x1 && k1 && k2 && k3 && k4) {
        double r[72];
        memcpy(r, rates, (size_t)(n + 1) * sizeof(double));
        build_csr_parallel(n, dim, r, rowPtr, valArr, colInd);
        if (nnz_out) *nnz_out = rowPtr[dim];
#pragma omp parallel for schedule(static)
        for (uint64_t i = 0; i < dim; i++) x[i] = 1.0 / (double)dim;
        if (build_secs) *build_secs = now_s() - tb;
        double t0 = 0, checksum = 0;
        for (int rep = -warm; rep < reps; rep++) {
            if (rep == 0) t0 = now_s();
            checksum = 0;
            rk4_step(1, dim, k1, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(2, dim, k2, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(3, dim, k3, x, x1, rowPtr, colInd, valArr, h);
            rk4_step(4, dim, k4, x, x1, rowPtr, colInd, valArr, h);
            for (uint64_t k = 0; k < dim; k++) {
                x[k] += (k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.;
                checksum += fabs((k1[k] + (2. * k2[k]) + (2. * k3[k]) + k4[k]) / 6.);
            }
        }
        secs = (now_s() - t0) / (reps > 0 ? reps : 1);
        if (!(checksum >= 0)) secs = -2.0;
    }
    free(rowPtr); free(valArr); free(colInd); free(x); free(x1);
    free(k1); free(k2); free(k3); free(k4);
    return secs;
}

int refh_max_threads(void) { return omp_get_max_threads(); }
