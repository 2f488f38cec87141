/*
 * tasep_oracle.c - CPU oracle (test infrastructure only; see tasep_oracle.h).
 *
 * Plain-C restatement of the reference TASEP master-equation path.  Every
 * function cites the reference file:line it follows.  Build with
 * -ffp-contract=off so that multiply-add pairs round exactly as the reference
 * (gcc -std=c99, ISO mode: no contraction) does.
 */
#include "tasep_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ORC_POW2(b) (UINT64_C(1) << (b))

/* src/lib/solv.c:81-135 (identical logic in src/lib/matgen.c:29-67). */
int orc_gen_row(int n, uint64_t i, const double *r, double *val, uint64_t *col)
{
    int c = 0;
    const int top = (int)((i >> (n - 1)) & 1);
    if (top) {                                   /* entry into site 0 */
        col[c] = i - ORC_POW2(n - 1);
        val[c] = r[0];
        c++;
    }
    double d = 0.0;                              /* diagonal, subtraction order kept */
    if (i & 1) d -= r[n];
    if (!top) d -= r[0];
    for (int j = 0; j < n - 1; j++)
        if (!((i >> j) & 1) && ((i >> (j + 1)) & 1)) d -= r[n - 1 - j];
    col[c] = i;
    val[c] = d;
    c++;
    if (!(i & 1)) {                              /* exit from site n-1 */
        col[c] = i + 1;
        val[c] = r[n];
        c++;
    }
    for (int k = 0; k < n - 1; k++)              /* hops, ascending bit */
        if (((i >> k) & 1) && !((i >> (k + 1)) & 1)) {
            col[c] = i + ORC_POW2(k);
            val[c] = r[n - 1 - k];
            c++;
        }
    return c;
}

/* Row sum in entry order, as the gather loop of src/lib/solv.c:9-13. */
static double row_sum(int n, uint64_t i, const double *r, const double *x)
{
    double val[72];
    uint64_t col[72];
    int c = orc_gen_row(n, i, r, val, col);
    double t = 0.0;
    for (int j = 0; j < c; j++) t += val[j] * x[col[j]];
    return t;
}

/* The generator as CSR, built once per run for constant rates: the reference's
 * -f path (gencrs, src/lib/matgen.c:7-74, then the CSR gather of
 * src/lib/solv.c:9-13).  Rows hold the same entries in the same order as
 * orc_gen_row, so every row sum is bit-identical to row_sum; the CSR only
 * saves regenerating the rows at every stage. */
typedef struct {
    uint64_t *rowptr, *col;
    double *val;
} orc_csr;

static int csr_build(int n, const double *r, orc_csr *m)
{
    const int64_t dim = (int64_t)ORC_POW2(n);
    const uint64_t nnz = 2 * (uint64_t)dim + (uint64_t)(n - 1) * ((uint64_t)dim >> 2); /* src/masterEquation.c:593 */
    m->rowptr = (uint64_t *)malloc(((size_t)dim + 1) * sizeof(uint64_t));
    m->col = (uint64_t *)malloc(((size_t)nnz + 1) * sizeof(uint64_t));
    m->val = (double *)malloc(((size_t)nnz + 1) * sizeof(double));
    if (!m->rowptr || !m->col || !m->val) {
        free(m->rowptr); free(m->col); free(m->val);
        return -1;
    }
    const uint64_t hopmask = ORC_POW2(n - 1) - 1;
    uint64_t acc = 0;
    for (int64_t i = 0; i < dim; i++) {  /* row lengths: diagonal, entry, exit, active hops */
        const uint64_t u = (uint64_t)i;
        m->rowptr[i] = acc;
        acc += 1 + ((u >> (n - 1)) & 1) + !(u & 1) + (uint64_t)__builtin_popcountll(u & ~(u >> 1) & hopmask);
    }
    m->rowptr[dim] = acc;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) orc_gen_row(n, (uint64_t)i, r, m->val + m->rowptr[i], m->col + m->rowptr[i]);
    return 0;
}

static void csr_free(orc_csr *m)
{
    free(m->rowptr); free(m->col); free(m->val);
}

static double csr_row(const orc_csr *m, uint64_t i, const double *x)
{
    double t = 0.0;
    for (uint64_t j = m->rowptr[i]; j < m->rowptr[i + 1]; j++) t += m->val[j] * x[m->col[j]];
    return t;
}

/* row i of M x: from the CSR when there is one, else generated on the fly */
#define ROW(csr, n, i, r, x) ((csr) ? csr_row((csr), (i), (x)) : row_sum((n), (i), (r), (x)))

void orc_apply(int n, const double *r, const double *x, double *y)
{
    const int64_t dim = (int64_t)ORC_POW2(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) y[i] = row_sum(n, (uint64_t)i, r, x);
}

/* src/lib/matvec.c:44-68 */
void orc_timevar_rates(int count, const double *period, const double *offset,
                       const double *amplitude, double t, const int *type,
                       const double *constant, double *out)
{
    for (int i = 0; i < count; i++) {
        switch (type[i]) {
        case ORC_FUN_SIN:
            out[i] = amplitude[i] * sin(t * period[i] + offset[i]) + constant[i];
            if (out[i] < 0) out[i] = 0.;
            break;
        case ORC_FUN_COS:
            out[i] = amplitude[i] * cos(t * period[i] + offset[i]) + constant[i];
            if (out[i] < 0) out[i] = 0.;
            break;
        case ORC_FUN_LIN:
            out[i] = amplitude[i] * t + constant[i];
            if (out[i] < 0.) out[i] = 0.;
            break;
        default:
            break;
        }
    }
}

/* src/masterEquation.c:628-642 with src/lib/solv.c:3-26. */
static double step_ref(int n, const double *r, const orc_csr *csr, double h, double *x, double *k)
{
    const int64_t dim = (int64_t)ORC_POW2(n);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) k[i] = h * ROW(csr, n, (uint64_t)i, r, x);
    double checksum = 0;
    for (int64_t i = 0; i < dim; i++) {
        /* k1 = k2 = k3 = k4 = k[i] */
        double d = (k[i] + (2. * k[i]) + (2. * k[i]) + k[i]) / 6.;
        x[i] += d;
        checksum += fabs(d);
    }
    return checksum;
}

double orc_step_ref(int n, const double *r, double h, double *x, double *k)
{
    return step_ref(n, r, NULL, h, x, k);
}

/* Classical RK4 with the stage vector of src/lib/solv.c:14-24 fed back as the
 * gather input of the next stage (csr: the constant-rate generator, or NULL). */
static double step_rk4(int n, const double *r1, const double *r2, const double *r3, const double *r4,
                       const orc_csr *csr, double h, double *x, double *s)
{
    const int64_t dim = (int64_t)ORC_POW2(n);
    double *k1 = s, *k2 = s + dim, *k3 = s + 2 * dim, *k4 = s + 3 * dim;
    double *u = s + 4 * dim, *v = s + 5 * dim;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) {
        double t = ROW(csr, n, (uint64_t)i, r1, x);
        k1[i] = h * t;
        u[i] = (0.5 * h * t) + x[i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) {
        double t = ROW(csr, n, (uint64_t)i, r2, u);
        k2[i] = h * t;
        v[i] = (0.5 * h * t) + x[i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) {
        double t = ROW(csr, n, (uint64_t)i, r3, v);
        k3[i] = h * t;
        u[i] = (h * t) + x[i];
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < dim; i++) k4[i] = h * ROW(csr, n, (uint64_t)i, r4, u);
    double checksum = 0;
    for (int64_t i = 0; i < dim; i++) {
        double d = (k1[i] + (2. * k2[i]) + (2. * k3[i]) + k4[i]) / 6.;
        x[i] += d;
        checksum += fabs(d);
    }
    return checksum;
}

double orc_step_rk4(int n, const double *r1, const double *r2, const double *r3,
                    const double *r4, double h, double *x, double *s)
{
    return step_rk4(n, r1, r2, r3, r4, NULL, h, x, s);
}

/* Largest n whose constant-rate runs keep the generator as CSR (about 0.5 GB). */
#define ORC_CSR_MAX_N 22

/* src/masterEquation.c:402-409 (uniform start), :586 (h), :628-682 (loop and
 * exit rule), :883-897 (time-var: rates at the step start, no exit test). */
int orc_run(const orc_run_cfg *c, double *x, orc_run_result *res)
{
    const int n = c->n;
    const uint64_t dim = ORC_POW2(n);
    if (c->x0) {
        memcpy(x, c->x0, dim * sizeof(double));
    } else if (c->init == ORC_INIT_EMPTY) {
        memset(x, 0, dim * sizeof(double));
        x[0] = 1.0;
    } else {
        double d = (double)ORC_POW2(n);
        double v = 1. / d;
        for (uint64_t i = 0; i < dim; i++) x[i] = v;
    }
    double *scratch = (double *)malloc((c->integrator == ORC_INT_RK4 ? 6 : 1) * dim * sizeof(double));
    if (!scratch) return -1;
    orc_csr csr_store, *csr = NULL;
    if (!c->timevar && n <= ORC_CSR_MAX_N && c->steps > 1 && csr_build(n, c->rates, &csr_store) == 0)
        csr = &csr_store;
    double ra[4][72];
    double t = c->t0, h = c->h, cs = 0;
    int early_stop = 0;
    uint64_t steps_at_stop = 0, i;
    for (i = 0; i < c->steps; i++) {
        if (c->timevar) {
            const double ts[4] = {t, t + h / 2, t + h / 2, t + h};
            for (int s = 0; s < 4; s++) {
                double tt = (c->integrator == ORC_INT_RK4) ? ts[s] : t;
                orc_timevar_rates(n + 1, c->tv_period, c->tv_offset, c->tv_amplitude, tt,
                                  c->tv_type, c->tv_constant, ra[s]);
            }
        } else {
            for (int s = 0; s < 4; s++) memcpy(ra[s], c->rates, (size_t)(n + 1) * sizeof(double));
        }
        if (c->integrator == ORC_INT_RK4)
            cs = step_rk4(n, ra[0], ra[1], ra[2], ra[3], csr, h, x, scratch);
        else
            cs = step_ref(n, ra[0], csr, h, x, scratch);
        t += h;
        if (c->exit_rule) {
            if (cs < c->stop_tol * h) {
                early_stop++;
                steps_at_stop = i;
            } else {
                early_stop = 0;
            }
            if (early_stop > c->stop_count) {
                i++;
                break;
            }
        }
    }
    free(scratch);
    if (csr) csr_free(csr);
    res->steps_done = i;
    res->steps_at_stop = steps_at_stop;
    res->early_stop = early_stop;
    res->last_checksum = cs;
    res->t_end = t;
    return 0;
}

/* src/lib/matvec.c:70-91 */
void orc_densities(int n, const double *x, double *y)
{
    const uint64_t dim = ORC_POW2(n);
    for (int b = 0; b < n; b++) y[b] = 0.;
    for (uint64_t k = 0; k < dim; k++)
        for (int b = 0; b < n; b++)
            if ((k >> b) & 1) y[b] += x[k];
}

/* src/masterEquation.c:1121-1139 and :1289-1302 */
void orc_covariance(int n, const double *x, const double *y, double *cov, double *mul)
{
    const uint64_t dim = ORC_POW2(n);
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) {
            double c = 0;
            for (uint64_t s = 0; s < dim; s++) {
                uint64_t xi = (s >> i) & 1, xk = (s >> k) & 1;
                c += (xk - y[k]) * (xi - y[i]) * x[s];
            }
            cov[(n - 1 - i) * n + (n - 1 - k)] = c;
            if (mul) mul[(n - 1 - i) * n + (n - 1 - k)] = y[k] * y[i] + c;
        }
}

/* src/masterEquation.c:32-45 */
double orc_key_fit(double x, uint64_t id, uint64_t key, int offset, int size)
{
    id >>= offset;
    for (int i = 0; i < size; i++)
        if (((key >> i) & 1) != ((id >> i) & 1)) return 0.;
    return x;
}

/* src/masterEquation.c:47-75.  The reference function falls off its end
 * without a return statement; this returns the value it computes last. */
double orc_high_order_corr(const double *x, uint64_t dim, uint64_t key, int key_size, int offset)
{
    uint64_t kl = key + ORC_POW2(key_size), kr = (key << 1) + 1;
    uint64_t klr = (key << 1) + 1 + ORC_POW2(key_size + 1);
    double lr = 0, no = 0, le = 0, re = 0;
    for (uint64_t i = 0; i < dim; i++) {
        lr += orc_key_fit(x[i], i, klr, offset - 1, key_size + 2);
        no += orc_key_fit(x[i], i, key, offset, key_size);
        le += orc_key_fit(x[i], i, kl, offset, key_size + 1);
        re += orc_key_fit(x[i], i, kr, offset - 1, key_size + 1);
    }
    double ret = lr * no - le * re;
    return ret / sqrt(le * (no - le) * re * (no - re));
}

/* src/masterEquation.c:77-101 */
double orc_error_guess(const double *x, uint64_t dim, uint64_t key, int key_size, int offset)
{
    uint64_t kl = key + ORC_POW2(key_size), kr = (key << 1) + 1;
    uint64_t klr = (key << 1) + 1 + ORC_POW2(key_size + 1);
    double lr = 0, no = 0, le = 0, re = 0;
    for (uint64_t i = 0; i < dim; i++) {
        lr += orc_key_fit(x[i], i, klr, offset - 1, key_size + 2);
        no += orc_key_fit(x[i], i, key, offset, key_size);
        le += orc_key_fit(x[i], i, kl, offset, key_size + 1);
        re += orc_key_fit(x[i], i, kr, offset - 1, key_size + 1);
    }
    return (lr / no - (le / no) * (re / no)) * no;
}

/* src/masterEquation.c:103-127 */
double orc_pf_approx(const double *x, uint64_t dim, uint64_t key, int key_size, int offset)
{
    uint64_t kl = key + ORC_POW2(key_size), kr = (key << 1) + 1;
    double no = 0, le = 0, re = 0;
    for (uint64_t i = 0; i < dim; i++) {
        no += orc_key_fit(x[i], i, key, offset, key_size);
        le += orc_key_fit(x[i], i, kl, offset, key_size + 1);
        re += orc_key_fit(x[i], i, kr, offset - 1, key_size + 1);
    }
    return (le * re) / no;
}

/* src/masterEquation.c:129-143 */
double orc_point_func(const double *x, uint64_t dim, uint64_t key, int key_size, int offset)
{
    double v = 0;
    for (uint64_t i = 0; i < dim; i++) v += orc_key_fit(x[i], i, key, offset, key_size);
    return v;
}

void orc_window4(int n, const double *x, double *p4)
{
    const uint64_t dim = ORC_POW2(n);
    for (int p = 0; p + 4 <= n; p++) {
        double acc[16] = {0};
        for (uint64_t i = 0; i < dim; i++) acc[(i >> p) & 15] += x[i];
        for (int q = 0; q < 16; q++) p4[p * 16 + q] = acc[q];
    }
}
