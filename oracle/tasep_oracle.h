/*
 * tasep_oracle.h - CPU oracle for the TASEP master-equation integrator.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (KilianPiochUBT/TASEP, src/lib/solv.c, src/lib/matgen.c,
 * src/lib/matvec.c, src/masterEquation.c).  It is the checker that tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg compare the CUDA
 * path against.  The product library (libtasep_cuda.so) never links it.
 *
 * Conventions (identical to the reference):
 *   N = 2^n states; bit b of a state index is site n-1-b (site 0 = entry).
 *   rates r[0..n]: r[0] = alpha (entry into site 0), r[j] = hop site j-1 -> j,
 *   r[n] = beta (exit from site n-1).
 */
#ifndef TASEP_ORACLE_H
#define TASEP_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { ORC_INT_REF = 0, ORC_INT_RK4 = 1 };
enum { ORC_INIT_UNIFORM = 0, ORC_INIT_EMPTY = 1 };
enum { ORC_FUN_SIN = 0, ORC_FUN_COS = 1, ORC_FUN_LIN = 2 };

/* One generator row in the reference's entry order (entry, diagonal, exit,
 * hops ascending).  Returns the entry count.  Follows src/lib/solv.c:81-135. */
int orc_gen_row(int n, uint64_t i, const double *r, double *val, uint64_t *col);

/* y = M x with each row summed in the reference's order, separate multiply
 * and add (src/lib/solv.c:9-13). */
void orc_apply(int n, const double *r, const double *x, double *y);

/* Time-dependent rates r_i(t), clamped at 0 (src/lib/matvec.c:44-68). */
void orc_timevar_rates(int count, const double *period, const double *offset,
                       const double *amplitude, double t, const int *type,
                       const double *constant, double *out);

/* Reference-compatible step: the four stage calls all gather from x
 * (src/masterEquation.c:630-636, src/lib/solv.c:13), so k1=k2=k3=k4=h*M*x;
 * x += (k1+2k2+2k3+k4)/6 with the reference's evaluation order.  Returns the
 * L1 norm of the increment, summed serially (src/masterEquation.c:639-642).
 * scratch: N doubles. */
double orc_step_ref(int n, const double *r, double h, double *x, double *scratch);

/* Classical RK4 with the stage inputs threaded: x1 = x + h/2*k1, x + h/2*k2,
 * x + h*k3 (the stage vector the reference writes at src/lib/solv.c:14-24 but
 * never reads).  r1..r4: rates at the four stage times.  scratch: 5N doubles.
 * Returns the serial L1 norm of the increment. */
double orc_step_rk4(int n, const double *r1, const double *r2, const double *r3,
                    const double *r4, double h, double *x, double *scratch);

typedef struct {
    int n;
    int integrator;          /* ORC_INT_REF | ORC_INT_RK4 */
    int init;                /* ORC_INIT_UNIFORM | ORC_INIT_EMPTY (ignored if x0) */
    const double *x0;        /* optional initial state, N doubles */
    const double *rates;     /* n+1 rates (constant-rate runs) */
    int timevar;             /* 1: rates from the time-variant functions */
    const int *tv_type;      /* n+1 each, when timevar */
    const double *tv_amplitude, *tv_period, *tv_offset, *tv_constant;
    double t0, h;
    uint64_t steps;
    double stop_tol;         /* exit when checksum < stop_tol*h ... */
    int stop_count;          /* ... for more than stop_count consecutive steps */
    int exit_rule;           /* 0: never exit early (reference time-var loop) */
} orc_run_cfg;

typedef struct {
    uint64_t steps_done;     /* loop iterations executed */
    uint64_t steps_at_stop;  /* last qualifying step index */
    int early_stop;          /* consecutive qualifying steps at the end */
    double last_checksum;
    double t_end;
} orc_run_result;

/* Full integration loop with the reference's exit rule
 * (src/masterEquation.c:628-682 constant rates; :883-921 time-var, which
 * evaluates all stage rates at the step start time).  x: N doubles (out). */
int orc_run(const orc_run_cfg *cfg, double *x, orc_run_result *res);

/* Per-bit densities y[b] = sum_{i: bit b set} x_i (src/lib/matvec.c:70-91). */
void orc_densities(int n, const double *x, double *y);

/* Covariance in site order, cov[(n-1-i)*n + (n-1-k)] =
 * sum_s (b_k(s)-y_k)(b_i(s)-y_i) x_s  (src/masterEquation.c:1121-1139);
 * mul[...] = y_k*y_i + that sum (src/masterEquation.c:1289-1302). */
void orc_covariance(int n, const double *x, const double *y, double *cov, double *mul);

/* Window observables (src/masterEquation.c:32-143). */
double orc_key_fit(double x, uint64_t id, uint64_t key, int offset, int size);
double orc_high_order_corr(const double *x, uint64_t dim, uint64_t key, int key_size, int offset);
double orc_error_guess(const double *x, uint64_t dim, uint64_t key, int key_size, int offset);
double orc_pf_approx(const double *x, uint64_t dim, uint64_t key, int key_size, int offset);
double orc_point_func(const double *x, uint64_t dim, uint64_t key, int key_size, int offset);

/* 4-bit window marginals P4[p*16 + pattern] = sum over states whose bits
 * p..p+3 equal pattern (bit p = pattern bit 0), p = 0..n-4. */
void orc_window4(int n, const double *x, double *p4);

#ifdef __cplusplus
}
#endif
#endif
