/*
 * me_host.h - host side of the drop-in masterEquation program: option state,
 * output writers and small utilities.  C99.
 */
#ifndef ME_HOST_H
#define ME_HOST_H

#include <stdint.h>
#include <stdio.h>

#define ME_MAX_N 33

/* Fatal error with a timestamp on stderr, as err_exit (reference
 * src/lib/io.c:13-19). */
void me_err_exit(const char *msg, int code);

/* Reads `count` doubles with fscanf("%lf"); returns 0 on success. */
int me_read_doubles(const char *path, int count, double *out, const char *sep_fmt);

/* Observables of the final state, everything the writers need. */
typedef struct {
    int n;
    double y[ME_MAX_N];                /* bit-order densities (condense)      */
    double cov[ME_MAX_N * ME_MAX_N];   /* site order                           */
    double mul[ME_MAX_N * ME_MAX_N];   /* site order                           */
    double p4[(ME_MAX_N - 3) * 16];    /* 4-bit window marginals               */
} me_obs;

/* Probability file: one line per state, site-0-first bit string then
 * "\t\t%.20g" (reference src/masterEquation.c:1021-1040).  Formatting runs on
 * `threads` threads; the file is written in index order. */
int me_write_probs(const char *path, int n, const double *x, int threads);

/* Snapshots of the -a option, one per step whose index is a multiple of the
 * resolution (src/masterEquation.c:646-666): the observables of each, the
 * state itself when the probability files are selected, and the 4-site
 * correlation values of the timed correlation file. */
typedef struct {
    int n;
    uint64_t dim;
    int keep_probs;
    size_t count, cap;
    me_obs *obs;   /* count entries */
    double *probs; /* count * dim when keep_probs */
    double *corr;  /* count * (n - 5) */
} me_snaps;

/* high_order_corr (src/masterEquation.c:47-75) evaluated on a full state
 * vector: the correlation coefficient of the window around bits
 * offset..offset+key_size-1. */
double me_state_corr(const double *x, int n, int key, int key_size, int offset);

/* The remaining files of src/masterEquation.c:1042-1539.  dt is the time the
 * reference assigns between snapshots (h times the resolution). */
void me_write_prb_txt(const char *path, const me_snaps *s, double dt);
void me_write_exp_timed(const char *o_filename, const me_snaps *s, double dt);
/* <o>_covariance_data/ (mul = 0) or <o>_multExpval_data/ (mul = 1):
 * <o>_fin.ppm, one <o>_<time>.ppm per snapshot and <o>_all.txt
 * (src/masterEquation.c:1197-1279, 1345-1417). */
void me_write_anim_dir(const char *o_filename, int mul, const me_obs *fin, const me_snaps *s, double dt);
void me_write_highcorr_timed(const char *o_filename, const me_snaps *s, double dt);
void me_write_exp_values(const char *o_filename, const me_obs *ob);
void me_write_cov(const char *path_mat, const char *path_ppm, const me_obs *ob);
void me_write_mul(const char *path_mat, const char *path_ppm, const me_obs *ob);
void me_write_windows(const char *o_filename, const me_obs *ob);

/* Window quantities from the 4-bit marginals (src/masterEquation.c:32-143);
 * offset as in the reference (bits offset..offset+key_size-1 hold the key). */
double me_win_point(const me_obs *ob, int key, int key_size, int offset);
double me_win_corr(const me_obs *ob, int key, int offset);
double me_win_error_guess(const me_obs *ob, int key, int offset);
double me_win_closure(const me_obs *ob, int key, int offset);

/* Learned warm start (--init learned): reads the shipped network parameters
 * (a float32 .npy of TASEP_MLP_PARAMS values), builds the network inputs
 * from the rates (first-order mean-field profile, 16 values per site),
 * predicts on the GPU and sets the pair-Markov initial measure.  Returns 0,
 * 1 if the prediction was infeasible (the handle is unchanged), -1 on error. */
struct tasep_meq;
int me_warm_params_load(const char *path, float *params);
void me_warm_mean_field(int n, const double *rates, double *rho);
void me_warm_features(int n, const double *rates, const double *mf, float *features);
int me_warm_start(struct tasep_meq *m, int n, const double *rates, const char *params_path, int device);

/* Minimal P6 writer (src/lib/graphlib.c:35-62 format). */
typedef struct {
    unsigned char r, g, b;
} me_pixel;
int me_write_ppm(const char *path, int rx, int ry, const me_pixel *data);

#endif
