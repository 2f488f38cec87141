/*
 * me_output.c - output files of the drop-in masterEquation program.
 *
 * File names, line formats and number formats follow the reference's writers
 * (src/masterEquation.c:1019-1539, src/lib/graphlib.c:35-62) so that scripts
 * reading the reference's files read these unchanged.  The values come from
 * the GPU observables (densities, covariance, 4-bit window marginals); only
 * the probability vector itself is copied to the host.
 */
#include "me_host.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <sys/stat.h>
#include <time.h>

void me_err_exit(const char *msg, int code) {
    char date[128];
    time_t t = time(NULL);
    struct tm *tmv = localtime(&t);
    if (!tmv || !strftime(date, sizeof date, "%c", tmv)) date[0] = 0;
    fprintf(stderr, "[%s]:%s\n", date, msg);
    exit(code);
}

int me_read_doubles(const char *path, int count, double *out, const char *fmt) {
    FILE *f = fopen(path, "r");
    if (!f) return -1;
    for (int i = 0; i < count; i++)
        if (fscanf(f, fmt, &out[i]) == EOF) {
            fclose(f);
            return -2;
        }
    fclose(f);
    return 0;
}

/* ---- probabilities --------------------------------------------------------- */

typedef struct {
    int n;
    const double *x;
    uint64_t begin, end;
    char *buf;
    size_t len;
} fmt_job;

static void *fmt_worker(void *arg) {
    fmt_job *j = (fmt_job *)arg;
    char *p = j->buf;
    const int n = j->n;
    for (uint64_t i = j->begin; i < j->end; i++) {
        for (int s = 0; s < n; s++) *p++ = ((i >> (n - 1 - s)) & 1) ? '1' : '0';
        p += sprintf(p, "\t\t%.20g\n", j->x[i]);
    }
    j->len = (size_t)(p - j->buf);
    return NULL;
}

/* Formats lines [b0, b1) on the threads of one buffer set; returns how many
 * jobs were started (tids[t] == 0 marks a job run on the calling thread). */
static int fmt_launch(fmt_job *jobs, pthread_t *tids, int threads, uint64_t per, int n, const double *x,
                      uint64_t b0, uint64_t b1) {
    int used = 0;
    for (int t = 0; t < threads; t++) {
        uint64_t s = b0 + (uint64_t)t * per, e = s + per;
        if (s >= b1) break;
        if (e > b1) e = b1;
        jobs[t].n = n;
        jobs[t].x = x;
        jobs[t].begin = s;
        jobs[t].end = e;
        if (pthread_create(&tids[t], NULL, fmt_worker, &jobs[t]) != 0) fmt_worker(&jobs[t]), tids[t] = 0;
        used++;
    }
    return used;
}

/* The file is written in blocks of 2^20 lines; two buffer sets alternate so
 * that the threads format block k+1 while block k is being written. */
int me_write_probs(const char *path, int n, const double *x, int threads) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    printf("Writing result vector to file '%s'\n", path);
    if (threads < 1) threads = 1;
    if (threads > 128) threads = 128;
    const uint64_t dim = (uint64_t)1 << n;
    const uint64_t block = (uint64_t)1 << 20;
    const size_t line_max = (size_t)n + 2 + 40;
    static fmt_job jobs[2][128];
    pthread_t tids[2][128];
    uint64_t per = (block + threads - 1) / threads;
    int ok = 1;
    for (int k = 0; k < 2; k++)
        for (int t = 0; t < threads; t++) {
            jobs[k][t].buf = (char *)malloc(per * line_max);
            if (!jobs[k][t].buf) ok = 0;
        }
    if (!ok) {
        for (int k = 0; k < 2; k++)
            for (int t = 0; t < threads; t++) free(jobs[k][t].buf);
        fclose(f);
        return -2;
    }
    int used[2] = {0, 0};
    used[0] = fmt_launch(jobs[0], tids[0], threads, per, n, x, 0, dim < block ? dim : block);
    for (uint64_t b0 = 0, k = 0; b0 < dim; b0 += block, k ^= 1) {
        const uint64_t b1 = b0 + block < dim ? b0 + block : dim;
        for (int t = 0; t < used[k]; t++)
            if (tids[k][t]) pthread_join(tids[k][t], NULL);
        if (b1 < dim) used[k ^ 1] = fmt_launch(jobs[k ^ 1], tids[k ^ 1], threads, per, n, x, b1,
                                                b1 + block < dim ? b1 + block : dim);
        for (int t = 0; t < used[k]; t++) fwrite(jobs[k][t].buf, 1, jobs[k][t].len, f);
        printf("-->%f%%\r", 100. * (double)b1 / (double)dim);
    }
    printf("\n");
    for (int k = 0; k < 2; k++)
        for (int t = 0; t < threads; t++) free(jobs[k][t].buf);
    fclose(f);
    return 0;
}

void me_write_prb_txt(const char *path, const me_snaps *s, double dt) {
    /* per-snapshot probabilities; empty without -a (src/masterEquation.c:1047-1062) */
    FILE *f = fopen(path, "w");
    if (!f) {
        printf("ERROR: Cant write to %s\n", path);
        return;
    }
    if (s && s->keep_probs) {
        for (size_t i = 0; i < s->count; i++) {
            const double *p = s->probs + i * s->dim;
            fprintf(f, "%f, ", dt * (double)i);
            for (uint64_t k = 0; k + 1 < s->dim; k++) fprintf(f, "%f, ", p[k]);
            fprintf(f, "%f\n", p[s->dim - 1]);
        }
    }
    fclose(f);
}

void me_write_exp_timed(const char *o, const me_snaps *s, double dt) {
    const size_t size = strlen(o) + 20;
    char *name = (char *)malloc(size);
    snprintf(name, size, "%s_exp_timed.txt", o);
    FILE *f = fopen(name, "w");
    if (f) {
        const int n = s->n;
        for (size_t i = 0; i < s->count; i++) {
            fprintf(f, "%f, ", dt * (double)i);
            for (int k = 0; k < n - 1; k++) fprintf(f, "%lf, ", s->obs[i].y[n - 1 - k]);
            fprintf(f, "%lf\n", s->obs[i].y[0]);
        }
        fclose(f);
    }
    free(name);
}

double me_state_corr(const double *x, int n, int key, int key_size, int offset) {
    const uint64_t dim = (uint64_t)1 << n;
    const uint64_t k_lr = ((uint64_t)key << 1) + 1 + ((uint64_t)1 << (key_size + 1));
    const uint64_t k_le = (uint64_t)key + ((uint64_t)1 << key_size), k_re = ((uint64_t)key << 1) + 1;
    const uint64_t m2 = ((uint64_t)1 << (key_size + 2)) - 1, m1 = ((uint64_t)1 << (key_size + 1)) - 1,
                   m0 = ((uint64_t)1 << key_size) - 1;
    double lr = 0, no = 0, le = 0, re = 0;
    for (uint64_t i = 0; i < dim; i++) {
        const uint64_t lo = i >> (offset - 1), at = i >> offset;
        if ((lo & m2) == (k_lr & m2)) lr += x[i];
        if ((at & m0) == ((uint64_t)key & m0)) no += x[i];
        if ((at & m1) == (k_le & m1)) le += x[i];
        if ((lo & m1) == (k_re & m1)) re += x[i];
    }
    return (lr * no - le * re) / sqrt(le * (no - le) * re * (no - re));
}

/* ---- densities ------------------------------------------------------------------ */

void me_write_exp_values(const char *o, const me_obs *ob) {
    const int n = ob->n;
    const size_t size = strlen(o) + 20;
    char *name = (char *)malloc(size);
    snprintf(name, size, "%s_exp_values_fin.vec", o);
    FILE *f = fopen(name, "w");
    if (f) {
        for (int i = 0; i < n - 1; i++) fprintf(f, "%lf, ", ob->y[n - 1 - i]);
        fprintf(f, "%lf", ob->y[0]);
        fclose(f);
    }
    snprintf(name, size, "%s_exp_values_fin.dat", o);
    f = fopen(name, "w");
    if (f) {
        for (int i = 0; i < n; i++) fprintf(f, "%d Pos%d %lf\n", i, i, ob->y[n - 1 - i]);
        fclose(f);
    }
    free(name);
}

/* ---- matrices and heat maps -------------------------------------------------------- */

int me_write_ppm(const char *path, int rx, int ry, const me_pixel *data) {
    FILE *f = fopen(path, "w");
    if (!f) return -1;
    fprintf(f, "P6\n%d %d\n255\n", rx, ry);
    for (int i = 0; i < rx * ry; i++) fwrite(&data[i], 1, 3, f);
    fclose(f);
    return 0;
}

static void write_matrix(const char *path, int n, const double *m) {
    FILE *f = fopen(path, "w");
    if (!f) return;
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) fprintf(f, k < n - 1 ? "%lf, " : "%lf\n", m[i * n + k]);
    fclose(f);
}

/* Colour of one covariance entry (src/masterEquation.c:1163-1190): blue for
 * negative, red for positive, green near zero; 255*|c|^(1/4) converted to
 * int, then stored in a byte. */
static me_pixel cov_colour(double c) {
    const double intensity = 0.25;
    int r, g, b;
    if (c < 0 && fabs(c) > 0.0001) {
        r = 0;
        g = 0;
        b = (-1) * pow(fabs(c), intensity) * 255;
    } else if (c > 0 && fabs(c) > 0.0001) {
        r = pow(c, intensity) * 255;
        g = 0;
        b = 0;
    } else {
        r = 0;
        g = fabs(pow(fabs(c), intensity) * 255);
        b = 0;
    }
    me_pixel p = {(unsigned char)r, (unsigned char)g, (unsigned char)b};
    return p;
}

/* Grey level of one product entry (src/masterEquation.c:1331-1341). */
static me_pixel mul_colour(double m) {
    const double intensity = 0.25;
    int v = (-1) * pow(fabs(m), intensity) * 255;
    me_pixel p = {(unsigned char)v, (unsigned char)v, (unsigned char)v};
    return p;
}

/* Pixel (x = i, y = k) shows matrix entry [i][k] (set_pixel, src/lib/graphlib.c:86-98). */
static void write_map(const char *path, int n, const double *m, me_pixel (*colour)(double)) {
    me_pixel *img = (me_pixel *)malloc(sizeof(me_pixel) * (size_t)n * (size_t)n);
    if (!img) return;
    for (int i = 0; i < n; i++)
        for (int k = 0; k < n; k++) img[k * n + i] = colour(m[i * n + k]);
    me_write_ppm(path, n, n, img);
    free(img);
}

void me_write_cov(const char *path_mat, const char *path_ppm, const me_obs *ob) {
    write_matrix(path_mat, ob->n, ob->cov);
    write_map(path_ppm, ob->n, ob->cov, cov_colour);
}

void me_write_mul(const char *path_mat, const char *path_ppm, const me_obs *ob) {
    write_matrix(path_mat, ob->n, ob->mul);
    write_map(path_ppm, ob->n, ob->mul, mul_colour);
}

/* ---- window observables ----------------------------------------------------------- */

/* Sum of probabilities of the states whose bits offset..offset+key_size-1
 * equal key (key_fit, src/masterEquation.c:32-45), from the marginals of the
 * 4-bit window that contains those bits. */
double me_win_point(const me_obs *ob, int key, int key_size, int offset) {
    int p = offset < ob->n - 4 ? offset : ob->n - 4;
    if (p < 0) return 0.0;
    const int sh = offset - p, mask = (1 << key_size) - 1;
    double s = 0.0;
    for (int q = 0; q < 16; q++)
        if (((q >> sh) & mask) == key) s += ob->p4[p * 16 + q];
    return s;
}

static void win_terms(const me_obs *ob, int key, int offset, double *lr, double *no, double *le, double *re) {
    const int key_size = 2;
    *lr = me_win_point(ob, (key << 1) + 1 + (1 << (key_size + 1)), key_size + 2, offset - 1);
    *no = me_win_point(ob, key, key_size, offset);
    *le = me_win_point(ob, key + (1 << key_size), key_size + 1, offset);
    *re = me_win_point(ob, (key << 1) + 1, key_size + 1, offset - 1);
}

/* high_order_corr (src/masterEquation.c:47-75): the correlation coefficient it
 * computes.  The reference function returns nothing (undefined behaviour). */
double me_win_corr(const me_obs *ob, int key, int offset) {
    double lr, no, le, re;
    win_terms(ob, key, offset, &lr, &no, &le, &re);
    return (lr * no - le * re) / sqrt(le * (no - le) * re * (no - re));
}

/* error_guess (src/masterEquation.c:77-101). */
double me_win_error_guess(const me_obs *ob, int key, int offset) {
    double lr, no, le, re;
    win_terms(ob, key, offset, &lr, &no, &le, &re);
    return (lr / no - (le / no) * (re / no)) * no;
}

/* higher_order_pf_approx (src/masterEquation.c:103-127): P(L)P(R)/P(middle). */
double me_win_closure(const me_obs *ob, int key, int offset) {
    double lr, no, le, re;
    win_terms(ob, key, offset, &lr, &no, &le, &re);
    return (le * re) / no;
}

void me_write_windows(const char *o, const me_obs *ob) {
    const int n = ob->n;
    int mask_size = 2;
    const size_t size = strlen(o) + 24;
    char *name = (char *)malloc(size);
    FILE *f;

    printf("Calculating Higher Order Correlations\n");
    snprintf(name, size, "%s_highcorr", o);
    if ((f = fopen(name, "w")) != NULL) {
        for (int i = 1; i < n - mask_size; i++) fprintf(f, "\t\t\t%d", i);
        fprintf(f, "\n");
        for (int key = 0; key < (1 << mask_size); key++) {
            for (int i = 0; i < mask_size; i++) fprintf(f, (key >> (mask_size - 1 - i)) & 1 ? "1" : "0");
            fprintf(f, "\t");
            for (int i = 1; i < n - mask_size; i++) fprintf(f, "%1.4g\t", me_win_corr(ob, key, n - mask_size - i));
            fprintf(f, "\n");
        }
        fclose(f);
    }

    const int mask = (1 << mask_size) - 1;
    printf("Calculating error guess\n");
    snprintf(name, size, "%s_error_guess", o);
    if ((f = fopen(name, "w")) != NULL) {
        for (int i = 1; i < n - mask_size; i++)
            fprintf(f, "Error guess for t_%d...t_%d:\t %lf\n", i - 1, i + mask_size,
                    me_win_error_guess(ob, mask, n - mask_size - i));
        fclose(f);
    }

    printf("Calculating closures\n");
    snprintf(name, size, "%s_closures", o);
    if ((f = fopen(name, "w")) != NULL) {
        for (int i = 1; i < n - mask_size; i++)
            fprintf(f, "Value for closure of t_%d...t_%d:\t %lf\n", i - 1, i + mask_size,
                    me_win_closure(ob, mask, n - mask_size - i));
        fclose(f);
    }

    /* the reference sizes this name one character short twice over
       (src/masterEquation.c:1499-1501): the file is "..._high_order_point_fun" */
    mask_size += 2;
    snprintf(name, size, "%s_high_order_point_fun", o);
    if ((f = fopen(name, "w")) != NULL) {
        for (int i = 0; i < n - mask_size + 1; i++)
            fprintf(f, "t_%d...t_%d = %lf\n", i, mask_size + i - 1,
                    me_win_point(ob, (1 << mask_size) - 1, mask_size, n - mask_size - i));
        fclose(f);
    }
    free(name);
}

/* ---- snapshot directories and the timed correlation file ---------------------------- */

void me_write_anim_dir(const char *o, int mul, const me_obs *fin, const me_snaps *s, double dt) {
    const int n = s->n;
    const size_t size = 2 * strlen(o) + 64;
    char *dir = (char *)malloc(size), *name = (char *)malloc(size);
    me_pixel (*colour)(double) = mul ? mul_colour : cov_colour;
    printf(mul ? "Creating directory for mulitplicative expected values animation data\n"
               : "Creating directory for covariance animation data\n");
    snprintf(dir, size, mul ? "%s_multExpval_data" : "%s_covariance_data", o);
    if (mkdir(dir, 0777) == -1) {
        printf("Cauton: Directory <%s> already exists, Data may be overriten or lost! Continue? [Y/N]  ", dir);
        char sel = 'N';
        if (scanf("%c", &sel) == EOF) me_err_exit("ERROR: Issue while reading from stdin", EOF);
        if (sel == 'N' || sel == 'n') exit(-1);
    }
    snprintf(name, size, "%s/%s_fin.ppm", dir, o);
    write_map(name, n, mul ? fin->mul : fin->cov, colour);
    printf(mul ? "Wrote final multiplicative expected values matrix ppm file to <%s>\n"
               : "Wrote final covariance matrix ppm file to <%s>\n", name);
    snprintf(name, size, "%s/%s_all.txt", dir, o);
    FILE *f = fopen(name, "w");
    if (f) {
        for (size_t j = 0; j < s->count; j++) {
            const double *m = mul ? s->obs[j].mul : s->obs[j].cov;
            snprintf(name, size, "%s/%s_%lf.ppm", dir, o, dt * (double)j);
            write_map(name, n, m, colour);
            fprintf(f, "%d Matrix:\n", (int)j);
            for (int i = 0; i < n; i++)
                for (int k = 0; k < n; k++) fprintf(f, k < n - 1 ? "%lf, " : "%lf\n", m[i * n + k]);
            fprintf(f, "\n\n");
        }
        fclose(f);
    }
    free(name);
    free(dir);
}

void me_write_highcorr_timed(const char *o, const me_snaps *s, double dt) {
    /* the reference sizes this name 4 characters short (src/masterEquation.c:1518-1521):
       the file is "<o>_highcorr_timed" */
    const int n = s->n, vals = n > 5 ? n - 5 : 0;
    const size_t size = strlen(o) + 24;
    char *name = (char *)malloc(size);
    snprintf(name, size, "%s_highcorr_timed", o);
    FILE *f = fopen(name, "w");
    if (f) {
        for (size_t i = 0; i < s->count; i++) {
            printf("-->%f%%\r", 100. * (double)(i + 1) / (double)s->count);
            fprintf(f, "%f ", dt * (double)i);
            for (int k = 0; k < vals; k++) fprintf(f, "%1.7g ", s->corr[i * vals + k]);
            fprintf(f, "\n");
        }
        fclose(f);
    }
    free(name);
}
