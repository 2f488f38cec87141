/*
 * me_warm.c - the learned warm start for the drop-in program (--init learned):
 * network inputs from the rates, the shipped trained parameters, prediction
 * on the GPU and the pair-Markov initial measure.  The inputs are built
 * exactly as tasep_b200/warmstart.py builds them (site_features,
 * mean_field_profile), so both front ends feed the network the same numbers.
 */
#include <stdlib.h>
#include <string.h>

#include "me_host.h"
#include "tasep.h"

#define ME_MF_STEPS 20000
#define ME_COV_SCALE 10.0

int me_warm_params_load(const char *path, float *params) {
    FILE *f = fopen(path, "rb");
    if (!f) return -1;
    unsigned char head[10];
    int rc = -2;
    if (fread(head, 1, 10, f) == 10 && memcmp(head, "\x93NUMPY", 6) == 0 && head[6] == 1) {
        const unsigned hlen = head[8] | (head[9] << 8);
        char *dict = (char *)malloc(hlen + 1);
        if (dict && fread(dict, 1, hlen, f) == hlen) {
            dict[hlen] = 0;
            char shape[32];
            snprintf(shape, sizeof shape, "(%d,)", TASEP_MLP_PARAMS);
            if (strstr(dict, "'<f4'") && strstr(dict, "'fortran_order': False") && strstr(dict, shape) &&
                fread(params, sizeof(float), TASEP_MLP_PARAMS, f) == TASEP_MLP_PARAMS)
                rc = 0;
        }
        free(dict);
    }
    fclose(f);
    return rc;
}

void me_warm_mean_field(int n, const double *r, double *rho) {
    double rmax = r[0];
    for (int i = 1; i <= n; i++)
        if (r[i] > rmax) rmax = r[i];
    const double dt = 0.25 / rmax;
    double *J = (double *)malloc(sizeof(double) * (size_t)(n + 1));
    for (int i = 0; i < n; i++) rho[i] = 0.5;
    for (int s = 0; s < ME_MF_STEPS; s++) {
        J[0] = r[0] * (1.0 - rho[0]);
        for (int i = 1; i < n; i++) J[i] = r[i] * rho[i - 1] * (1.0 - rho[i]);
        J[n] = r[n] * rho[n - 1];
        for (int i = 0; i < n; i++) rho[i] += dt * (J[i] - J[i + 1]);
    }
    for (int i = 0; i < n; i++) rho[i] = rho[i] < 1e-6 ? 1e-6 : (rho[i] > 1.0 - 1e-6 ? 1.0 - 1e-6 : rho[i]);
    free(J);
}

void me_warm_features(int n, const double *r, const double *mf, float *f) {
    for (int j = 0; j < n; j++) {
        float *o = f + (size_t)j * TASEP_MLP_IN;
        for (int w = 0; w < 9; w++) {
            const int k = j - 4 + w;
            o[w] = (float)(k >= 0 && k <= n ? r[k] : 0.0);
        }
        o[9] = (float)(1.0 / (j + 1));
        o[10] = (float)(1.0 / (n - j));
        o[11] = (float)r[0];
        o[12] = (float)r[n];
        o[13] = (float)(j > 0 ? mf[j - 1] : 0.0);
        o[14] = (float)mf[j];
        o[15] = (float)(j + 1 < n ? mf[j + 1] : 1.0);
    }
}

int me_warm_start(tasep_meq *m, int n, const double *rates, const char *params_path, int device) {
    float *params = (float *)malloc(sizeof(float) * TASEP_MLP_PARAMS);
    float *feat = (float *)malloc(sizeof(float) * (size_t)n * TASEP_MLP_IN);
    float *y = (float *)malloc(sizeof(float) * (size_t)n * TASEP_MLP_OUT);
    double *mf = (double *)malloc(sizeof(double) * (size_t)n);
    double *rho = (double *)malloc(sizeof(double) * (size_t)n), *cov = (double *)malloc(sizeof(double) * (size_t)n);
    tasep_mlp *net = NULL;
    int rc = -1;
    if (!params || !feat || !y || !mf || !rho || !cov) goto out;
    if (me_warm_params_load(params_path, params) != 0) {
        printf("ERROR: Cannot read the warm-start parameters <%s>\n", params_path);
        goto out;
    }
    me_warm_mean_field(n, rates, mf);
    me_warm_features(n, rates, mf, feat);
    if (tasep_mlp_create(device, 0, &net) != TASEP_OK || tasep_mlp_set_params(net, params) != TASEP_OK ||
        tasep_mlp_predict(net, feat, n, y) != TASEP_OK)
        goto out;
    for (int j = 0; j < n; j++) {
        rho[j] = (double)y[j * TASEP_MLP_OUT];
        cov[j] = (double)y[j * TASEP_MLP_OUT + 1] / ME_COV_SCALE;
    }
    tasep_status st = tasep_meq_init_pair_markov(m, rho, cov);
    if (st == TASEP_OK) rc = 0;
    else if (st == TASEP_ERR_INVALID) rc = 1; /* infeasible prediction: the caller starts empty */
out:
    if (net) tasep_mlp_destroy(net);
    free(params);
    free(feat);
    free(y);
    free(mf);
    free(rho);
    free(cov);
    return rc;
}
