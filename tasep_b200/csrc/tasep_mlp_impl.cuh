// tasep_mlp_impl.cuh - C ABI of the learned warm start (tasep_mlp_*,
// tasep_meq_init_pair_markov; include/tasep.h).  Included at the end of
// tasep_api.cu.
#pragma once

#include <cmath>

#include "meq_mlp.cuh"

static_assert(TASEP_MLP_PARAMS == kMlpParams, "parameter count");
static_assert(TASEP_MLP_IN == kMlpIn && TASEP_MLP_OUT == kMlpOut, "network shape");

struct tasep_mlp {
    int device = 0;
    float *master = nullptr, *m1 = nullptr, *m2 = nullptr, *gsum = nullptr, *grows = nullptr, *loss = nullptr;
    __nv_bfloat16 *w = nullptr;
    int *err = nullptr;  // set by a kernel whose tensor-core wait timed out
    int grow_cap = 0;
    long long adam_t = 0;
};

namespace {

uint64_t mlp_rng(uint64_t &s) {  // splitmix64
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}
double mlp_unif(uint64_t &s) { return double(mlp_rng(s) >> 11) * (1.0 / 9007199254740992.0); }

tasep_status mlp_configure() {
    static std::atomic<bool> done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!done[dev & 63].load(std::memory_order_acquire)) {
        CU_TRY(cudaFuncSetAttribute(mlp_forward_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(kMlpForwardSmem)));
        CU_TRY(cudaFuncSetAttribute(mlp_grad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kMlpGradSmem)));
        done[dev & 63].store(true, std::memory_order_release);
    }
    return TASEP_OK;
}

tasep_status mlp_rows(tasep_mlp *m, int rows) {
    if (rows <= m->grow_cap) return TASEP_OK;
    cudaFree(m->grows);
    cudaFree(m->loss);
    m->grows = nullptr;
    m->loss = nullptr;
    CU_TRY(cudaMalloc(&m->grows, sizeof(float) * size_t(rows) * kMlpParams));
    CU_TRY(cudaMalloc(&m->loss, sizeof(float) * rows));
    m->grow_cap = rows;
    return TASEP_OK;
}

// Reads and clears the kernels' error flag (after a synchronisation).
tasep_status mlp_check(tasep_mlp *m) {
    int e = 0;
    CU_TRY(cudaMemcpy(&e, m->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (!e) return TASEP_OK;
    CU_TRY(cudaMemset(m->err, 0, sizeof(int)));
    return fail(TASEP_ERR_TIMEOUT, "a tensor-core wait of the network kernels expired");
}

// gradient of the loss over n device-resident samples into m->gsum; mean
// loss into *loss_host (if not NULL)
tasep_status mlp_grad_device(tasep_mlp *m, const float *xd, const float *td, int n, const float *ow, float *loss_host) {
    const int rows = (n + kMlpTile - 1) / kMlpTile;
    tasep_status s = mlp_rows(m, rows);
    if (s) return s;
    mlp_grad_kernel<<<rows, kMlpThreads, kMlpGradSmem>>>(m->w, xd, td, n, ow[0], ow[1], m->grows, m->loss, m->err);
    CU_TRY(cudaGetLastError());
    mlp_reduce_kernel<<<(kMlpParams + 255) / 256, 256>>>(m->grows, rows, m->gsum);
    CU_TRY(cudaGetLastError());
    if (loss_host) {
        std::vector<float> l(rows);
        CU_TRY(cudaMemcpy(l.data(), m->loss, sizeof(float) * rows, cudaMemcpyDeviceToHost));
        float tot = 0.f;
        for (float v : l) tot += v;
        *loss_host = tot;
        return mlp_check(m);
    }
    return TASEP_OK;
}

}  // namespace

extern "C" {

tasep_status tasep_mlp_create(int device, uint64_t seed, tasep_mlp **out) {
    if (!out) return fail(TASEP_ERR_INVALID, "null argument");
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TASEP_ERR_NODEV, "no CUDA device");
    }
    int dev = device;
    if (dev < 0) CU_TRY(cudaGetDevice(&dev));
    CU_TRY(cudaSetDevice(dev));
    tasep_mlp *m = new tasep_mlp();
    m->device = dev;
    bool ok = cudaMalloc(&m->master, sizeof(float) * kMlpParams) == cudaSuccess &&
              cudaMalloc(&m->m1, sizeof(float) * kMlpParams) == cudaSuccess &&
              cudaMalloc(&m->m2, sizeof(float) * kMlpParams) == cudaSuccess &&
              cudaMalloc(&m->gsum, sizeof(float) * kMlpParams) == cudaSuccess &&
              cudaMalloc(&m->w, sizeof(__nv_bfloat16) * kMlpParams) == cudaSuccess &&
              cudaMalloc(&m->err, sizeof(int)) == cudaSuccess && cudaMemset(m->err, 0, sizeof(int)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        tasep_mlp_destroy(m);
        return fail(TASEP_ERR_NOMEM, "network allocation failed");
    }
    // Glorot-uniform weights, zero biases
    std::vector<float> p(kMlpParams, 0.f);
    uint64_t s = seed;
    auto fill = [&](int off, int fan_out, int fan_in) {
        const double a = std::sqrt(6.0 / double(fan_in + fan_out));
        for (int i = 0; i < fan_out * fan_in; ++i) p[off + i] = float((2.0 * mlp_unif(s) - 1.0) * a);
    };
    fill(kMlpW1, kMlpHid, kMlpIn);
    fill(kMlpW2, kMlpHid, kMlpHid);
    fill(kMlpW3, kMlpHid, kMlpHid);
    fill(kMlpW4, kMlpOut, kMlpHid);
    *out = m;
    return tasep_mlp_set_params(m, p.data());
}

tasep_status tasep_mlp_destroy(tasep_mlp *m) {
    if (!m) return TASEP_OK;
    cudaSetDevice(m->device);
    cudaFree(m->master);
    cudaFree(m->m1);
    cudaFree(m->m2);
    cudaFree(m->gsum);
    cudaFree(m->grows);
    cudaFree(m->loss);
    cudaFree(m->w);
    cudaFree(m->err);
    delete m;
    return TASEP_OK;
}

tasep_status tasep_mlp_set_params(tasep_mlp *m, const float *params) {
    if (!m || !params) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaMemcpy(m->master, params, sizeof(float) * kMlpParams, cudaMemcpyHostToDevice));
    CU_TRY(cudaMemset(m->m1, 0, sizeof(float) * kMlpParams));
    CU_TRY(cudaMemset(m->m2, 0, sizeof(float) * kMlpParams));
    mlp_to_bf16_kernel<<<(kMlpParams + 255) / 256, 256>>>(m->master, m->w);
    CU_TRY(cudaGetLastError());
    CU_TRY(cudaDeviceSynchronize());
    m->adam_t = 0;
    return TASEP_OK;
}

tasep_status tasep_mlp_get_params(tasep_mlp *m, float *params) {
    if (!m || !params) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaMemcpy(params, m->master, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost));
    return TASEP_OK;
}

tasep_status tasep_mlp_loss_grad(tasep_mlp *m, const float *x, const float *t, int n, const float *out_weights,
                                 float *loss, float *grad) {
    if (!m || !x || !t || n < 1 || !out_weights) return fail(TASEP_ERR_INVALID, "bad argument");
    CU_TRY(cudaSetDevice(m->device));
    tasep_status s = mlp_configure();
    if (s) return s;
    float *xd = nullptr, *td = nullptr;
    CU_TRY(cudaMalloc(&xd, sizeof(float) * size_t(n) * kMlpIn));
    CU_TRY(cudaMalloc(&td, sizeof(float) * size_t(n) * kMlpOut));
    CU_TRY(cudaMemcpy(xd, x, sizeof(float) * size_t(n) * kMlpIn, cudaMemcpyHostToDevice));
    CU_TRY(cudaMemcpy(td, t, sizeof(float) * size_t(n) * kMlpOut, cudaMemcpyHostToDevice));
    s = mlp_grad_device(m, xd, td, n, out_weights, loss);
    if (!s && cudaDeviceSynchronize() != cudaSuccess) s = fail(TASEP_ERR_CUDA, "gradient failed");
    if (!s) s = mlp_check(m);
    if (!s && grad) {
        cudaError_t e = cudaMemcpy(grad, m->gsum, sizeof(float) * kMlpParams, cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) s = fail(TASEP_ERR_CUDA, "%s", cudaGetErrorString(e));
    }
    cudaFree(xd);
    cudaFree(td);
    return s;
}

tasep_status tasep_mlp_train(tasep_mlp *m, const float *x, const float *t, int n, const float *out_weights,
                             int epochs, int batch, float lr, uint64_t seed, float *loss_per_epoch) {
    if (!m || !x || !t || n < 1 || !out_weights || epochs < 0 || batch < 1) return fail(TASEP_ERR_INVALID, "bad argument");
    CU_TRY(cudaSetDevice(m->device));
    tasep_status s = mlp_configure();
    if (s) return s;
    std::vector<float> xs(size_t(n) * kMlpIn), ts(size_t(n) * kMlpOut);
    std::vector<int> perm(n);
    for (int i = 0; i < n; ++i) perm[i] = i;
    float *xd = nullptr, *td = nullptr;
    CU_TRY(cudaMalloc(&xd, sizeof(float) * size_t(n) * kMlpIn));
    CU_TRY(cudaMalloc(&td, sizeof(float) * size_t(n) * kMlpOut));
    uint64_t rs = seed;
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int ep = 0; ep < epochs && !s; ++ep) {
        for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[int(mlp_rng(rs) % uint64_t(i + 1))]);
        for (int i = 0; i < n; ++i) {
            memcpy(&xs[size_t(i) * kMlpIn], &x[size_t(perm[i]) * kMlpIn], sizeof(float) * kMlpIn);
            memcpy(&ts[size_t(i) * kMlpOut], &t[size_t(perm[i]) * kMlpOut], sizeof(float) * kMlpOut);
        }
        if (cudaMemcpy(xd, xs.data(), sizeof(float) * xs.size(), cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(td, ts.data(), sizeof(float) * ts.size(), cudaMemcpyHostToDevice) != cudaSuccess) {
            s = fail(TASEP_ERR_CUDA, "upload");
            break;
        }
        double ep_loss = 0.0;
        for (int b0 = 0; b0 < n && !s; b0 += batch) {
            const int nb = std::min(batch, n - b0);
            float l = 0.f;
            s = mlp_grad_device(m, xd + size_t(b0) * kMlpIn, td + size_t(b0) * kMlpOut, nb, out_weights,
                                loss_per_epoch ? &l : nullptr);
            if (s) break;
            ep_loss += double(l) * nb;
            m->adam_t += 1;
            const float c1 = 1.f - std::pow(b1, float(m->adam_t)), c2 = 1.f - std::pow(b2, float(m->adam_t));
            mlp_adam_kernel<<<(kMlpParams + 255) / 256, 256>>>(m->master, m->w, m->m1, m->m2, m->gsum, lr, b1, b2,
                                                              eps, c1, c2);
            if (cudaGetLastError() != cudaSuccess) s = fail(TASEP_ERR_CUDA, "adam launch");
        }
        if (loss_per_epoch) loss_per_epoch[ep] = float(ep_loss / n);
    }
    cudaFree(xd);
    cudaFree(td);
    if (!s && cudaDeviceSynchronize() != cudaSuccess) s = fail(TASEP_ERR_CUDA, "training failed");
    if (!s) s = mlp_check(m);
    return s;
}

tasep_status tasep_mlp_predict(tasep_mlp *m, const float *x, int n, float *y) {
    if (!m || !x || !y || n < 1) return fail(TASEP_ERR_INVALID, "bad argument");
    CU_TRY(cudaSetDevice(m->device));
    tasep_status s = mlp_configure();
    if (s) return s;
    float *xd = nullptr, *yd = nullptr;
    CU_TRY(cudaMalloc(&xd, sizeof(float) * size_t(n) * kMlpIn));
    CU_TRY(cudaMalloc(&yd, sizeof(float) * size_t(n) * kMlpOut));
    cudaError_t e = cudaMemcpy(xd, x, sizeof(float) * size_t(n) * kMlpIn, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        const int grid = std::min((n + kMlpTile - 1) / kMlpTile, 1024);
        mlp_forward_kernel<<<grid, kMlpThreads, kMlpForwardSmem>>>(m->w, xd, yd, n, m->err);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(y, yd, sizeof(float) * size_t(n) * kMlpOut, cudaMemcpyDeviceToHost);
    cudaFree(xd);
    cudaFree(yd);
    if (e != cudaSuccess) return fail(TASEP_ERR_CUDA, "prediction: %s", cudaGetErrorString(e));
    return mlp_check(m);
}

tasep_status tasep_mean_field_profile(int n, int count, int steps, const double *rates, double *rho) {
    if (n < 1 || n > TASEP_MAX_N || count < 0 || steps < 0 || (count > 0 && (!rates || !rho)))
        return fail(TASEP_ERR_INVALID, "mean-field profile: n=%d count=%d steps=%d", n, count, steps);
    double J[TASEP_MAX_N + 1];
    for (int c = 0; c < count; ++c) {
        const double *r = rates + size_t(c) * (n + 1);
        double *x = rho + size_t(c) * n;
        double rmax = r[0];
        for (int i = 1; i <= n; ++i) rmax = r[i] > rmax ? r[i] : rmax;
        const double dt = 0.25 / rmax;
        for (int i = 0; i < n; ++i) x[i] = 0.5;
        for (int s = 0; s < steps; ++s) {
            J[0] = r[0] * (1.0 - x[0]);
            for (int i = 1; i < n; ++i) J[i] = r[i] * x[i - 1] * (1.0 - x[i]);
            J[n] = r[n] * x[n - 1];
            for (int i = 0; i < n; ++i) x[i] += dt * (J[i] - J[i + 1]);
        }
        for (int i = 0; i < n; ++i) x[i] = x[i] < 1e-6 ? 1e-6 : (x[i] > 1.0 - 1e-6 ? 1.0 - 1e-6 : x[i]);
    }
    return TASEP_OK;
}

tasep_status tasep_meq_init_pair_markov(tasep_meq *m, const double *rho, const double *cov) {
    if (!valid_handle(m) || !rho || (!cov && m->n > 1)) return fail(TASEP_ERR_INVALID, "null argument");
    const int n = m->n;
    const double eps = 1e-12;
    for (int j = 0; j < n; ++j)
        if (!(rho[j] > eps && rho[j] < 1.0 - eps))
            return fail(TASEP_ERR_INVALID, "infeasible prediction: density %g at site %d", rho[j], j);
    double p0[2] = {1.0 - rho[0], rho[0]};
    std::vector<double> T(4 * size_t(n > 1 ? n - 1 : 1));
    for (int j = 0; j + 1 < n; ++j) {
        const double a = rho[j], b = rho[j + 1];
        const double lo = std::max(0.0, a + b - 1.0), hi = std::min(a, b);
        double p11 = cov[j] + a * b;
        const double margin = 1e-9 * (hi - lo);
        p11 = std::min(std::max(p11, lo + margin), hi - margin);
        const double p10 = a - p11, p01 = b - p11, p00 = 1.0 - a - b + p11;
        T[4 * j + 0] = p00 / (1.0 - a);
        T[4 * j + 1] = p01 / (1.0 - a);
        T[4 * j + 2] = p10 / a;
        T[4 * j + 3] = p11 / a;
    }
    CU_TRY(cudaSetDevice(m->device));
    double *d = nullptr;
    CU_TRY(cudaMalloc(&d, sizeof(double) * (2 + T.size())));
    cudaError_t e = cudaMemcpy(d, p0, sizeof p0, cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d + 2, T.data(), sizeof(double) * T.size(), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        pair_markov_kernel<<<std::max(1, m->nsm * 8), 256, 0, m->stream>>>(n, d, d + 2, m->X[0]);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(TASEP_ERR_CUDA, "pair-Markov measure: %s", cudaGetErrorString(e));
    m->cur = 0;
    m->state_set = true;
    return TASEP_OK;
}

}  // extern "C"
