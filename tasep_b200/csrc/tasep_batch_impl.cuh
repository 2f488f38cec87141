// tasep_batch_impl.cuh - C ABI of the batched parameter sweep (tasep_batch_*,
// include/tasep.h).  Included at the end of tasep_api.cu (one translation
// unit, so the error helpers are shared).
#pragma once

#include "meq_batch.cuh"

namespace {

// Per-bit densities of each system: one CTA per system, fixed-order sums.
__global__ void batch_density_kernel(int n, const double *x, double *rho) {
    const unsigned long long N = 1ull << n;
    const double *xs = x + blockIdx.x * N;
    double acc[24];
    for (int b = 0; b < n; ++b) acc[b] = 0.0;
    for (unsigned long long i = threadIdx.x; i < N; i += blockDim.x) {
        const double v = xs[i];
        for (int b = 0; b < n; ++b)
            if ((i >> b) & 1) acc[b] += v;
    }
    __shared__ double red[8][24];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int b = 0; b < n; ++b) {
        const double w = warp_sum(acc[b]);
        if (lane == 0) red[warp][b] = w;
    }
    __syncthreads();
    if (threadIdx.x < n) {
        double s = 0.0;
        for (int w = 0; w < int(blockDim.x / 32); ++w) s += red[w][threadIdx.x];
        rho[blockIdx.x * n + threadIdx.x] = s;
    }
}

template <int S, typename E> tasep_status configure_batch() {
    CU_TRY(cudaFuncSetAttribute(meq_batch_kernel<S, E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                batch_smem_bytes<S, E>()));
    return TASEP_OK;
}

// Sets the shared-memory limit of every stage kernel (before any capture).
template <typename E> tasep_status configure_batch_all() {
    tasep_status s;
    if ((s = configure_batch<ST_H1, E>()) || (s = configure_batch<ST_H2, E>()) || (s = configure_batch<ST_H3, E>()) ||
        (s = configure_batch<ST_H4, E>()))
        return s;
    return TASEP_OK;
}

template <int S, typename E> tasep_status launch_batch(const BatchParams &p, int grid, cudaStream_t st) {
    meq_batch_kernel<S, E><<<grid, kTileThreads, batch_smem_bytes<S, E>(), st>>>(p);
    CU_TRY(cudaGetLastError());
    return TASEP_OK;
}

}  // namespace

struct tasep_batch {
    int n = 0, nsys = 0, precision = 0, device = 0, nsm = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    unsigned long long N = 0;
    double *X = nullptr;
    void *V[3] = {nullptr, nullptr, nullptr};
    double *rates = nullptr;
    double *dtab_d = nullptr;
    float *dtab_f = nullptr;
    double *partials = nullptr;
    unsigned *counters = nullptr;
    BatchExit *ex = nullptr;
    int *active = nullptr, *error = nullptr;
    int *list = nullptr, *count = nullptr;
    int *active_host = nullptr;
    bool rates_set = false, state_set = false;
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    int graph_steps = 0;
    double graph_key[4] = {0, 0, 0, 0};
};

namespace {

template <typename E> tasep_status batch_enqueue_step_t(tasep_batch *b, const BatchParams &base, int grid) {
    BatchParams p = base;
    tasep_status s;
    const double h = base.h;
    p.g = b->X; p.out = b->V[0]; p.dtab = b->dtab_d; p.hc = 0.0;
    if ((s = launch_batch<ST_H1, E>(p, grid, b->stream))) return s;
    p.g = b->V[0]; p.out = b->V[1]; p.hc = h / 4;
    p.dtab = (sizeof(E) == 4) ? static_cast<const void *>(b->dtab_f) : static_cast<const void *>(b->dtab_d);
    if ((s = launch_batch<ST_H2, E>(p, grid, b->stream))) return s;
    p.g = b->V[1]; p.s0 = b->V[0]; p.out = b->V[2]; p.hc = h / 3;
    if ((s = launch_batch<ST_H3, E>(p, grid, b->stream))) return s;
    p.g = b->V[2]; p.s0 = b->V[0]; p.s1 = b->X; p.out = b->X; p.hc = h / 2;
    if ((s = launch_batch<ST_H4, E>(p, grid, b->stream))) return s;
    // systems that converged in this step leave the running list
    batch_compact_kernel<<<1, 1024, 0, b->stream>>>(b->ex, b->nsys, b->list, b->count);
    CU_TRY(cudaGetLastError());
    return TASEP_OK;
}

tasep_status batch_enqueue_step(tasep_batch *b, const BatchParams &base, int grid) {
    return b->precision == TASEP_PRECISION_MIXED ? batch_enqueue_step_t<float>(b, base, grid)
                                                 : batch_enqueue_step_t<double>(b, base, grid);
}

void batch_drop_graphs(tasep_batch *b) {
    for (auto &gx : b->graph)
        if (gx) {
            cudaGraphExecDestroy(gx);
            gx = nullptr;
        }
}

// Captures `steps` steps with the given schedule into a graph.
tasep_status batch_capture(tasep_batch *b, const BatchParams &base, int sched, int steps) {
    BatchParams p = base;
    p.sys_major = sched;
    const int grid = b->nsm;
    tasep_status cs = b->precision == TASEP_PRECISION_MIXED ? configure_batch_all<float>() : configure_batch_all<double>();
    if (cs) return cs;
    cudaGraph_t gr = nullptr;
    CU_TRY(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
    tasep_status s = TASEP_OK;
    for (int i = 0; i < steps && !s; ++i) s = batch_enqueue_step(b, p, grid);
    cudaError_t e = cudaStreamEndCapture(b->stream, &gr);
    if (s) {
        if (gr) cudaGraphDestroy(gr);
        return s;
    }
    if (e != cudaSuccess) return fail(TASEP_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
    e = cudaGraphInstantiate(&b->graph[sched], gr, 0);
    cudaGraphDestroy(gr);
    if (e != cudaSuccess) return fail(TASEP_ERR_CUDA, "graph instantiation: %s", cudaGetErrorString(e));
    return TASEP_OK;
}

}  // namespace

extern "C" {

tasep_status tasep_batch_create(int n, int nsys, int precision, int device, void *stream, tasep_batch **out) {
    if (!out) return fail(TASEP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n <= kTileBits || n > 24) return fail(TASEP_ERR_INVALID, "batched systems need %d < n <= 24", kTileBits);
    if (nsys < 1) return fail(TASEP_ERR_INVALID, "nsys=%d", nsys);
    if (precision != TASEP_PRECISION_FP64 && precision != TASEP_PRECISION_MIXED)
        return fail(TASEP_ERR_INVALID, "unknown precision %d", precision);
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TASEP_ERR_NODEV, "no CUDA device");
    }
    int dev = device;
    if (dev < 0) CU_TRY(cudaGetDevice(&dev));
    CU_TRY(cudaSetDevice(dev));
    tasep_batch *b = new tasep_batch();
    b->n = n;
    b->nsys = nsys;
    b->precision = precision;
    b->device = dev;
    b->N = 1ull << n;
    cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, dev);
    auto bail = [&](tasep_status s) {
        tasep_batch_destroy(b);
        return s;
    };
    if (stream) {
        b->stream = static_cast<cudaStream_t>(stream);
    } else {
        if (cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(TASEP_ERR_CUDA, "stream creation failed"));
        b->own_stream = true;
    }
    const size_t tot = size_t(nsys) * b->N;
    const size_t sv = precision == TASEP_PRECISION_MIXED ? sizeof(float) : sizeof(double);
    const size_t tps = b->N >> kTileBits;
    bool ok = cudaMalloc(&b->X, tot * sizeof(double)) == cudaSuccess;
    for (int i = 0; i < 3 && ok; ++i) ok = cudaMalloc(&b->V[i], tot * sv) == cudaSuccess;
    ok = ok && cudaMalloc(&b->rates, sizeof(double) * nsys * (n + 1)) == cudaSuccess &&
         cudaMalloc(&b->dtab_d, sizeof(double) * nsys * 2 * kTile) == cudaSuccess &&
         cudaMalloc(&b->dtab_f, sizeof(float) * nsys * 2 * kTile) == cudaSuccess &&
         cudaMalloc(&b->partials, sizeof(double) * nsys * tps * kConsumerWarps) == cudaSuccess &&
         cudaMalloc(&b->counters, sizeof(unsigned) * nsys) == cudaSuccess &&
         cudaMalloc(&b->ex, sizeof(BatchExit) * nsys) == cudaSuccess &&
         cudaMalloc(&b->active, sizeof(int)) == cudaSuccess && cudaMalloc(&b->error, sizeof(int)) == cudaSuccess &&
         cudaMalloc(&b->list, sizeof(int) * nsys) == cudaSuccess && cudaMalloc(&b->count, sizeof(int)) == cudaSuccess &&
         cudaMallocHost(&b->active_host, 2 * sizeof(int)) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        return bail(fail(TASEP_ERR_NOMEM, "not enough device memory for %d systems of n=%d", nsys, n));
    }
    *out = b;
    return TASEP_OK;
}

tasep_status tasep_batch_destroy(tasep_batch *b) {
    if (!b) return TASEP_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_drop_graphs(b);
    cudaFree(b->X);
    for (auto &v : b->V) cudaFree(v);
    cudaFree(b->rates);
    cudaFree(b->dtab_d);
    cudaFree(b->dtab_f);
    cudaFree(b->partials);
    cudaFree(b->counters);
    cudaFree(b->ex);
    cudaFree(b->active);
    cudaFree(b->error);
    cudaFree(b->list);
    cudaFree(b->count);
    if (b->active_host) cudaFreeHost(b->active_host);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return TASEP_OK;
}

tasep_status tasep_batch_set_rates(tasep_batch *b, const double *rates) {
    if (!b || !rates) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(b->device));
    CU_TRY(cudaMemcpy(b->rates, rates, sizeof(double) * b->nsys * (b->n + 1), cudaMemcpyHostToDevice));
    batch_setup_kernel<double><<<256, 256, 0, b->stream>>>(b->n, b->nsys, b->rates, b->dtab_d);
    CU_TRY(cudaGetLastError());
    batch_setup_kernel<float><<<256, 256, 0, b->stream>>>(b->n, b->nsys, b->rates, b->dtab_f);
    CU_TRY(cudaGetLastError());
    CU_TRY(cudaStreamSynchronize(b->stream));
    b->rates_set = true;
    return TASEP_OK;
}

tasep_status tasep_batch_init(tasep_batch *b, int kind) {
    if (!b) return fail(TASEP_ERR_INVALID, "null handle");
    if (kind != TASEP_INIT_EMPTY && kind != TASEP_INIT_UNIFORM) return fail(TASEP_ERR_INVALID, "unknown initial state");
    std::vector<double> sys(b->N, kind == TASEP_INIT_EMPTY ? 0.0 : 1.0 / double(b->N));
    if (kind == TASEP_INIT_EMPTY) sys[0] = 1.0;
    CU_TRY(cudaSetDevice(b->device));
    for (int s = 0; s < b->nsys; ++s)
        CU_TRY(cudaMemcpy(b->X + size_t(s) * b->N, sys.data(), sizeof(double) * b->N, cudaMemcpyHostToDevice));
    b->state_set = true;
    return TASEP_OK;
}

tasep_status tasep_batch_load(tasep_batch *b, const double *host_x) {
    if (!b || !host_x) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(b->device));
    CU_TRY(cudaMemcpy(b->X, host_x, sizeof(double) * b->N * b->nsys, cudaMemcpyHostToDevice));
    b->state_set = true;
    return TASEP_OK;
}

tasep_status tasep_batch_run(tasep_batch *b, const tasep_run_config *rc, int schedule, tasep_run_result *res,
                             int *schedule_used) {
    if (!b || !rc) return fail(TASEP_ERR_INVALID, "null argument");
    if (!b->rates_set || !b->state_set) return fail(TASEP_ERR_INVALID, "rates or initial state not set");
    if (schedule < -1 || schedule > 1) return fail(TASEP_ERR_INVALID, "schedule %d", schedule);
    CU_TRY(cudaSetDevice(b->device));
    BatchParams base;
    memset(&base, 0, sizeof base);
    base.n = b->n;
    base.tps_bits = b->n - kTileBits;
    base.nsys = b->nsys;
    base.h = rc->h;
    base.rates = b->rates;
    base.partials = b->partials;
    base.counters = b->counters;
    base.ex = b->ex;
    base.active = b->active;
    base.list = b->list;
    base.count = b->count;
    base.error = b->error;
    base.thresh = rc->stop_tol * rc->h;
    base.stop_count = rc->stop_count;
    base.exit_rule = rc->exit_rule;
    base.max_steps = rc->steps;
    const int K = 16;  // steps per graph replay
    const double key[4] = {rc->h, base.thresh, double(rc->stop_count) + 1e6 * rc->exit_rule, double(rc->steps)};
    if (b->graph_steps != K || memcmp(key, b->graph_key, sizeof key) != 0) {
        batch_drop_graphs(b);
        tasep_status s;
        for (int sc = 0; sc < 2; ++sc)
            if ((s = batch_capture(b, base, sc, K))) return s;
        b->graph_steps = K;
        memcpy(b->graph_key, key, sizeof key);
    }
    CU_TRY(cudaMemsetAsync(b->ex, 0, sizeof(BatchExit) * b->nsys, b->stream));
    CU_TRY(cudaMemsetAsync(b->counters, 0, sizeof(unsigned) * b->nsys, b->stream));
    CU_TRY(cudaMemsetAsync(b->error, 0, sizeof(int), b->stream));
    b->active_host[0] = b->nsys;
    CU_TRY(cudaMemcpyAsync(b->active, b->active_host, sizeof(int), cudaMemcpyHostToDevice, b->stream));
    batch_compact_kernel<<<1, 1024, 0, b->stream>>>(b->ex, b->nsys, b->list, b->count);
    CU_TRY(cudaGetLastError());
    cudaEvent_t e0, e1;
    CU_TRY(cudaEventCreate(&e0));
    CU_TRY(cudaEventCreate(&e1));
    // autotuner: time one replay of each schedule at the start and again each
    // time the number of running systems has halved (the best way to spread
    // tiles over the SMs changes as systems retire)
    int sched = schedule < 0 ? 0 : schedule;
    int tuned_at = schedule < 0 ? 2 * b->nsys + 2 : -1;  // running count at the last tuning
    unsigned long long launched = 0;
    tasep_status st = TASEP_OK;
    while (launched < rc->steps) {
        const int active = b->active_host[0];
        const bool tune = schedule < 0 && 2 * active <= tuned_at;
        if (tune) {
            float best = 1e30f;
            int best_s = sched;
            for (int sc = 0; sc < 2 && launched < rc->steps; ++sc) {
                cudaEventRecord(e0, b->stream);
                if (cudaGraphLaunch(b->graph[sc], b->stream) != cudaSuccess) { st = fail(TASEP_ERR_CUDA, "graph launch"); break; }
                cudaEventRecord(e1, b->stream);
                launched += K;
                cudaEventSynchronize(e1);
                float ms = 0.f;
                cudaEventElapsedTime(&ms, e0, e1);
                if (ms < best) { best = ms; best_s = sc; }
            }
            if (st) break;
            sched = best_s;
            tuned_at = active;
        } else {
            if (cudaGraphLaunch(b->graph[sched], b->stream) != cudaSuccess) { st = fail(TASEP_ERR_CUDA, "graph launch"); break; }
            launched += K;
        }
        CU_TRY(cudaMemcpyAsync(b->active_host, b->active, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        CU_TRY(cudaMemcpyAsync(b->active_host + 1, b->error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
        CU_TRY(cudaStreamSynchronize(b->stream));
        if (b->active_host[1]) { st = fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired"); break; }
        if (b->active_host[0] <= 0) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (st) return st;
    if (schedule_used) *schedule_used = sched;
    if (res) {
        std::vector<BatchExit> ex(b->nsys);
        CU_TRY(cudaMemcpy(ex.data(), b->ex, sizeof(BatchExit) * b->nsys, cudaMemcpyDeviceToHost));
        for (int s = 0; s < b->nsys; ++s) {
            res[s].steps_done = ex[s].steps_done;
            res[s].steps_at_stop = ex[s].steps_at_stop;
            res[s].early_stop = ex[s].early_stop;
            res[s].converged = ex[s].converged;
            res[s].last_checksum = ex[s].last_checksum;
            double t = rc->t0;
            for (unsigned long long k = 0; k < ex[s].steps_done; ++k) t += rc->h;
            res[s].t_end = t;
        }
    }
    return TASEP_OK;
}

tasep_status tasep_batch_store(const tasep_batch *b, int sys, double *host_x) {
    if (!b || !host_x || sys < 0 || sys >= b->nsys) return fail(TASEP_ERR_INVALID, "bad argument");
    CU_TRY(cudaSetDevice(b->device));
    CU_TRY(cudaMemcpy(host_x, b->X + size_t(sys) * b->N, sizeof(double) * b->N, cudaMemcpyDeviceToHost));
    return TASEP_OK;
}

tasep_status tasep_batch_densities(tasep_batch *b, double *rho) {
    if (!b || !rho) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(b->device));
    double *d = nullptr;
    CU_TRY(cudaMalloc(&d, sizeof(double) * b->nsys * b->n));
    batch_density_kernel<<<b->nsys, 256, 0, b->stream>>>(b->n, b->X, d);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaMemcpyAsync(rho, d, sizeof(double) * b->nsys * b->n, cudaMemcpyDeviceToHost, b->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    cudaFree(d);
    if (e != cudaSuccess) return fail(TASEP_ERR_CUDA, "densities: %s", cudaGetErrorString(e));
    return TASEP_OK;
}

}  // extern "C"
