// tasep_batch_impl.cuh - C ABI of the batched parameter sweep (tasep_batch_*,
// include/tasep.h).  Included at the end of tasep_api.cu (one translation
// unit, so the error helpers are shared).
#pragma once

#include "meq_batch.cuh"
#include "meq_cluster.cuh"

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
    CU_TRY(launch_pdl(meq_batch_kernel<S, E>, dim3(grid), dim3(kTileThreads), size_t(batch_smem_bytes<S, E>()), st, p));
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
    // last run: schedule, states per CTA and CTAs per system
    int last_schedule = -1, last_states_per_cta = 0, last_ctas_per_system = 0;
};

namespace {

template <typename E> tasep_status batch_enqueue_step_t(tasep_batch *b, const BatchParams &base, int grid) {
    BatchParams p = base;
    tasep_status s;
    const double h = base.h;
    // classical RK4 in factored form, as the single-system sweep (Rk4Factors)
    static const Rk4Factors F = rk4_factors();
    p.g = b->X; p.out = b->V[0]; p.hc = 0.0;
    if ((s = launch_batch<ST_H1, E>(p, grid, b->stream))) return s;
    p.g = b->V[0]; p.out = b->V[1]; p.hc = h; p.cx = -F.r;
    if ((s = launch_batch<ST_H2, E>(p, grid, b->stream))) return s;
    p.g = b->V[1]; p.out = b->V[2]; p.hc = h; p.cx = F.p;
    if ((s = launch_batch<ST_H3, E>(p, grid, b->stream))) return s;
    p.g = b->V[2]; p.s0 = b->V[1]; p.s1 = b->X; p.out = b->X; p.hc = h / 24; p.cx = F.q / 24;
    if ((s = launch_batch<ST_H4, E>(p, grid, b->stream))) return s;
    // systems that converged in this step leave the running list
    CU_TRY(launch_pdl(batch_compact_kernel, dim3(1), dim3(1024), 0, b->stream, b->ex, b->nsys, b->list, b->count));
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

// ---- cluster-resident engine (schedule 2, n <= kClMaxN) ----

// The cluster kernel is instantiated for 2, 4 and 8 pairs per thread (2^11,
// 2^12, 2^13 states per CTA).
template <typename E, int NP> tasep_status cluster_config_np(int cs_log2, cudaLaunchConfig_t &cfg,
                                                             cudaLaunchAttribute *at, int nclusters, cudaStream_t st) {
    const int sbits = 10 + (NP == 8 ? 3 : NP == 4 ? 2 : 1);
    const size_t smem = ClLayout<E>::bytes(sbits);
    CU_TRY(cudaFuncSetAttribute(meq_cluster_kernel<E, NP>, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    if ((1 << cs_log2) > 8)
        CU_TRY(cudaFuncSetAttribute(meq_cluster_kernel<E, NP>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    memset(&cfg, 0, sizeof cfg);
    cfg.gridDim = dim3(unsigned(nclusters) << cs_log2);
    cfg.blockDim = dim3(kClThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    at[0].id = cudaLaunchAttributeClusterDimension;
    at[0].val.clusterDim.x = 1u << cs_log2;
    at[0].val.clusterDim.y = 1;
    at[0].val.clusterDim.z = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return TASEP_OK;
}

template <typename E, int NP> tasep_status cluster_capacity_np(int cs_log2, int *count) {
    *count = 0;
    if (ClLayout<E>::bytes(10 + (NP == 8 ? 3 : NP == 4 ? 2 : 1)) > size_t(kSmemMax)) return TASEP_OK;
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    tasep_status s = cluster_config_np<E, NP>(cs_log2, cfg, at, 1, nullptr);
    if (s) return s;
    int num = 0;
    if (cudaOccupancyMaxActiveClusters(&num, meq_cluster_kernel<E, NP>, &cfg) != cudaSuccess) {
        cudaGetLastError();  // shape not launchable on this device
        num = 0;
    }
    *count = num;
    return TASEP_OK;
}

template <typename E, int NP> tasep_status cluster_launch_np(const ClusterParams &p, int nclusters, cudaStream_t st) {
    cudaLaunchConfig_t cfg;
    cudaLaunchAttribute at[1];
    tasep_status s = cluster_config_np<E, NP>(p.cs_log2, cfg, at, nclusters, st);
    if (s) return s;
    CU_TRY(cudaLaunchKernelEx(&cfg, meq_cluster_kernel<E, NP>, p));
    return TASEP_OK;
}

template <typename E> tasep_status cluster_capacity(int cs_log2, int sbits, int *count) {
    switch (sbits) {
    case 13: return cluster_capacity_np<E, 8>(cs_log2, count);
    case 12: return cluster_capacity_np<E, 4>(cs_log2, count);
    case 11: return cluster_capacity_np<E, 2>(cs_log2, count);
    default: *count = 0; return TASEP_OK;
    }
}

template <typename E> tasep_status cluster_launch(const ClusterParams &p, int nclusters, cudaStream_t st) {
    switch (p.sbits) {
    case 13: return cluster_launch_np<E, 8>(p, nclusters, st);
    case 12: return cluster_launch_np<E, 4>(p, nclusters, st);
    case 11: return cluster_launch_np<E, 2>(p, nclusters, st);
    default: return fail(TASEP_ERR_INVALID, "no cluster kernel for 2^%d states per CTA", p.sbits);
    }
}

tasep_status cluster_capacity_p(const tasep_batch *b, int cs_log2, int sbits, int *count) {
    return b->precision == TASEP_PRECISION_MIXED ? cluster_capacity<float>(cs_log2, sbits, count)
                                                 : cluster_capacity<double>(cs_log2, sbits, count);
}
tasep_status cluster_launch_p(const tasep_batch *b, const ClusterParams &p, int nclusters) {
    return b->precision == TASEP_PRECISION_MIXED ? cluster_launch<float>(p, nclusters, b->stream)
                                                 : cluster_launch<double>(p, nclusters, b->stream);
}

bool cluster_eligible(const tasep_batch *b) { return b->n >= kTileBits + 1 && b->n <= kClMaxN; }

// Every system on its own cluster until its exit rule.  With schedule < 0 the
// autotuner times the feasible shapes - 2^11, 2^12 or 2^13 states per CTA,
// i.e. 2^(n-11) .. 2^(n-13) CTAs per system - on a short run of copies of
// the first systems and keeps the fastest.
tasep_status batch_run_cluster(tasep_batch *b, const tasep_run_config *rc, int schedule, tasep_run_result *res,
                               int *schedule_used) {
    const int n = b->n;
    struct Shape { int cs_log2, sbits, clusters; };
    std::vector<Shape> shapes;
    for (int sb = 13; sb >= 11; --sb) {
        const int cl = n - sb;  // log2 CTAs per system
        if (sb > n || cl > 4) continue;
        int cap = 0;
        tasep_status s = cluster_capacity_p(b, cl, sb, &cap);
        if (s) return s;
        if (cap > 0) shapes.push_back({cl, sb, cap});
    }
    if (shapes.empty()) return fail(TASEP_ERR_UNSUPPORTED, "no cluster shape fits n=%d on this device", n);
    ClusterParams base;
    memset(&base, 0, sizeof base);
    base.n = n;
    base.nsys = b->nsys;
    base.h = rc->h;
    base.rates = b->rates;
    base.ex = b->ex;
    base.queue = b->counters;
    base.error = b->error;
    base.thresh = rc->stop_tol * rc->h;
    base.stop_count = rc->stop_count;
    base.exit_rule = rc->exit_rule;
    size_t best = 0;
    if (shapes.size() > 1 && schedule < 0) {
        // probe: copies of the first systems (the stage buffers are free here), 32 steps each
        const size_t vec_bytes = (b->precision == TASEP_PRECISION_MIXED ? sizeof(float) : sizeof(double)) * b->N;
        const int cap = int(std::min<size_t>(size_t(b->nsys), (vec_bytes * b->nsys) / (sizeof(double) * b->N)));
        cudaEvent_t e0, e1;
        CU_TRY(cudaEventCreate(&e0));
        CU_TRY(cudaEventCreate(&e1));
        float best_ms = 1e30f;
        for (size_t k = 0; k < shapes.size(); ++k) {
            const int sys = std::min(cap, std::max(1, shapes[k].clusters));
            CU_TRY(cudaMemcpyAsync(b->V[0], b->X, sizeof(double) * b->N * sys, cudaMemcpyDeviceToDevice, b->stream));
            CU_TRY(cudaMemsetAsync(b->counters, 0, sizeof(unsigned), b->stream));
            CU_TRY(cudaMemsetAsync(b->error, 0, sizeof(int), b->stream));
            ClusterParams p = base;
            p.X = static_cast<double *>(b->V[0]);
            p.cs_log2 = shapes[k].cs_log2;
            p.sbits = shapes[k].sbits;
            p.max_steps = 32;
            p.exit_rule = 0;
            p.sys_limit = sys;
            CU_TRY(cudaEventRecord(e0, b->stream));
            tasep_status s = cluster_launch_p(b, p, std::min(shapes[k].clusters, sys));
            if (s) return s;
            CU_TRY(cudaEventRecord(e1, b->stream));
            CU_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            CU_TRY(cudaEventElapsedTime(&ms, e0, e1));
            // time per system-step with every cluster busy
            const float per = ms / float(sys) * float(std::min(shapes[k].clusters, sys)) / float(shapes[k].clusters);
            if (per < best_ms) {
                best_ms = per;
                best = k;
            }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        int herr = 0;
        CU_TRY(cudaMemcpy(&herr, b->error, sizeof(int), cudaMemcpyDeviceToHost));
        if (herr) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired");
    }
    const Shape &sh = shapes[best];
    ClusterParams p = base;
    p.X = b->X;
    p.cs_log2 = sh.cs_log2;
    p.sbits = sh.sbits;
    p.max_steps = rc->steps;
    p.sys_limit = b->nsys;
    CU_TRY(cudaMemsetAsync(b->ex, 0, sizeof(BatchExit) * b->nsys, b->stream));
    CU_TRY(cudaMemsetAsync(b->counters, 0, sizeof(unsigned), b->stream));
    CU_TRY(cudaMemsetAsync(b->error, 0, sizeof(int), b->stream));
    tasep_status s = cluster_launch_p(b, p, std::min(sh.clusters, b->nsys));
    if (s) return s;
    int herr = 0;
    CU_TRY(cudaMemcpyAsync(&herr, b->error, sizeof(int), cudaMemcpyDeviceToHost, b->stream));
    CU_TRY(cudaStreamSynchronize(b->stream));
    if (herr) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired");
    b->last_schedule = 2;
    b->last_states_per_cta = 1 << sh.sbits;
    b->last_ctas_per_system = 1 << sh.cs_log2;
    if (schedule_used) *schedule_used = 2;
    if (res) {
        std::vector<BatchExit> ex(b->nsys);
        CU_TRY(cudaMemcpy(ex.data(), b->ex, sizeof(BatchExit) * b->nsys, cudaMemcpyDeviceToHost));
        for (int k = 0; k < b->nsys; ++k) {
            res[k].steps_done = ex[k].steps_done;
            res[k].steps_at_stop = ex[k].steps_at_stop;
            res[k].early_stop = ex[k].early_stop;
            res[k].converged = ex[k].converged;
            res[k].last_checksum = ex[k].last_checksum;
            double t = rc->t0;
            for (unsigned long long q = 0; q < ex[k].steps_done; ++q) t += rc->h;
            res[k].t_end = t;
        }
    }
    return TASEP_OK;
}

}  // namespace

extern "C" {

tasep_status tasep_batch_create(int n, int nsys, int precision, int device, void *stream, tasep_batch **out) {
    if (!out) return fail(TASEP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (n <= kTileBits || n > 24) return fail(TASEP_ERR_INVALID, "batched systems need %d < n <= 24", kTileBits);
    if (nsys < 1) return fail(TASEP_ERR_INVALID, "nsys=%d", nsys);
    if ((uint64_t(nsys) << (n - kTileBits)) >= (1ull << 31))  // 32-bit tile indices in the sweep
        return fail(TASEP_ERR_INVALID, "nsys=%d systems of n=%d exceed 2^31 tiles", nsys, n);
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
    if (schedule < -1 || schedule > 2) return fail(TASEP_ERR_INVALID, "schedule %d", schedule);
    if (schedule == 2 && !cluster_eligible(b))
        return fail(TASEP_ERR_UNSUPPORTED, "the cluster-resident schedule needs %d < n <= %d", kTileBits, kClMaxN);
    CU_TRY(cudaSetDevice(b->device));
    // the cluster-resident engine runs when asked for; measured on B200 it is
    // slower than the tile engines for the standard n = 16 sweep, so the
    // automatic choice stays with schedules 0 and 1
    if (schedule == 2) return batch_run_cluster(b, rc, -1, res, schedule_used);
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
    CU_TRY(launch_pdl(batch_compact_kernel, dim3(1), dim3(1024), 0, b->stream, b->ex, b->nsys, b->list, b->count));
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
    b->last_schedule = sched;
    b->last_states_per_cta = kTile;
    b->last_ctas_per_system = 0;
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

tasep_status tasep_batch_last_config(const tasep_batch *b, int *schedule, int *states_per_cta,
                                     int *ctas_per_system) {
    if (!b) return fail(TASEP_ERR_INVALID, "null handle");
    if (schedule) *schedule = b->last_schedule;
    if (states_per_cta) *states_per_cta = b->last_states_per_cta;
    if (ctas_per_system) *ctas_per_system = b->last_ctas_per_system;
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
