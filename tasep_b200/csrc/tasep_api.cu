// tasep_api.cu - C ABI of libtasep_cuda.so (declared in include/tasep.h).
#include <atomic>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "tasep.h"
#include "meq_common.cuh"
#include "meq_obs.cuh"
#include "meq_small.cuh"
#include "meq_tile.cuh"

using namespace tasep;

namespace {

thread_local std::string g_last_error;

tasep_status fail(tasep_status st, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

#define CU_TRY(expr)                                                                            \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) {                                                                \
            if (e_ == cudaErrorMemoryAllocation) {                                              \
                cudaGetLastError();                                                             \
                return fail(TASEP_ERR_NOMEM, "%s: %s", #expr, cudaGetErrorString(e_));          \
            }                                                                                   \
            return fail(TASEP_ERR_CUDA, "%s: %s", #expr, cudaGetErrorString(e_));               \
        }                                                                                       \
    } while (0)

const char *const kStageNames[ST_COUNT] = {"meq_ref_step",  "meq_rk4_h1", "meq_rk4_h2", "meq_rk4_h3",
                                           "meq_rk4_h4",    "meq_rk4_u1", "meq_rk4_u2", "meq_rk4_u3",
                                           "meq_rk4_u4",    "meq_apply"};
constexpr int kProfSlots = 4;  // + small kernel, observables
const char *const kExtraNames[kProfSlots] = {"meq_small_run", "meq_observables", "", ""};

// Per-device scratch of the device-pointer operators.
struct DevScratch {
    double *partials = nullptr;
    unsigned *counter = nullptr;
    ExitState *ex = nullptr;
    int nsm = 0;
};
std::mutex g_scratch_mu;
DevScratch g_scratch[64];

tasep_status get_scratch(int dev, DevScratch **out) {
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (dev < 0 || dev >= 64) return fail(TASEP_ERR_INVALID, "device ordinal %d out of range", dev);
    DevScratch &s = g_scratch[dev];
    if (!s.ex) {
        CU_TRY(cudaDeviceGetAttribute(&s.nsm, cudaDevAttrMultiProcessorCount, dev));
        CU_TRY(cudaMalloc(&s.partials, sizeof(double) * 4096));
        CU_TRY(cudaMalloc(&s.counter, 64));
        CU_TRY(cudaMemset(s.counter, 0, 64));
        CU_TRY(cudaMalloc(&s.ex, sizeof(ExitState)));
        CU_TRY(cudaMemset(s.ex, 0, sizeof(ExitState)));
    }
    *out = &s;
    return TASEP_OK;
}

template <int S, typename E, bool kTuned> tasep_status launch_tile_t(const TileParams &p, int grid, cudaStream_t st) {
    // set once per device; concurrent first calls may both set it (idempotent)
    static std::atomic<bool> configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const int bytes = TileLayout<S, E>::bytes;
    if (!configured[dev & 63].load(std::memory_order_acquire)) {
        CU_TRY(cudaFuncSetAttribute(meq_tile_kernel<S, E, kTuned>, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
        configured[dev & 63].store(true, std::memory_order_release);
    }
    CU_TRY(launch_pdl(meq_tile_kernel<S, E, kTuned>, dim3(grid), dim3(kTileThreads), size_t(bytes), st, p));
    return TASEP_OK;
}

// The lean instantiation unless a non-default L2 policy or the test hook is set.
template <int S, typename E> tasep_status launch_tile(const TileParams &p, int grid, cudaStream_t st) {
    if (p.l2_near < 64 || p.l2_flags || p.skip_copy_plus1) return launch_tile_t<S, E, true>(p, grid, st);
    return launch_tile_t<S, E, false>(p, grid, st);
}

template <typename E> tasep_status launch_small(const SmallParams &p, cudaStream_t st) {
    static std::atomic<bool> configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t bytes = small_smem_bytes(p.n);
    if (!configured[dev & 63].load(std::memory_order_acquire)) {
        CU_TRY(cudaFuncSetAttribute(meq_small_kernel<E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(small_smem_bytes(kSmallMaxN))));
        configured[dev & 63].store(true, std::memory_order_release);
    }
    meq_small_kernel<E><<<1, kSmallThreads, bytes, st>>>(p);
    CU_TRY(cudaGetLastError());
    return TASEP_OK;
}

// Default L2 policy of the tile sweep (L2F_* in meq_tile.cuh).
int g_l2_near_default = 64;
int g_l2_flags_default = 0;

// tasep_test_inject_wait_expiry: wait limit and left-out partner copy of
// every tile launch (0 = off).
std::atomic<unsigned long long> g_test_wait_ns{0};
std::atomic<int> g_test_skip_copy{0};

void apply_test_hook(TileParams &p) {
    p.wait_ns = g_test_wait_ns.load();
    p.skip_copy_plus1 = g_test_skip_copy.load();
}

void fill_const_rates(RateSpec &rs, int n, const double *r) {
    memset(&rs, 0, sizeof rs);
    for (int i = 0; i <= n; ++i) rs.r[i] = r[i];
    rs.timevar = 0;
}

}  // namespace

struct tasep_meq {
    int n = 0, integrator = 0, precision = 0, device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    unsigned long long N = 0, ntiles = 0;
    int nsm = 0, grid = 0;
    double *X[2] = {nullptr, nullptr};
    void *V[3] = {nullptr, nullptr, nullptr};  // v1, v2, w (factored RK4) or U2,U3,U4 (time-variant RK4)
    double *partials = nullptr;
    unsigned *counter = nullptr;
    ExitState *ex = nullptr;
    ExitState *ex_host = nullptr;  // pinned
    double *obs_part = nullptr, *obs_out = nullptr;
    int obs_rows = 0;
    int cur = 0;
    int l2_near = 64, l2_flags = 0;  // L2 policy of the tile sweep
    bool rates_set = false, state_set = false;
    RateSpec rs{};
    // profiling
    bool prof = false;
    std::vector<cudaEvent_t> ev_pool;
    std::vector<int> pend_kind;  // kernel kind per pending event pair
    int ev_used = 0;
    double prof_ms[ST_COUNT + kProfSlots] = {};
    uint64_t prof_n[ST_COUNT + kProfSlots] = {};
};

namespace {

tasep_status prof_flush(tasep_meq *m) {
    if (!m->ev_used) return TASEP_OK;
    CU_TRY(cudaEventSynchronize(m->ev_pool[2 * m->ev_used - 1]));
    for (int i = 0; i < m->ev_used; ++i) {
        float ms = 0.f;
        CU_TRY(cudaEventElapsedTime(&ms, m->ev_pool[2 * i], m->ev_pool[2 * i + 1]));
        m->prof_ms[m->pend_kind[i]] += ms;
        m->prof_n[m->pend_kind[i]] += 1;
    }
    m->ev_used = 0;
    return TASEP_OK;
}

tasep_status prof_begin(tasep_meq *m, int kind) {
    if (!m->prof) return TASEP_OK;
    if (m->ev_used * 2 + 2 > int(m->ev_pool.size())) {
        tasep_status s = prof_flush(m);
        if (s) return s;
    }
    m->pend_kind[m->ev_used] = kind;
    CU_TRY(cudaEventRecord(m->ev_pool[2 * m->ev_used], m->stream));
    return TASEP_OK;
}

tasep_status prof_end(tasep_meq *m) {
    if (!m->prof) return TASEP_OK;
    CU_TRY(cudaEventRecord(m->ev_pool[2 * m->ev_used + 1], m->stream));
    m->ev_used++;
    return TASEP_OK;
}

template <int S, typename E> tasep_status run_stage(tasep_meq *m, TileParams &p) {
    tasep_status s = prof_begin(m, S);
    if (s) return s;
    s = launch_tile<S, E>(p, m->grid, m->stream);
    if (s) return s;
    return prof_end(m);
}

TileParams base_params(tasep_meq *m, double h, unsigned long long step, double thresh, int stop_count,
                       int exit_rule) {
    TileParams p;
    memset(&p, 0, sizeof p);
    p.n = m->n;
    p.l2_near = m->l2_near;
    p.l2_flags = m->l2_flags;
    apply_test_hook(p);
    p.ntiles = m->ntiles;
    p.h = h;
    p.partials = m->partials;
    p.counter = m->counter;
    p.ex = m->ex;
    p.step = step;
    p.thresh = thresh;
    p.stop_count = stop_count;
    p.exit_rule = exit_rule;
    p.skip_if_done = 1;
    p.rs = m->rs;
    return p;
}

// Enqueues one step (n > kSmallMaxN).
template <typename E>
tasep_status enqueue_step_t(tasep_meq *m, unsigned long long step, double t, double h, double thresh,
                            int stop_count, int exit_rule) {
    TileParams p = base_params(m, h, step, thresh, stop_count, exit_rule);
    tasep_status s;
    if (m->integrator == TASEP_INTEGRATOR_REF) {
        p.g = m->X[m->cur];
        p.out = m->X[m->cur ^ 1];
        p.t = t;
        s = run_stage<ST_REF, double>(m, p);
        m->cur ^= 1;
        return s;
    }
    double *X = m->X[0];
    if (m->rs.timevar) {
        p.t = t; p.g = X; p.out = m->V[0]; p.hc = 0.5 * h;
        if ((s = run_stage<ST_U1, double>(m, p))) return s;
        p.t = t + h / 2; p.g = m->V[0]; p.s0 = X; p.out = m->V[1]; p.hc = 0.5 * h;
        if ((s = run_stage<ST_U2, double>(m, p))) return s;
        p.t = t + h / 2; p.g = m->V[1]; p.s0 = X; p.out = m->V[2]; p.hc = h;
        if ((s = run_stage<ST_U3, double>(m, p))) return s;
        p.t = t + h; p.g = m->V[2]; p.s0 = X; p.s1 = m->V[0]; p.s2 = m->V[1]; p.out = X;
        return run_stage<ST_U4, double>(m, p);
    }
    // classical RK4 in factored form (Rk4Factors): v1 = z x, v2 = (z - r) v1,
    // w = (z + p) v2, x' = x + (z w + q v2) / 24
    static const Rk4Factors F = rk4_factors();
    p.t = t;
    p.g = X; p.out = m->V[0];
    if ((s = run_stage<ST_H1, E>(m, p))) return s;
    p.g = m->V[0]; p.out = m->V[1]; p.hc = h; p.cx = -F.r;
    if ((s = run_stage<ST_H2, E>(m, p))) return s;
    p.g = m->V[1]; p.out = m->V[2]; p.hc = h; p.cx = F.p;
    if ((s = run_stage<ST_H3, E>(m, p))) return s;
    p.g = m->V[2]; p.s0 = m->V[1]; p.s1 = X; p.out = X; p.hc = h / 24; p.cx = F.q / 24;
    return run_stage<ST_H4, E>(m, p);
}

tasep_status enqueue_step(tasep_meq *m, unsigned long long step, double t, double h, double thresh,
                          int stop_count, int exit_rule) {
    if (m->precision == TASEP_PRECISION_MIXED)
        return enqueue_step_t<float>(m, step, t, h, thresh, stop_count, exit_rule);
    return enqueue_step_t<double>(m, step, t, h, thresh, stop_count, exit_rule);
}

tasep_status small_run(tasep_meq *m, double t0, double h, unsigned long long steps, unsigned long long step0,
                       double thresh, int stop_count, int exit_rule) {
    SmallParams sp;
    memset(&sp, 0, sizeof sp);
    sp.n = m->n;
    sp.mode = SM_RUN;
    sp.integrator = m->integrator == TASEP_INTEGRATOR_REF ? SI_REF : (m->rs.timevar ? SI_UFORM : SI_HORNER);
    sp.x_in = m->X[m->cur];
    sp.x_out = m->X[m->cur];
    sp.h = h;
    sp.t0 = t0;
    sp.max_steps = steps;
    sp.step0 = step0;
    sp.thresh = thresh;
    sp.stop_count = stop_count;
    sp.exit_rule = exit_rule;
    sp.ex = m->ex;
    sp.rs = m->rs;
    tasep_status s = prof_begin(m, ST_COUNT + 0);
    if (s) return s;
    s = (m->precision == TASEP_PRECISION_MIXED && sp.integrator == SI_HORNER) ? launch_small<float>(sp, m->stream)
                                                                               : launch_small<double>(sp, m->stream);
    if (s) return s;
    return prof_end(m);
}

// The step's RN(s / 6) applied to a vector (tasep_test_div6).
__global__ void div6_kernel(double *v, uint64_t count) {
    for (uint64_t i = blockIdx.x * uint64_t(blockDim.x) + threadIdx.x; i < count; i += uint64_t(gridDim.x) * blockDim.x)
        v[i] = div6_rn(v[i]);
}

bool valid_handle(const tasep_meq *m) { return m != nullptr && m->n >= 1; }

}  // namespace

extern "C" {

const char *tasep_last_error(void) { return g_last_error.c_str(); }

tasep_status tasep_test_inject_wait_expiry(uint64_t wait_limit_ns, int skip_partner_copy) {
    if (skip_partner_copy < -1) return fail(TASEP_ERR_INVALID, "skip_partner_copy %d < -1", skip_partner_copy);
    g_test_wait_ns.store(wait_limit_ns);
    g_test_skip_copy.store(skip_partner_copy + 1);
    return TASEP_OK;
}
tasep_status tasep_test_div6(const double *host_in, double *host_out, uint64_t count) {
    if ((!host_in || !host_out) && count) return fail(TASEP_ERR_INVALID, "null argument");
    if (count == 0) return TASEP_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TASEP_ERR_NODEV, "no CUDA device");
    }
    double *d = nullptr;
    CU_TRY(cudaMalloc(&d, sizeof(double) * count));
    struct Free {
        double *p;
        ~Free() { cudaFree(p); }
    } guard{d};
    CU_TRY(cudaMemcpy(d, host_in, sizeof(double) * count, cudaMemcpyHostToDevice));
    div6_kernel<<<unsigned((count + 255) / 256 < 65535 ? (count + 255) / 256 : 65535), 256>>>(d, count);
    CU_TRY(cudaGetLastError());
    CU_TRY(cudaMemcpy(host_out, d, sizeof(double) * count, cudaMemcpyDeviceToHost));
    return TASEP_OK;
}

int tasep_abi_version(void) { return TASEP_ABI_VERSION; }

uint64_t tasep_meq_footprint(int n, int integrator, int precision, int timevar) {
    if (n < 1 || n > TASEP_MAX_N) return 0;
    const uint64_t N = 1ull << n;
    if (integrator == TASEP_INTEGRATOR_REF) return 2 * 8 * N;
    if (precision == TASEP_PRECISION_MIXED && !timevar) return 8 * N + 3 * 4 * N;
    return 4 * 8 * N;
}

tasep_status tasep_meq_create(const tasep_meq_config *cfg, tasep_meq **out) {
    if (!cfg || !out) return fail(TASEP_ERR_INVALID, "null argument");
    *out = nullptr;
    if (cfg->n < 1 || cfg->n > TASEP_MAX_N) return fail(TASEP_ERR_INVALID, "n=%d outside 1..%d", cfg->n, TASEP_MAX_N);
    if (cfg->integrator != TASEP_INTEGRATOR_REF && cfg->integrator != TASEP_INTEGRATOR_RK4)
        return fail(TASEP_ERR_INVALID, "unknown integrator %d", cfg->integrator);
    if (cfg->precision != TASEP_PRECISION_FP64 && cfg->precision != TASEP_PRECISION_MIXED)
        return fail(TASEP_ERR_INVALID, "unknown precision %d", cfg->precision);
    if (cfg->precision == TASEP_PRECISION_MIXED && cfg->integrator != TASEP_INTEGRATOR_RK4)
        return fail(TASEP_ERR_UNSUPPORTED, "mixed precision applies to the RK4 integrator only");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(TASEP_ERR_NODEV, "no CUDA device");
    }
    int dev = cfg->device;
    if (dev < 0) CU_TRY(cudaGetDevice(&dev));
    if (dev >= ndev) return fail(TASEP_ERR_INVALID, "device %d of %d", dev, ndev);
    CU_TRY(cudaSetDevice(dev));
    tasep_meq *m = new tasep_meq();
    m->n = cfg->n;
    m->integrator = cfg->integrator;
    m->precision = cfg->precision;
    m->device = dev;
    m->N = 1ull << cfg->n;
    m->l2_near = g_l2_near_default;
    m->l2_flags = g_l2_flags_default;
    m->ntiles = cfg->n > kSmallMaxN ? (m->N >> kTileBits) : 1;
    cudaDeviceGetAttribute(&m->nsm, cudaDevAttrMultiProcessorCount, dev);
    m->grid = int(m->ntiles < (unsigned long long)m->nsm ? m->ntiles : m->nsm);
    auto bail = [&](tasep_status s) {
        tasep_meq_destroy(m);
        return s;
    };
    if (cfg->stream) {
        m->stream = static_cast<cudaStream_t>(cfg->stream);
    } else {
        if (cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) != cudaSuccess)
            return bail(fail(TASEP_ERR_CUDA, "stream creation failed"));
        m->own_stream = true;
    }
    const size_t vec = sizeof(double) * m->N;
    auto alloc = [&](void **p, size_t bytes) -> bool {
        if (cudaMalloc(p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        return true;
    };
    const size_t sv = (m->precision == TASEP_PRECISION_MIXED ? sizeof(float) : sizeof(double)) * m->N;
    bool ok = alloc(reinterpret_cast<void **>(&m->X[0]), vec);
    if (ok && (m->integrator == TASEP_INTEGRATOR_REF)) ok = alloc(reinterpret_cast<void **>(&m->X[1]), vec);
    if (ok && m->integrator == TASEP_INTEGRATOR_RK4)
        for (int i = 0; i < 3 && ok; ++i) ok = alloc(&m->V[i], m->n > kSmallMaxN ? sv : 8);
    if (!ok)
        return bail(fail(TASEP_ERR_NOMEM, "not enough device memory for n=%d (%llu bytes of state vectors)", m->n,
                         (unsigned long long)tasep_meq_footprint(m->n, m->integrator, m->precision, 0)));
    m->obs_rows = int(std::min<unsigned long long>(2ull * m->nsm, 1ull << (m->n - std::min(m->n, kObsBits))));
    ok = alloc(reinterpret_cast<void **>(&m->partials), sizeof(double) * 4096) &&
         alloc(reinterpret_cast<void **>(&m->counter), 64) &&
         alloc(reinterpret_cast<void **>(&m->ex), sizeof(ExitState)) &&
         alloc(reinterpret_cast<void **>(&m->obs_part), sizeof(double) * size_t(m->obs_rows) * obs_count(m->n)) &&
         alloc(reinterpret_cast<void **>(&m->obs_out), sizeof(double) * obs_count(m->n));
    if (!ok) return bail(fail(TASEP_ERR_NOMEM, "not enough device memory for scratch"));
    if (cudaMallocHost(&m->ex_host, sizeof(ExitState)) != cudaSuccess)
        return bail(fail(TASEP_ERR_NOMEM, "pinned host allocation failed"));
    if (cudaMemset(m->counter, 0, 64) != cudaSuccess || cudaMemset(m->ex, 0, sizeof(ExitState)) != cudaSuccess)
        return bail(fail(TASEP_ERR_CUDA, "memset failed"));
    m->ev_pool.resize(2048);
    m->pend_kind.resize(1024);
    for (auto &e : m->ev_pool)
        if (cudaEventCreate(&e) != cudaSuccess) return bail(fail(TASEP_ERR_CUDA, "event creation failed"));
    *out = m;
    return TASEP_OK;
}

tasep_status tasep_meq_destroy(tasep_meq *m) {
    if (!m) return TASEP_OK;
    cudaSetDevice(m->device);
    if (m->stream) cudaStreamSynchronize(m->stream);
    cudaFree(m->X[0]);
    cudaFree(m->X[1]);
    for (auto &v : m->V) cudaFree(v);
    cudaFree(m->partials);
    cudaFree(m->counter);
    cudaFree(m->ex);
    cudaFree(m->obs_part);
    cudaFree(m->obs_out);
    if (m->ex_host) cudaFreeHost(m->ex_host);
    for (auto &e : m->ev_pool)
        if (e) cudaEventDestroy(e);
    if (m->own_stream && m->stream) cudaStreamDestroy(m->stream);
    delete m;
    return TASEP_OK;
}

tasep_status tasep_meq_set_rates(tasep_meq *m, const double *rates) {
    if (!valid_handle(m) || !rates) return fail(TASEP_ERR_INVALID, "null argument");
    const int tv = m->rs.timevar;
    RateSpec keep = m->rs;
    fill_const_rates(m->rs, m->n, rates);
    if (tv) {  // keep the functions; constant rates stand for unknown function types
        memcpy(m->rs.amp, keep.amp, sizeof keep.amp);
        memcpy(m->rs.per, keep.per, sizeof keep.per);
        memcpy(m->rs.off, keep.off, sizeof keep.off);
        memcpy(m->rs.cst, keep.cst, sizeof keep.cst);
        memcpy(m->rs.type, keep.type, sizeof keep.type);
        m->rs.timevar = 1;
    }
    m->rates_set = true;
    return TASEP_OK;
}

tasep_status tasep_meq_set_timevar(tasep_meq *m, const int *type, const double *amplitude, const double *period,
                                   const double *offset, const double *constant) {
    if (!valid_handle(m) || !type || !amplitude || !period || !offset || !constant)
        return fail(TASEP_ERR_INVALID, "null argument");
    if (m->integrator == TASEP_INTEGRATOR_RK4 && m->precision == TASEP_PRECISION_MIXED)
        return fail(TASEP_ERR_UNSUPPORTED, "time-variant rates need FP64 with the RK4 integrator");
    for (int i = 0; i <= m->n; ++i) {
        m->rs.type[i] = type[i];
        m->rs.amp[i] = amplitude[i];
        m->rs.per[i] = period[i];
        m->rs.off[i] = offset[i];
        m->rs.cst[i] = constant[i];
    }
    m->rs.timevar = 1;
    m->rates_set = true;
    return TASEP_OK;
}

tasep_status tasep_meq_clear_timevar(tasep_meq *m) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    m->rs.timevar = 0;
    return TASEP_OK;
}

tasep_status tasep_meq_init(tasep_meq *m, int kind) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    CU_TRY(cudaSetDevice(m->device));
    m->cur = 0;
    if (kind == TASEP_INIT_EMPTY) {
        CU_TRY(cudaMemsetAsync(m->X[0], 0, sizeof(double) * m->N, m->stream));
        const double one = 1.0;
        CU_TRY(cudaMemcpyAsync(m->X[0], &one, sizeof one, cudaMemcpyHostToDevice, m->stream));
        CU_TRY(cudaStreamSynchronize(m->stream));
    } else if (kind == TASEP_INIT_UNIFORM) {
        // 1./d with d = 2^n (src/masterEquation.c:400-409): an exact power of two
        const double v = 1.0 / double(m->N);
        // fill by doubling copies from a small seed
        std::vector<double> seed(std::min<unsigned long long>(m->N, 1ull << 16), v);
        CU_TRY(cudaMemcpy(m->X[0], seed.data(), sizeof(double) * seed.size(), cudaMemcpyHostToDevice));
        unsigned long long have = seed.size();
        while (have < m->N) {
            const unsigned long long cnt = std::min(have, m->N - have);
            CU_TRY(cudaMemcpyAsync(m->X[0] + have, m->X[0], sizeof(double) * cnt, cudaMemcpyDeviceToDevice,
                                   m->stream));
            have += cnt;
        }
        CU_TRY(cudaStreamSynchronize(m->stream));
    } else {
        return fail(TASEP_ERR_INVALID, "unknown initial state %d", kind);
    }
    m->state_set = true;
    return TASEP_OK;
}

tasep_status tasep_meq_load(tasep_meq *m, const double *host_x) {
    if (!valid_handle(m) || !host_x) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(m->device));
    m->cur = 0;
    CU_TRY(cudaMemcpyAsync(m->X[0], host_x, sizeof(double) * m->N, cudaMemcpyHostToDevice, m->stream));
    CU_TRY(cudaStreamSynchronize(m->stream));
    m->state_set = true;
    return TASEP_OK;
}

tasep_status tasep_meq_store(const tasep_meq *m, double *host_x, uint64_t offset, uint64_t count) {
    if (!valid_handle(m) || (!host_x && count)) return fail(TASEP_ERR_INVALID, "null argument");
    if (offset > m->N || count > m->N - offset) return fail(TASEP_ERR_INVALID, "range outside the state");
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaMemcpyAsync(host_x, m->X[m->cur] + offset, sizeof(double) * count, cudaMemcpyDeviceToHost,
                           m->stream));
    CU_TRY(cudaStreamSynchronize(m->stream));
    return TASEP_OK;
}

static tasep_status check_ready(tasep_meq *m, double h) {
    if (!m->rates_set) return fail(TASEP_ERR_INVALID, "rates not set");
    if (!m->state_set) return fail(TASEP_ERR_INVALID, "initial state not set");
    if (!(h == h)) return fail(TASEP_ERR_INVALID, "step size is NaN");
    return TASEP_OK;
}

tasep_status tasep_meq_run(tasep_meq *m, const tasep_run_config *rc, tasep_run_result *res) {
    if (!valid_handle(m) || !rc || !res) return fail(TASEP_ERR_INVALID, "null argument");
    tasep_status s = check_ready(m, rc->h);
    if (s) return s;
    CU_TRY(cudaSetDevice(m->device));
    memset(res, 0, sizeof *res);
    const double thresh = rc->stop_tol * rc->h;
    CU_TRY(cudaMemsetAsync(m->ex, 0, sizeof(ExitState), m->stream));
    const int cur0 = m->cur;
    unsigned long long done = 0;
    if (m->n <= kSmallMaxN) {
        if ((s = small_run(m, rc->t0, rc->h, rc->steps, 0, thresh, rc->stop_count, rc->exit_rule))) return s;
        CU_TRY(cudaMemcpyAsync(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost, m->stream));
        CU_TRY(cudaStreamSynchronize(m->stream));
    } else {
        const int shift = 30 - m->n;
        const unsigned long long chunk = shift >= 10 ? 1024ull : (shift <= 2 ? 4ull : (1ull << shift));
        double t = rc->t0;
        unsigned long long i = 0;
        while (i < rc->steps) {
            const unsigned long long c = std::min(chunk, rc->steps - i);
            for (unsigned long long j = 0; j < c; ++j, ++i) {
                if ((s = enqueue_step(m, i, t, rc->h, thresh, rc->stop_count, rc->exit_rule))) return s;
                t += rc->h;
            }
            CU_TRY(cudaMemcpyAsync(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost, m->stream));
            CU_TRY(cudaStreamSynchronize(m->stream));
            if (m->ex_host->done || m->ex_host->error) break;
        }
        if (m->prof && (s = prof_flush(m))) return s;
    }
    const ExitState &e = *m->ex_host;
    if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
    done = e.steps_done;
    if (m->integrator == TASEP_INTEGRATOR_REF && m->n > kSmallMaxN) m->cur = int((cur0 + done) & 1ull);
    res->steps_done = done;
    res->steps_at_stop = e.steps_at_stop;
    res->early_stop = e.early_stop;
    res->converged = e.converged;
    res->last_checksum = e.last_checksum;
    double t = rc->t0;
    for (unsigned long long k = 0; k < done; ++k) t += rc->h;
    res->t_end = t;
    return TASEP_OK;
}

tasep_status tasep_meq_run_snapshots(tasep_meq *m, const tasep_run_config *rc, uint64_t every,
                                     tasep_snapshot_fn fn, void *user, tasep_run_result *res) {
    if (!valid_handle(m) || !rc || !res || !fn || every < 1) return fail(TASEP_ERR_INVALID, "bad argument");
    tasep_status s = check_ready(m, rc->h);
    if (s) return s;
    CU_TRY(cudaSetDevice(m->device));
    memset(res, 0, sizeof *res);
    const double thresh = rc->stop_tol * rc->h;
    CU_TRY(cudaMemsetAsync(m->ex, 0, sizeof(ExitState), m->stream));
    const int cur0 = m->cur;
    const bool small = m->n <= kSmallMaxN;
    const int shift = 30 - m->n;
    const unsigned long long chunk = shift >= 10 ? 1024ull : (shift <= 2 ? 4ull : (1ull << shift));
    double t = rc->t0;
    unsigned long long i = 0;
    while (i < rc->steps) {
        // run steps i..last: up to the next snapshot step, the end, or a chunk
        const unsigned long long snap = (i + every - 1) / every * every;
        unsigned long long last = std::min<unsigned long long>(snap, rc->steps - 1);
        if (!small) last = std::min(last, i + chunk - 1);
        if (small) {
            if ((s = small_run(m, t, rc->h, last - i + 1, i, thresh, rc->stop_count, rc->exit_rule))) return s;
            for (unsigned long long j = i; j <= last; ++j) t += rc->h;
        } else {
            for (unsigned long long j = i; j <= last; ++j) {
                if ((s = enqueue_step(m, j, t, rc->h, thresh, rc->stop_count, rc->exit_rule))) return s;
                t += rc->h;
            }
        }
        i = last + 1;
        CU_TRY(cudaMemcpyAsync(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost, m->stream));
        CU_TRY(cudaStreamSynchronize(m->stream));
        const ExitState e = *m->ex_host;
        if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
        if (last % every == 0 && e.steps_done > last) {  // step `last` ran: snapshot it
            if (m->prof && (s = prof_flush(m))) return s;
            fn(m, last, t, user);
        }
        if (e.done) break;
    }
    if (m->prof && (s = prof_flush(m))) return s;
    CU_TRY(cudaMemcpy(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost));
    const ExitState &e = *m->ex_host;
    if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
    const unsigned long long done = e.steps_done;
    if (m->integrator == TASEP_INTEGRATOR_REF && !small) m->cur = int((cur0 + done) & 1ull);
    res->steps_done = done;
    res->steps_at_stop = e.steps_at_stop;
    res->early_stop = e.early_stop;
    res->converged = e.converged;
    res->last_checksum = e.last_checksum;
    double tt = rc->t0;
    for (unsigned long long k = 0; k < done; ++k) tt += rc->h;
    res->t_end = tt;
    return TASEP_OK;
}

tasep_status tasep_meq_enqueue_steps(tasep_meq *m, double t0, double h, uint64_t steps) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    tasep_status s = check_ready(m, h);
    if (s) return s;
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaMemsetAsync(m->ex, 0, sizeof(ExitState), m->stream));
    if (m->n <= kSmallMaxN) return small_run(m, t0, h, steps, 0, 0.0, 0, 0);
    double t = t0;
    for (uint64_t i = 0; i < steps; ++i) {
        if ((s = enqueue_step(m, i, t, h, 0.0, 0, 0))) return s;
        t += h;
    }
    return TASEP_OK;
}

tasep_status tasep_meq_synchronize(tasep_meq *m) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaStreamSynchronize(m->stream));
    if (m->prof) {
        tasep_status s = prof_flush(m);
        if (s) return s;
    }
    CU_TRY(cudaMemcpy(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost));
    if (m->ex_host->error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired");
    return TASEP_OK;
}

}  // extern "C"

namespace {

// Enqueues the observables of X[cur] into out (obs_count(n) raw sums).
tasep_status obs_enqueue(tasep_meq *m, double *out, cudaStream_t st) {
    const int n = m->n, na = obs_count(n);
    static std::atomic<bool> configured[64] = {};
    if (!configured[m->device & 63].load(std::memory_order_acquire)) {
        CU_TRY(cudaFuncSetAttribute(meq_obs_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    int(obs_smem_bytes(TASEP_MAX_N))));
        configured[m->device & 63].store(true, std::memory_order_release);
    }
    ObsParams op{n, m->X[m->cur], m->obs_part};
    meq_obs_kernel<<<m->obs_rows, kObsThreads, obs_smem_bytes(n), st>>>(op);
    CU_TRY(cudaGetLastError());
    meq_obs_reduce<<<(na + 255) / 256, 256, 0, st>>>(m->obs_part, m->obs_rows, na, out);
    CU_TRY(cudaGetLastError());
    return TASEP_OK;
}

// Raw sums (total, second moments, 4-bit window marginals) to the outputs of
// tasep_meq_observables.
void obs_convert(int n, const double *o, double *rho, double *cov, double *mul, double *window4, double *mass) {
    const double S0 = o[0];
    std::vector<double> y(n);
    for (int a = 0; a < n; ++a) y[a] = o[obs_tri(n, a, a)];
    if (rho)
        for (int a = 0; a < n; ++a) rho[a] = y[a];
    if (mass) *mass = S0;
    if (cov || mul) {
        // sum_s (b_k - y_k)(b_i - y_i) x_s = M_ik - y_i y_k (2 - S0), site order
        for (int i = 0; i < n; ++i)
            for (int k = 0; k < n; ++k) {
                const int a = i < k ? i : k, b = i < k ? k : i;
                const double Mik = o[obs_tri(n, a, b)];
                const double c = Mik - y[i] * y[k] * (2.0 - S0);
                if (cov) cov[(n - 1 - i) * n + (n - 1 - k)] = c;
                if (mul) mul[(n - 1 - i) * n + (n - 1 - k)] = y[k] * y[i] + c;
            }
    }
    if (window4 && n >= 4)
        for (int p = 0; p + 4 <= n; ++p)
            for (int q = 0; q < 16; ++q) window4[p * 16 + q] = o[obs_p4(n, p, q)];
}

}  // namespace

extern "C" {

tasep_status tasep_meq_observables(tasep_meq *m, double *rho, double *cov, double *mul, double *window4,
                                   double *mass) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    if (!m->state_set) return fail(TASEP_ERR_INVALID, "initial state not set");
    CU_TRY(cudaSetDevice(m->device));
    const int na = obs_count(m->n);
    tasep_status s = prof_begin(m, ST_COUNT + 1);
    if (s) return s;
    if ((s = obs_enqueue(m, m->obs_out, m->stream))) return s;
    if ((s = prof_end(m))) return s;
    std::vector<double> o(na);
    CU_TRY(cudaMemcpyAsync(o.data(), m->obs_out, sizeof(double) * na, cudaMemcpyDeviceToHost, m->stream));
    CU_TRY(cudaStreamSynchronize(m->stream));
    obs_convert(m->n, o.data(), rho, cov, mul, window4, mass);
    return TASEP_OK;
}

tasep_status tasep_meq_run_stream(tasep_meq *m, const tasep_run_config *rc, uint64_t every, int with_probs,
                                  tasep_stream_fn fn, void *user, tasep_run_result *res) {
    if (!valid_handle(m) || !rc || !res || !fn || every < 1) return fail(TASEP_ERR_INVALID, "bad argument");
    tasep_status s = check_ready(m, rc->h);
    if (s) return s;
    CU_TRY(cudaSetDevice(m->device));
    memset(res, 0, sizeof *res);
    constexpr int K = 2;  // snapshots in flight
    const int n = m->n, na = obs_count(n);
    const size_t pb = with_probs ? sizeof(double) * m->N : 0;
    // device ring (observables, state copy, exit state per slot) and its pinned host mirror
    struct Res {
        double *d_obs = nullptr, *d_x = nullptr;
        ExitState *d_ex = nullptr;
        double *h_obs = nullptr, *h_x = nullptr;
        ExitState *h_ex = nullptr, *h_chk = nullptr;
        cudaStream_t main = nullptr, cp = nullptr;
        cudaEvent_t ready[K] = {}, landed[K] = {}, chk[2] = {};
        ~Res() {  // on every return: nothing in flight may still use the rings
            if (main) cudaStreamSynchronize(main);
            if (cp) cudaStreamSynchronize(cp);
            cudaFree(d_obs); cudaFree(d_x); cudaFree(d_ex);
            cudaFreeHost(h_obs); cudaFreeHost(h_x); cudaFreeHost(h_ex); cudaFreeHost(h_chk);
            for (auto e : ready) if (e) cudaEventDestroy(e);
            for (auto e : landed) if (e) cudaEventDestroy(e);
            for (auto e : chk) if (e) cudaEventDestroy(e);
            if (cp) cudaStreamDestroy(cp);
        }
    } r;
    r.main = m->stream;
    CU_TRY(cudaMalloc(&r.d_obs, sizeof(double) * na * K));
    CU_TRY(cudaMalloc(&r.d_ex, sizeof(ExitState) * K));
    CU_TRY(cudaMallocHost(&r.h_obs, sizeof(double) * na * K));
    CU_TRY(cudaMallocHost(&r.h_ex, sizeof(ExitState) * K));
    CU_TRY(cudaMallocHost(&r.h_chk, sizeof(ExitState) * 2));
    if (pb) {
        CU_TRY(cudaMalloc(&r.d_x, pb * K));
        CU_TRY(cudaMallocHost(&r.h_x, pb * K));
    }
    CU_TRY(cudaStreamCreateWithFlags(&r.cp, cudaStreamNonBlocking));
    for (int k = 0; k < K; ++k) {
        CU_TRY(cudaEventCreateWithFlags(&r.ready[k], cudaEventDisableTiming));
        CU_TRY(cudaEventCreateWithFlags(&r.landed[k], cudaEventDisableTiming));
    }
    for (auto &e : r.chk) CU_TRY(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    std::vector<double> rho(n), cov(size_t(n) * n), mul(size_t(n) * n), w4(n >= 4 ? (n - 3) * 16 : 1);
    struct Snap { int slot; uint64_t step; double t; };
    std::vector<Snap> queue;  // taken, not yet delivered (oldest first)
    bool stopped = false;     // a delivered snapshot showed the loop had ended before it
    auto deliver_oldest = [&]() -> tasep_status {
        const Snap sn = queue.front();
        queue.erase(queue.begin());
        CU_TRY(cudaEventSynchronize(r.landed[sn.slot]));
        const ExitState &e = r.h_ex[sn.slot];
        if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
        if (stopped || e.steps_done <= sn.step) {  // the loop ended before this step
            stopped = true;
            return TASEP_OK;
        }
        obs_convert(n, r.h_obs + size_t(sn.slot) * na, rho.data(), cov.data(), mul.data(), n >= 4 ? w4.data() : nullptr,
                    nullptr);
        fn(m, sn.step, sn.t, rho.data(), cov.data(), mul.data(), n >= 4 ? w4.data() : nullptr,
           pb ? r.h_x + size_t(sn.slot) * m->N : nullptr, user);
        return TASEP_OK;
    };
    const double thresh = rc->stop_tol * rc->h;
    CU_TRY(cudaMemsetAsync(m->ex, 0, sizeof(ExitState), m->stream));
    const int cur0 = m->cur;
    const bool small = m->n <= kSmallMaxN;
    const int shift = 30 - m->n;
    const unsigned long long chunk = shift >= 10 ? 1024ull : (shift <= 2 ? 4ull : (1ull << shift));
    double t = rc->t0;
    unsigned long long i = 0, nsnap = 0, nchunk = 0;
    while (i < rc->steps) {
        // the exit state two chunks back tells whether to go on (one chunk of lookahead)
        if (nchunk >= 2) {
            CU_TRY(cudaEventSynchronize(r.chk[nchunk & 1]));
            const ExitState &e = r.h_chk[nchunk & 1];
            if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
            if (e.done) break;
        }
        const unsigned long long snap = (i + every - 1) / every * every;
        unsigned long long last = std::min<unsigned long long>(snap, rc->steps - 1);
        if (!small) last = std::min(last, i + chunk - 1);
        if (small) {
            if ((s = small_run(m, t, rc->h, last - i + 1, i, thresh, rc->stop_count, rc->exit_rule))) return s;
            for (unsigned long long j = i; j <= last; ++j) t += rc->h;
        } else {
            for (unsigned long long j = i; j <= last; ++j) {
                if ((s = enqueue_step(m, j, t, rc->h, thresh, rc->stop_count, rc->exit_rule))) return s;
                t += rc->h;
            }
        }
        i = last + 1;
        if (last % every == 0) {  // snapshot of step `last`, taken on the device in order
            if (queue.size() == size_t(K) && (s = deliver_oldest())) return s;
            const int slot = int(nsnap % K);
            if ((s = obs_enqueue(m, r.d_obs + size_t(slot) * na, m->stream))) return s;
            if (pb)
                CU_TRY(cudaMemcpyAsync(r.d_x + size_t(slot) * m->N, m->X[m->cur], pb, cudaMemcpyDeviceToDevice,
                                       m->stream));
            CU_TRY(cudaMemcpyAsync(r.d_ex + slot, m->ex, sizeof(ExitState), cudaMemcpyDeviceToDevice, m->stream));
            CU_TRY(cudaEventRecord(r.ready[slot], m->stream));
            // to the host on the copy stream, while the integration goes on
            CU_TRY(cudaStreamWaitEvent(r.cp, r.ready[slot], 0));
            CU_TRY(cudaMemcpyAsync(r.h_obs + size_t(slot) * na, r.d_obs + size_t(slot) * na, sizeof(double) * na,
                                   cudaMemcpyDeviceToHost, r.cp));
            CU_TRY(cudaMemcpyAsync(r.h_ex + slot, r.d_ex + slot, sizeof(ExitState), cudaMemcpyDeviceToHost, r.cp));
            if (pb)
                CU_TRY(cudaMemcpyAsync(r.h_x + size_t(slot) * m->N, r.d_x + size_t(slot) * m->N, pb,
                                       cudaMemcpyDeviceToHost, r.cp));
            CU_TRY(cudaEventRecord(r.landed[slot], r.cp));
            queue.push_back({slot, last, t});
            ++nsnap;
        }
        CU_TRY(cudaMemcpyAsync(r.h_chk + (nchunk & 1), m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost, m->stream));
        CU_TRY(cudaEventRecord(r.chk[nchunk & 1], m->stream));
        ++nchunk;
        // hand over snapshots that have landed, without waiting for the others
        while (!queue.empty() && cudaEventQuery(r.landed[queue.front().slot]) == cudaSuccess)
            if ((s = deliver_oldest())) return s;
    }
    CU_TRY(cudaStreamSynchronize(m->stream));
    while (!queue.empty())
        if ((s = deliver_oldest())) return s;
    if (m->prof && (s = prof_flush(m))) return s;
    CU_TRY(cudaMemcpy(m->ex_host, m->ex, sizeof(ExitState), cudaMemcpyDeviceToHost));
    const ExitState &e = *m->ex_host;
    if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired during the integration");
    const unsigned long long done = e.steps_done;
    if (m->integrator == TASEP_INTEGRATOR_REF && !small) m->cur = int((cur0 + done) & 1ull);
    res->steps_done = done;
    res->steps_at_stop = e.steps_at_stop;
    res->early_stop = e.early_stop;
    res->converged = e.converged;
    res->last_checksum = e.last_checksum;
    double tt = rc->t0;
    for (unsigned long long k = 0; k < done; ++k) tt += rc->h;
    res->t_end = tt;
    return TASEP_OK;
}

void *tasep_meq_stream(const tasep_meq *m) { return m ? static_cast<void *>(m->stream) : nullptr; }

tasep_status tasep_meq_set_cache_policy(tasep_meq *m, int near_bits, int flags) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    if (near_bits < 0 || near_bits > 64 || (flags & ~(TASEP_L2_OWN_FIRST | TASEP_L2_DEMOTE | TASEP_L2_FAR_FIRST)))
        return fail(TASEP_ERR_INVALID, "cache policy near_bits=%d flags=%d out of range", near_bits, flags);
    m->l2_near = near_bits;
    m->l2_flags = flags;
    return TASEP_OK;
}

tasep_status tasep_meq_get_cache_policy(const tasep_meq *m, int *near_bits, int *flags) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    if (near_bits) *near_bits = m->l2_near;
    if (flags) *flags = m->l2_flags;
    return TASEP_OK;
}

tasep_status tasep_meq_profile(tasep_meq *m, int enable) {
    if (!valid_handle(m)) return fail(TASEP_ERR_INVALID, "null handle");
    if (m->prof) {
        tasep_status s = prof_flush(m);
        if (s) return s;
    }
    m->prof = enable != 0;
    memset(m->prof_ms, 0, sizeof m->prof_ms);
    memset(m->prof_n, 0, sizeof m->prof_n);
    return TASEP_OK;
}

tasep_status tasep_meq_profile_read(tasep_meq *m, const char **names, double *ms, uint64_t *launches, int cap,
                                    int *count) {
    if (!valid_handle(m) || !count) return fail(TASEP_ERR_INVALID, "null argument");
    CU_TRY(cudaSetDevice(m->device));
    CU_TRY(cudaStreamSynchronize(m->stream));
    tasep_status s = prof_flush(m);
    if (s) return s;
    int c = 0;
    for (int k = 0; k < ST_COUNT + kProfSlots; ++k) {
        if (!m->prof_n[k]) continue;
        if (c < cap) {
            if (names) names[c] = k < ST_COUNT ? kStageNames[k] : kExtraNames[k - ST_COUNT];
            if (ms) ms[c] = m->prof_ms[k];
            if (launches) launches[c] = m->prof_n[k];
        }
        ++c;
    }
    *count = c;
    return TASEP_OK;
}

// ---- device-pointer operators -----------------------------------------------

tasep_status tasep_apply_device(int n, const double *rates, const double *x, double *y, void *stream) {
    if (n < 1 || n > TASEP_MAX_N || !rates || !x || !y) return fail(TASEP_ERR_INVALID, "bad argument");
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    DevScratch *sc = nullptr;
    tasep_status s = get_scratch(dev, &sc);
    if (s) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n <= kSmallMaxN) {
        SmallParams sp;
        memset(&sp, 0, sizeof sp);
        sp.n = n;
        sp.mode = SM_APPLY;
        sp.x_in = x;
        sp.x_out = y;
        sp.ex = sc->ex;
        fill_const_rates(sp.rs, n, rates);
        return launch_small<double>(sp, st);
    }
    TileParams p;
    memset(&p, 0, sizeof p);
    p.n = n;
    p.l2_near = g_l2_near_default;
    p.l2_flags = g_l2_flags_default;
    apply_test_hook(p);
    p.ntiles = (1ull << n) >> kTileBits;
    p.g = x;
    p.out = y;
    p.ex = sc->ex;
    p.partials = sc->partials;
    p.counter = sc->counter;
    fill_const_rates(p.rs, n, rates);
    const int grid = int(std::min<unsigned long long>(p.ntiles, sc->nsm));
    return launch_tile<ST_APPLY, double>(p, grid, st);
}

tasep_status tasep_step_ref_device(int n, const double *rates, double h, const double *x, double *x_out,
                                   double *checksum_host, void *stream) {
    if (n < 1 || n > TASEP_MAX_N || !rates || !x || !x_out) return fail(TASEP_ERR_INVALID, "bad argument");
    if (x == x_out) return fail(TASEP_ERR_INVALID, "x and x_out must not overlap");
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    DevScratch *sc = nullptr;
    tasep_status s = get_scratch(dev, &sc);
    if (s) return s;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    CU_TRY(cudaMemsetAsync(sc->ex, 0, sizeof(ExitState), st));
    if (n <= kSmallMaxN) {
        SmallParams sp;
        memset(&sp, 0, sizeof sp);
        sp.n = n;
        sp.mode = SM_RUN;
        sp.integrator = SI_REF;
        sp.x_in = x;
        sp.x_out = x_out;
        sp.h = h;
        sp.max_steps = 1;
        sp.ex = sc->ex;
        fill_const_rates(sp.rs, n, rates);
        if ((s = launch_small<double>(sp, st))) return s;
    } else {
        TileParams p;
        memset(&p, 0, sizeof p);
        p.n = n;
        p.l2_near = g_l2_near_default;
        p.l2_flags = g_l2_flags_default;
        apply_test_hook(p);
        p.ntiles = (1ull << n) >> kTileBits;
        p.g = x;
        p.out = x_out;
        p.h = h;
        p.ex = sc->ex;
        p.partials = sc->partials;
        p.counter = sc->counter;
        fill_const_rates(p.rs, n, rates);
        const int grid = int(std::min<unsigned long long>(p.ntiles, sc->nsm));
        if ((s = launch_tile<ST_REF, double>(p, grid, st))) return s;
    }
    if (checksum_host) {
        ExitState e;
        CU_TRY(cudaMemcpyAsync(&e, sc->ex, sizeof e, cudaMemcpyDeviceToHost, st));
        CU_TRY(cudaStreamSynchronize(st));
        if (e.error) return fail(TASEP_ERR_TIMEOUT, "a bounded device wait expired");
        *checksum_host = e.last_checksum;
    }
    return TASEP_OK;
}

}  // extern "C"

// ---- reference step without any device allocation ----------------------------
// The scratch of the L1 norm lives in this file-scope device array instead of
// memory from cudaMalloc.  Host code must not pass the array's name to a
// kernel (on the host it only stands for the symbol); the device address is
// looked up once per device with cudaGetSymbolAddress.
namespace {
constexpr int kNoAllocMaxCtas = 1024;
struct NoAllocScratch {
    ExitState ex;       // status and L1 norm of the last step
    unsigned counter;   // last-CTA ticket
    unsigned pad[15];
    double partials[kNoAllocMaxCtas];
};
std::mutex g_noalloc_mu;
NoAllocScratch *g_noalloc_addr[64] = {};
int g_noalloc_nsm[64] = {};
}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[sizeof(NoAllocScratch)];

extern "C" tasep_status tasep_step_ref_device_noalloc(int n, const double *rates, double h, const double *x,
                                                      double *x_out, double *checksum_dev, void *stream) {
    if (n < 1 || n > TASEP_MAX_N || !rates || !x || !x_out) return fail(TASEP_ERR_INVALID, "bad argument");
    if (x == x_out) return fail(TASEP_ERR_INVALID, "x and x_out must not overlap");
    int dev = 0;
    CU_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return fail(TASEP_ERR_INVALID, "device ordinal %d out of range", dev);
    NoAllocScratch *sc = nullptr;
    int nsm = 0;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_addr[dev]) {  // set-up on the first call on this device
            void *addr = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
            if (e != cudaSuccess || addr == nullptr)
                return fail(TASEP_ERR_CUDA, "cudaGetSymbolAddress of the static scratch failed: %s",
                            cudaGetErrorString(e));
            CU_TRY(cudaDeviceGetAttribute(&g_noalloc_nsm[dev], cudaDevAttrMultiProcessorCount, dev));
            g_noalloc_addr[dev] = static_cast<NoAllocScratch *>(addr);
        }
        sc = g_noalloc_addr[dev];
        nsm = g_noalloc_nsm[dev];
    }
    const unsigned long long ntiles = n > kSmallMaxN ? ((1ull << n) >> kTileBits) : 1ull;
    const int grid = int(std::min<unsigned long long>(ntiles, (unsigned long long)nsm));
    if (grid > kNoAllocMaxCtas)
        return fail(TASEP_ERR_INVALID,
                    "the step needs %d CTAs but the static scratch holds %d per-CTA partial sums", grid,
                    kNoAllocMaxCtas);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the array keeps the previous call's contents: clear the status and the ticket
    CU_TRY(cudaMemsetAsync(sc, 0, offsetof(NoAllocScratch, partials), st));
    tasep_status s;
    if (n <= kSmallMaxN) {
        SmallParams sp;
        memset(&sp, 0, sizeof sp);
        sp.n = n;
        sp.mode = SM_RUN;
        sp.integrator = SI_REF;
        sp.x_in = x;
        sp.x_out = x_out;
        sp.h = h;
        sp.max_steps = 1;
        sp.ex = &sc->ex;
        fill_const_rates(sp.rs, n, rates);
        s = launch_small<double>(sp, st);
    } else {
        TileParams p;
        memset(&p, 0, sizeof p);
        p.n = n;
        p.l2_near = g_l2_near_default;
        p.l2_flags = g_l2_flags_default;
        apply_test_hook(p);
        p.ntiles = ntiles;
        p.g = x;
        p.out = x_out;
        p.h = h;
        p.ex = &sc->ex;
        p.partials = sc->partials;
        p.counter = &sc->counter;
        fill_const_rates(p.rs, n, rates);
        s = launch_tile<ST_REF, double>(p, grid, st);
    }
    if (s) return s;
    if (checksum_dev)
        CU_TRY(cudaMemcpyAsync(checksum_dev, &sc->ex.last_checksum, sizeof(double), cudaMemcpyDeviceToDevice, st));
    return TASEP_OK;
}

#include "tasep_batch_impl.cuh"

#include "tasep_mlp_impl.cuh"
