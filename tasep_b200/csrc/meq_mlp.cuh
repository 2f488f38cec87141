// meq_mlp.cuh - the per-site surrogate network and the pair-Markov initial
// measure of the learned warm start.
//
// Network: 16 inputs (a window of 9 rates around the site, inverse distances to
// both ends, the boundary rates, and the mean-field densities of the site and
// its two neighbours; the host builds them), three hidden layers of 64 tanh
// units, 2 linear outputs (the site's density and its nearest-neighbour
// covariance).  The forward and backward passes use BF16 copies of
// the weights and accumulate in FP32; Adam updates FP32 master weights and
// refreshes the BF16 copies.  Each CTA writes its gradient to its own row and
// a second kernel adds the rows in CTA order, so training is deterministic.
//
// Pair-Markov measure: P(tau) = P(tau_0) prod_j P(tau_(j+1) | tau_j) built from
// predicted densities and nearest-neighbour joint probabilities; it sums to 1
// by construction and has the predicted one- and two-site marginals.  Site j
// is bit n-1-j of the state index, as everywhere else.
#pragma once

#include <cuda_bf16.h>

#include "meq_common.cuh"

namespace tasep {

constexpr int kMlpIn = 16, kMlpHid = 64, kMlpOut = 2;
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpHid * kMlpIn;
constexpr int kMlpW2 = kMlpB1 + kMlpHid, kMlpB2 = kMlpW2 + kMlpHid * kMlpHid;
constexpr int kMlpW3 = kMlpB2 + kMlpHid, kMlpB3 = kMlpW3 + kMlpHid * kMlpHid;
constexpr int kMlpW4 = kMlpB3 + kMlpHid, kMlpB4 = kMlpW4 + kMlpOut * kMlpHid;
constexpr int kMlpParams = kMlpB4 + kMlpOut;  // 9538
__device__ __forceinline__ float bf(const __nv_bfloat16 *w, int i) { return __bfloat162float(w[i]); }

constexpr int kMlpTile = 128;   // samples per CTA pass: the M of one tcgen05.mma, one sample per TMEM lane
constexpr int kMlpThreads = 128; // one warpgroup: thread t owns sample row t (TMEM lane t)
constexpr int kMlpTmemCols = 64; // FP32 accumulator of a 128 x 64 layer output

// ---- tcgen05 helpers ----------------------------------------------------------
//
// Operands live in shared memory in the no-swizzle K-major layout: 8x8 core
// matrices of 128 contiguous bytes (8 rows of 16 bytes); core matrices adjacent
// along K are 128 B apart (leading byte offset), 8-row groups K/8*128 B apart
// (stride byte offset).  One kind::f16 MMA consumes K = 16, two core matrices.

__device__ __forceinline__ int kmaj(int r, int k, int K) {  // element offset of (r, k) in an R x K operand
    return (((r >> 3) * (K >> 3) + (k >> 3)) << 6) + ((r & 7) << 3) + (k & 7);
}

__device__ __forceinline__ uint64_t umma_desc(const void *base, int K) {
    const uint64_t a = smem_u32(base);
    return ((a & 0x3FFFFull) >> 4) | (uint64_t(128 >> 4) << 16) | (uint64_t((K >> 3) * 128 >> 4) << 32) |
           (1ull << 46);  // descriptor version of sm_100; layout type 0 = no swizzle
}

// kind::f16 instruction descriptor: BF16 A and B (K-major), FP32 accumulator, M x N.
template <int M, int N> __device__ __forceinline__ constexpr uint32_t umma_idesc_bf16() {
    return (1u << 4) | (1u << 7) | (1u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
    const uint32_t no_mask = 0;  // no output lane disabled
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(tmem_d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate), "r"(no_mask));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
                 : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 consecutive FP32 columns of this thread's TMEM lane.
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float *v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared state of the tensor-core forward pass.  A value a enters an MMA as two
// BF16 operands, hi = bf16(a) and lo = bf16(a - hi) (16 significant bits), so
// the products with the BF16 weights are accurate to ~1e-5 and accumulate in
// FP32 in tensor memory.
struct MlpTc {
    __nv_bfloat16 ahi[kMlpTile * kMlpHid];  // layer input, hi part (K-major)
    __nv_bfloat16 alo[kMlpTile * kMlpHid];  // layer input, lo part
    __nv_bfloat16 w1[kMlpHid * kMlpIn];     // weights, K-major (N = 64 rows)
    __nv_bfloat16 w2[kMlpHid * kMlpHid];
    __nv_bfloat16 w3[kMlpHid * kMlpHid];
    float bias[3][kMlpHid];
    float w4[kMlpOut][kMlpHid];
    float b4[kMlpOut];
    uint64_t bar;    // MMA completion
    uint32_t tmem;   // accumulator base address
    int err;
};

// Per-thread-row activations kept for the backward pass.
struct MlpKeep {
    float x[kMlpTile][kMlpIn];
    float h1[kMlpTile][kMlpHid], h2[kMlpTile][kMlpHid], h3[kMlpTile][kMlpHid];
};

// Backward-pass buffers of the gradient kernel.
struct MlpBack {
    float gy[kMlpTile][kMlpOut];
    float g3[kMlpTile][kMlpHid], g2[kMlpTile][kMlpHid];
};

__device__ __forceinline__ void split_store(MlpTc &s, int r, int k, int K, float a) {
    const __nv_bfloat16 hi = __float2bfloat16(a);
    const int o = kmaj(r, k, K);
    s.ahi[o] = hi;
    s.alo[o] = __float2bfloat16(a - __bfloat162float(hi));
}

// Weights into shared memory (once per CTA), TMEM allocation by warp 0.
__device__ void tc_setup(MlpTc &s, const __nv_bfloat16 *w) {
    const int t = threadIdx.x;
    for (int e = t; e < kMlpHid * kMlpIn; e += kMlpThreads) s.w1[kmaj(e / kMlpIn, e % kMlpIn, kMlpIn)] = w[kMlpW1 + e];
    for (int e = t; e < kMlpHid * kMlpHid; e += kMlpThreads) {
        s.w2[kmaj(e / kMlpHid, e % kMlpHid, kMlpHid)] = w[kMlpW2 + e];
        s.w3[kmaj(e / kMlpHid, e % kMlpHid, kMlpHid)] = w[kMlpW3 + e];
    }
    for (int e = t; e < kMlpHid; e += kMlpThreads) {
        s.bias[0][e] = bf(w, kMlpB1 + e);
        s.bias[1][e] = bf(w, kMlpB2 + e);
        s.bias[2][e] = bf(w, kMlpB3 + e);
    }
    for (int e = t; e < kMlpOut * kMlpHid; e += kMlpThreads) s.w4[e / kMlpHid][e % kMlpHid] = bf(w, kMlpW4 + e);
    if (t < kMlpOut) s.b4[t] = bf(w, kMlpB4 + t);
    if (t == 0) {
        mbar_init(&s.bar, 1);
        s.err = 0;
        fence_mbar_init();
    }
    if ((t >> 5) == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s.tmem)),
                     "r"(kMlpTmemCols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // weights are read by the tensor cores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
}

__device__ void tc_teardown(MlpTc &s) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if ((threadIdx.x >> 5) == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(s.tmem), "r"(kMlpTmemCols)
                     : "memory");
}

// One hidden layer on the tensor cores: D[128 x 64] = (hi + lo)[128 x K] W^T,
// the input already stored; then this thread's row of D (+ bias, tanh) into
// out[64].  Returns false if the MMA did not complete within the wait limit.
template <int K>
__device__ bool tc_layer(MlpTc &s, const __nv_bfloat16 *W, const float *bias, uint32_t &phase, float *out) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // the input rows were generic stores
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        constexpr uint32_t idesc = umma_idesc_bf16<kMlpTile, kMlpHid>();
#pragma unroll
        for (int k = 0; k < K / 16; ++k) {
            const uint64_t bd = umma_desc(W + k * 128, K);  // two core matrices (16 K values) per step
            umma_bf16(s.tmem, umma_desc(s.ahi + k * 128, K), bd, idesc, k > 0);
            umma_bf16(s.tmem, umma_desc(s.alo + k * 128, K), bd, idesc, 1);
        }
        umma_commit(&s.bar);
    }
    volatile int *errf = &s.err;
    const bool ok = mbar_wait(&s.bar, phase, errf);
    phase ^= 1;
    if (!__syncthreads_and(ok)) return false;  // every thread takes the same path
    tc_fence_after();
    const uint32_t lane_base = s.tmem + ((uint32_t(threadIdx.x) & ~31u) << 16);
    tmem_ld32(lane_base, out);
    tmem_ld32(lane_base + 32, out + 32);
#pragma unroll
    for (int i = 0; i < kMlpHid; ++i) out[i] = tanhf(out[i] + bias[i]);
    return true;
}

// Forward pass of this thread's sample (row r of the tile; rows past the end
// carry zeros): h1..h3 (kept if keep != nullptr) and the two outputs.
__device__ bool tc_forward(MlpTc &s, const float *xrow, bool valid, uint32_t &phase, MlpKeep *keep, float *y) {
    const int r = threadIdx.x;
    float h[kMlpHid];
#pragma unroll
    for (int k = 0; k < kMlpIn; ++k) {
        const float v = valid ? xrow[k] : 0.f;
        split_store(s, r, k, kMlpIn, v);
        if (keep) keep->x[r][k] = v;
    }
    if (!tc_layer<kMlpIn>(s, s.w1, s.bias[0], phase, h)) return false;
#pragma unroll
    for (int k = 0; k < kMlpHid; ++k) {
        split_store(s, r, k, kMlpHid, h[k]);
        if (keep) keep->h1[r][k] = h[k];
    }
    if (!tc_layer<kMlpHid>(s, s.w2, s.bias[1], phase, h)) return false;
#pragma unroll
    for (int k = 0; k < kMlpHid; ++k) {
        split_store(s, r, k, kMlpHid, h[k]);
        if (keep) keep->h2[r][k] = h[k];
    }
    if (!tc_layer<kMlpHid>(s, s.w3, s.bias[2], phase, h)) return false;
    // 64 -> 2 output layer: too narrow for an MMA (N >= 8), done in registers
#pragma unroll
    for (int o = 0; o < kMlpOut; ++o) {
        float acc = s.b4[o];
#pragma unroll
        for (int i = 0; i < kMlpHid; ++i) acc = fmaf(h[i], s.w4[o][i], acc);
        y[o] = acc;
    }
    if (keep)
#pragma unroll
        for (int k = 0; k < kMlpHid; ++k) keep->h3[r][k] = h[k];
    return true;
}

// Inference: y[n][2] for n samples, 128 per CTA pass.
__global__ void __launch_bounds__(kMlpThreads) mlp_forward_kernel(const __nv_bfloat16 *w, const float *x, float *y,
                                                                  int n, int *err) {
    extern __shared__ __align__(128) unsigned char mlp_smem[];
    MlpTc &s = *reinterpret_cast<MlpTc *>(mlp_smem);
    tc_setup(s, w);
    uint32_t phase = 0;
    for (int b0 = blockIdx.x * kMlpTile; b0 < n; b0 += gridDim.x * kMlpTile) {
        const int r = b0 + threadIdx.x;
        float yo[kMlpOut];
        if (!tc_forward(s, x + size_t(r) * kMlpIn, r < n, phase, nullptr, yo)) {  // uniform over the CTA
            if (threadIdx.x == 0) atomicExch(err, 1);
            break;
        }
        if (r < n)
            for (int o = 0; o < kMlpOut; ++o) y[size_t(r) * kMlpOut + o] = yo[o];
    }
    if (s.err) mbar_drain(&s.bar, phase ^ 1, 100000000ull);  // an MMA still in flight must land first
    tc_teardown(s);
}

// Loss = sum over samples and outputs of ow[o] * (y - t)^2 / n.  CTA c takes
// samples [128c, 128c + 128): forward on the tensor cores, backward in FP32
// on the CUDA cores; its gradient goes to grad[c][...], its loss share to
// loss[c].
__global__ void __launch_bounds__(kMlpThreads) mlp_grad_kernel(const __nv_bfloat16 *w, const float *x,
                                                               const float *t, int n, float ow0, float ow1,
                                                               float *grad, float *loss, int *err) {
    extern __shared__ __align__(128) unsigned char mlp_smem[];
    MlpTc &s = *reinterpret_cast<MlpTc *>(mlp_smem);
    MlpKeep &kp = *reinterpret_cast<MlpKeep *>(mlp_smem + sizeof(MlpTc));
    MlpBack &bk = *reinterpret_cast<MlpBack *>(mlp_smem + sizeof(MlpTc) + sizeof(MlpKeep));
    __shared__ float lsum[kMlpThreads];
    float *g = grad + size_t(blockIdx.x) * kMlpParams;
    tc_setup(s, w);
    const int b0 = blockIdx.x * kMlpTile, nb = min(kMlpTile, n - b0), r = threadIdx.x;
    uint32_t phase = 0;
    float yo[kMlpOut];
    const bool ok = tc_forward(s, x + size_t(b0 + r) * kMlpIn, r < nb, phase, &kp, yo);  // uniform
    if (!ok) {
        if (r == 0) atomicExch(err, 1);
        mbar_drain(&s.bar, phase ^ 1, 100000000ull);  // an MMA still in flight must land first
    }
    tc_teardown(s);
    if (!ok) return;
    // output layer: dL/dy = 2 ow (y - t) / n
    const float inv_n = 1.f / float(n);
    float lacc = 0.f;
    for (int o = 0; o < kMlpOut; ++o) {
        float gyo = 0.f;
        if (r < nb) {
            const float d = yo[o] - t[size_t(b0 + r) * kMlpOut + o];
            const float owo = o == 0 ? ow0 : ow1;
            lacc += owo * d * d * inv_n;
            gyo = 2.f * owo * d * inv_n;
        }
        bk.gy[r][o] = gyo;
    }
    __syncthreads();
    // W4, b4 and dL/dh3
    for (int e = r; e < kMlpOut * kMlpHid; e += kMlpThreads) {
        const int o = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc = fmaf(bk.gy[b][o], kp.h3[b][i], acc);
        g[kMlpW4 + e] = acc;
    }
    if (r < kMlpOut) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += bk.gy[b][r];
        g[kMlpB4 + r] = acc;
    }
    for (int e = r; e < nb * kMlpHid; e += kMlpThreads) {
        const int b = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int o = 0; o < kMlpOut; ++o) acc = fmaf(bk.gy[b][o], bf(w + kMlpW4, o * kMlpHid + i), acc);
        bk.g3[b][i] = acc * (1.f - kp.h3[b][i] * kp.h3[b][i]);  // through tanh
    }
    __syncthreads();
    // W3, b3 and dL/dh2 (into g2 through tanh)
    for (int e = r; e < kMlpHid * kMlpHid; e += kMlpThreads) {
        const int o = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc = fmaf(bk.g3[b][o], kp.h2[b][i], acc);
        g[kMlpW3 + e] = acc;
    }
    for (int o = r; o < kMlpHid; o += kMlpThreads) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += bk.g3[b][o];
        g[kMlpB3 + o] = acc;
    }
    for (int e = r; e < nb * kMlpHid; e += kMlpThreads) {
        const int b = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int o = 0; o < kMlpHid; ++o) acc = fmaf(bk.g3[b][o], bf(w + kMlpW3, o * kMlpHid + i), acc);
        bk.g2[b][i] = acc * (1.f - kp.h2[b][i] * kp.h2[b][i]);
    }
    __syncthreads();
    // W2, b2 and dL/dh1 (into g3, now free)
    for (int e = r; e < kMlpHid * kMlpHid; e += kMlpThreads) {
        const int o = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc = fmaf(bk.g2[b][o], kp.h1[b][i], acc);
        g[kMlpW2 + e] = acc;
    }
    for (int o = r; o < kMlpHid; o += kMlpThreads) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += bk.g2[b][o];
        g[kMlpB2 + o] = acc;
    }
    __syncthreads();
    for (int e = r; e < nb * kMlpHid; e += kMlpThreads) {
        const int b = e / kMlpHid, i = e % kMlpHid;
        float acc = 0.f;
        for (int o = 0; o < kMlpHid; ++o) acc = fmaf(bk.g2[b][o], bf(w + kMlpW2, o * kMlpHid + i), acc);
        bk.g3[b][i] = acc * (1.f - kp.h1[b][i] * kp.h1[b][i]);
    }
    __syncthreads();
    // W1, b1
    for (int e = r; e < kMlpHid * kMlpIn; e += kMlpThreads) {
        const int o = e / kMlpIn, i = e % kMlpIn;
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc = fmaf(bk.g3[b][o], kp.x[b][i], acc);
        g[kMlpW1 + e] = acc;
    }
    for (int o = r; o < kMlpHid; o += kMlpThreads) {
        float acc = 0.f;
        for (int b = 0; b < nb; ++b) acc += bk.g3[b][o];
        g[kMlpB1 + o] = acc;
    }
    lsum[r] = lacc;
    __syncthreads();
    if (r == 0) {
        float tot = 0.f;
        for (int i = 0; i < kMlpThreads; ++i) tot += lsum[i];
        loss[blockIdx.x] = tot;
    }
}

constexpr size_t kMlpForwardSmem = sizeof(MlpTc);
constexpr size_t kMlpGradSmem = sizeof(MlpTc) + sizeof(MlpKeep) + sizeof(MlpBack);

// Adds the per-CTA gradient rows in CTA order.
__global__ void mlp_reduce_kernel(const float *grad, int rows, float *out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kMlpParams; e += gridDim.x * blockDim.x) {
        float s = 0.f;
        for (int r = 0; r < rows; ++r) s += grad[size_t(r) * kMlpParams + e];
        out[e] = s;
    }
}

// Adam step on the FP32 master weights; refreshes the BF16 copies.
__global__ void mlp_adam_kernel(float *master, __nv_bfloat16 *w, float *m1, float *m2, const float *g, float lr,
                                float b1, float b2, float eps, float c1, float c2) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kMlpParams; e += gridDim.x * blockDim.x) {
        const float gi = g[e];
        const float a = b1 * m1[e] + (1.f - b1) * gi;
        const float v = b2 * m2[e] + (1.f - b2) * gi * gi;
        m1[e] = a;
        m2[e] = v;
        const float p = master[e] - lr * (a / c1) / (sqrtf(v / c2) + eps);
        master[e] = p;
        w[e] = __float2bfloat16(p);
    }
}

__global__ void mlp_to_bf16_kernel(const float *master, __nv_bfloat16 *w) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kMlpParams; e += gridDim.x * blockDim.x)
        w[e] = __float2bfloat16(master[e]);
}

// P(tau) = p0[tau_0] * prod_j T_j[tau_j][tau_(j+1)]; T holds the n-1 transition
// matrices (4 doubles each, row = tau_j), p0 the distribution of site 0.
__global__ void pair_markov_kernel(int n, const double *p0, const double *T, double *x) {
    const unsigned long long N = 1ull << n;
    for (unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; i < N;
         i += (unsigned long long)gridDim.x * blockDim.x) {
        int prev = int((i >> (n - 1)) & 1);
        double v = p0[prev];
        for (int j = 0; j + 1 < n; ++j) {
            const int cur = int((i >> (n - 2 - j)) & 1);
            v *= T[4 * j + 2 * prev + cur];
            prev = cur;
        }
        x[i] = v;
    }
}

}  // namespace tasep
