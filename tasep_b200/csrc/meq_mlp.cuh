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
constexpr int kMlpBatch = 64;                 // samples per CTA per pass
constexpr int kMlpThreads = 256;

struct MlpSmem {
    float x[kMlpBatch][kMlpIn];
    float h1[kMlpBatch][kMlpHid], h2[kMlpBatch][kMlpHid], h3[kMlpBatch][kMlpHid];
    float y[kMlpBatch][kMlpOut];
    float g3[kMlpBatch][kMlpHid], g2[kMlpBatch][kMlpHid];
};

__device__ __forceinline__ float bf(const __nv_bfloat16 *w, int i) { return __bfloat162float(w[i]); }

// out[b][o] = act(sum_i in[b][i] * W[o][i] + bias[o]) for the CTA's batch.
template <int IN, int OUT, bool TANH>
__device__ __forceinline__ void mlp_layer(const float (*in)[IN], float (*out)[OUT], const __nv_bfloat16 *W,
                                          const __nv_bfloat16 *bias, int nb) {
    for (int e = threadIdx.x; e < nb * OUT; e += blockDim.x) {
        const int b = e / OUT, o = e % OUT;
        float acc = bf(bias, o);
        const __nv_bfloat16 *w = W + o * IN;
#pragma unroll 8
        for (int i = 0; i < IN; ++i) acc = fmaf(in[b][i], bf(w, i), acc);
        out[b][o] = TANH ? tanhf(acc) : acc;
    }
}

__device__ void mlp_forward_block(MlpSmem &s, const __nv_bfloat16 *w, int nb) {
    mlp_layer<kMlpIn, kMlpHid, true>(s.x, s.h1, w + kMlpW1, w + kMlpB1, nb);
    __syncthreads();
    mlp_layer<kMlpHid, kMlpHid, true>(s.h1, s.h2, w + kMlpW2, w + kMlpB2, nb);
    __syncthreads();
    mlp_layer<kMlpHid, kMlpHid, true>(s.h2, s.h3, w + kMlpW3, w + kMlpB3, nb);
    __syncthreads();
    mlp_layer<kMlpHid, kMlpOut, false>(s.h3, s.y, w + kMlpW4, w + kMlpB4, nb);
    __syncthreads();
}

// Inference: y[n][2] for n samples.
__global__ void __launch_bounds__(kMlpThreads) mlp_forward_kernel(const __nv_bfloat16 *w, const float *x, float *y,
                                                                  int n) {
    extern __shared__ __align__(16) unsigned char mlp_smem[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(mlp_smem);
    for (int b0 = blockIdx.x * kMlpBatch; b0 < n; b0 += gridDim.x * kMlpBatch) {
        const int nb = min(kMlpBatch, n - b0);
        for (int e = threadIdx.x; e < nb * kMlpIn; e += blockDim.x) s.x[e / kMlpIn][e % kMlpIn] = x[size_t(b0) * kMlpIn + e];
        __syncthreads();
        mlp_forward_block(s, w, nb);
        for (int e = threadIdx.x; e < nb * kMlpOut; e += blockDim.x) y[size_t(b0) * kMlpOut + e] = s.y[e / kMlpOut][e % kMlpOut];
        __syncthreads();
    }
}

// Loss = sum over samples and outputs of ow[o] * (y - t)^2 / n; this CTA's
// gradient goes to grad[blockIdx.x][...] and its loss share to loss[blockIdx.x].
__global__ void __launch_bounds__(kMlpThreads) mlp_grad_kernel(const __nv_bfloat16 *w, const float *x,
                                                               const float *t, int n, float ow0, float ow1,
                                                               float *grad, float *loss) {
    extern __shared__ __align__(16) unsigned char mlp_smem[];
    MlpSmem &s = *reinterpret_cast<MlpSmem *>(mlp_smem);
    float *g = grad + size_t(blockIdx.x) * kMlpParams;
    for (int e = threadIdx.x; e < kMlpParams; e += blockDim.x) g[e] = 0.f;
    __shared__ float lsum[kMlpThreads];
    float lacc = 0.f;
    const float inv_n = 1.f / float(n);
    __syncthreads();
    for (int b0 = blockIdx.x * kMlpBatch; b0 < n; b0 += gridDim.x * kMlpBatch) {
        const int nb = min(kMlpBatch, n - b0);
        for (int e = threadIdx.x; e < nb * kMlpIn; e += blockDim.x) s.x[e / kMlpIn][e % kMlpIn] = x[size_t(b0) * kMlpIn + e];
        __syncthreads();
        mlp_forward_block(s, w, nb);
        // output layer: dL/dy = 2 ow (y - t) / n (kept in s.y)
        for (int e = threadIdx.x; e < nb * kMlpOut; e += blockDim.x) {
            const int b = e / kMlpOut, o = e % kMlpOut;
            const float d = s.y[b][o] - t[size_t(b0 + b) * kMlpOut + o];
            const float ow = o == 0 ? ow0 : ow1;
            lacc += ow * d * d * inv_n;
            s.y[b][o] = 2.f * ow * d * inv_n;
        }
        __syncthreads();
        // W4, b4 and dL/dh3
        for (int e = threadIdx.x; e < kMlpOut * kMlpHid; e += blockDim.x) {
            const int o = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc = fmaf(s.y[b][o], s.h3[b][i], acc);
            g[kMlpW4 + e] += acc;
        }
        if (threadIdx.x < kMlpOut) {
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc += s.y[b][threadIdx.x];
            g[kMlpB4 + threadIdx.x] += acc;
        }
        for (int e = threadIdx.x; e < nb * kMlpHid; e += blockDim.x) {
            const int b = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int o = 0; o < kMlpOut; ++o) acc = fmaf(s.y[b][o], bf(w + kMlpW4, o * kMlpHid + i), acc);
            s.g3[b][i] = acc * (1.f - s.h3[b][i] * s.h3[b][i]);  // through tanh
        }
        __syncthreads();
        // W3, b3 and dL/dh2 (into g2 through tanh)
        for (int e = threadIdx.x; e < kMlpHid * kMlpHid; e += blockDim.x) {
            const int o = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc = fmaf(s.g3[b][o], s.h2[b][i], acc);
            g[kMlpW3 + e] += acc;
        }
        for (int o = threadIdx.x; o < kMlpHid; o += blockDim.x) {
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc += s.g3[b][o];
            g[kMlpB3 + o] += acc;
        }
        for (int e = threadIdx.x; e < nb * kMlpHid; e += blockDim.x) {
            const int b = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int o = 0; o < kMlpHid; ++o) acc = fmaf(s.g3[b][o], bf(w + kMlpW3, o * kMlpHid + i), acc);
            s.g2[b][i] = acc * (1.f - s.h2[b][i] * s.h2[b][i]);
        }
        __syncthreads();
        // W2, b2 and dL/dh1 (into g3, now free)
        for (int e = threadIdx.x; e < kMlpHid * kMlpHid; e += blockDim.x) {
            const int o = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc = fmaf(s.g2[b][o], s.h1[b][i], acc);
            g[kMlpW2 + e] += acc;
        }
        for (int o = threadIdx.x; o < kMlpHid; o += blockDim.x) {
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc += s.g2[b][o];
            g[kMlpB2 + o] += acc;
        }
        for (int e = threadIdx.x; e < nb * kMlpHid; e += blockDim.x) {
            const int b = e / kMlpHid, i = e % kMlpHid;
            float acc = 0.f;
            for (int o = 0; o < kMlpHid; ++o) acc = fmaf(s.g2[b][o], bf(w + kMlpW2, o * kMlpHid + i), acc);
            s.g3[b][i] = acc * (1.f - s.h1[b][i] * s.h1[b][i]);
        }
        __syncthreads();
        // W1, b1
        for (int e = threadIdx.x; e < kMlpHid * kMlpIn; e += blockDim.x) {
            const int o = e / kMlpIn, i = e % kMlpIn;
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc = fmaf(s.g3[b][o], s.x[b][i], acc);
            g[kMlpW1 + e] += acc;
        }
        for (int o = threadIdx.x; o < kMlpHid; o += blockDim.x) {
            float acc = 0.f;
            for (int b = 0; b < nb; ++b) acc += s.g3[b][o];
            g[kMlpB1 + o] += acc;
        }
        __syncthreads();
    }
    lsum[threadIdx.x] = lacc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float tot = 0.f;
        for (int i = 0; i < kMlpThreads; ++i) tot += lsum[i];
        loss[blockIdx.x] = tot;
    }
}

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
