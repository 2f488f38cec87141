// meq_obs.cuh - one pass over the state for all observables.
//
// Per chunk of 2^C states (C = min(n, kObsBits)) the CTA computes, from
// shared memory, the chunk sum S0, the in-chunk first/second moments
// S2[a][b] = sum_{i: b_a(i)=b_b(i)=1} x_i (a <= b < C) and the marginals of the
// 4-bit windows that lie inside the chunk or straddle its upper edge.  Terms
// that involve bits above the chunk follow from the chunk index.  Each
// accumulator is owned by one thread, chunks are visited in a fixed order and
// a second kernel adds the per-CTA rows in CTA order, so the result is
// deterministic.  These feed condense / exp_val_eval (src/lib/matvec.c:10-91),
// the covariance and product matrices (src/masterEquation.c:1121-1139,
// :1289-1302) and the window observables (src/masterEquation.c:32-143).
#pragma once

#include "meq_common.cuh"

namespace tasep {

constexpr int kObsBits = 11;
constexpr int kObsThreads = 256;

// Accumulator layout (doubles): [0] S0, then M[a][b] (a <= b < n) packed
// row-major over the upper triangle, then P4[p][16] for p = 0..n-4.
__host__ __device__ inline int obs_tri(int n, int a, int b) {  // a <= b
    return 1 + a * n - (a * (a - 1)) / 2 + (b - a);
}
__host__ __device__ inline int obs_p4(int n, int p, int q) { return 1 + n * (n + 1) / 2 + p * 16 + q; }
__host__ __device__ inline int obs_count(int n) { return 1 + n * (n + 1) / 2 + (n >= 4 ? (n - 3) * 16 : 0); }

struct ObsParams {
    int n;
    const double *x;
    double *partials;  // gridDim.x * obs_count(n)
};

// Insert a 1 bit at position a (bits >= a shift up).
__device__ __forceinline__ uint32_t ins1(uint32_t k, int a) {
    const uint32_t lo = k & ((1u << a) - 1u);
    return ((k >> a) << (a + 1)) | (1u << a) | lo;
}

__global__ void __launch_bounds__(kObsThreads) meq_obs_kernel(const ObsParams p) {
    extern __shared__ __align__(16) double osm[];
    const int n = p.n;
    const int C = n < kObsBits ? n : kObsBits;
    const uint32_t CH = 1u << C;
    const int NA = obs_count(n);
    double *xs = osm;        // chunk
    double *acc = xs + CH;   // NA accumulators of this CTA
    double *q = acc + NA;    // in-chunk quantities
    // quantity index map: [0] S0; [1..] S2[a][b] a<=b<C; P4 inside; straddle lows
    const int nS2 = C * (C + 1) / 2;
    const int nP4in = C >= 4 ? (C - 3) * 16 : 0;
    const int qS2 = 1, qP4 = qS2 + nS2, qL = qP4 + nP4in;
    const int nL = (n > C) ? 14 : 0;  // windows p = C-3..C-1 with w = C-p low bits (2+4+8)
    const int NQ = qL + nL;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned long long nchunks = 1ull << (n - C);

    for (int i = tid; i < NA; i += kObsThreads) acc[i] = 0.0;
    __syncthreads();

    for (unsigned long long H = blockIdx.x; H < nchunks; H += gridDim.x) {
        for (uint32_t i = tid; i < CH; i += kObsThreads) xs[i] = p.x[H * CH + i];
        __syncthreads();
        for (int qi = warp; qi < NQ; qi += kObsThreads / 32) {
            double s = 0.0;
            if (qi == 0) {
                for (uint32_t k = lane; k < CH; k += 32) s += xs[k];
            } else if (qi < qP4) {
                int t = qi - qS2, a = 0;
                while (t >= C - a) { t -= C - a; ++a; }
                const int b = a + t;
                if (a == b) {
                    for (uint32_t k = lane; k < (CH >> 1); k += 32) s += xs[ins1(k, a)];
                } else {
                    for (uint32_t k = lane; k < (CH >> 2); k += 32) s += xs[ins1(ins1(k, a), b)];
                }
            } else if (qi < qL) {
                const int t = qi - qP4, pw = t >> 4, pat = t & 15;
                for (uint32_t k = lane; k < (CH >> 4); k += 32) {
                    const uint32_t i = ((k >> pw) << (pw + 4)) | (uint32_t(pat) << pw) | (k & ((1u << pw) - 1u));
                    s += xs[i];
                }
            } else {
                // low part of a straddling window: w bits C-w..C-1 equal lq
                int t = qi - qL, w = 1;
                while (t >= (1 << w)) { t -= (1 << w); ++w; }
                const uint32_t lq = uint32_t(t);
                const int pw = C - w;
                for (uint32_t k = lane; k < (1u << pw); k += 32) s += xs[(lq << pw) | k];
            }
            s = warp_sum(s);
            if (lane == 0) q[qi] = s;
        }
        __syncthreads();
        // fold into the owned accumulators
        const double S0 = q[0];
        for (int e = tid; e < NA; e += kObsThreads) {
            double v = 0.0;
            if (e == 0) {
                v = S0;
            } else if (e < 1 + n * (n + 1) / 2) {
                int t = e - 1, a = 0;
                while (t >= n - a) { t -= n - a; ++a; }
                const int b = a + t;
                if (b < C) {
                    int ti = 0;
                    for (int aa = 0; aa < a; ++aa) ti += C - aa;
                    v = q[qS2 + ti + (b - a)];
                } else if (a < C) {
                    if ((H >> (b - C)) & 1) {
                        int ti = 0;
                        for (int aa = 0; aa < a; ++aa) ti += C - aa;
                        v = q[qS2 + ti];  // S1[a]
                    }
                } else {
                    if (((H >> (a - C)) & 1) && ((H >> (b - C)) & 1)) v = S0;
                }
            } else {
                const int t = e - (1 + n * (n + 1) / 2), pw = t >> 4, pat = t & 15;
                if (pw + 4 <= C) {
                    v = q[qP4 + t];
                } else if (pw < C) {
                    const int w = C - pw;  // low bits inside the chunk
                    const uint32_t hpat = uint32_t(H & ((1ull << (4 - w)) - 1ull));
                    if ((uint32_t(pat) >> w) == hpat) {
                        int off = 0;
                        for (int ww = 1; ww < w; ++ww) off += 1 << ww;
                        v = q[qL + off + (pat & ((1 << w) - 1))];
                    }
                } else {
                    if (uint32_t((H >> (pw - C)) & 15ull) == uint32_t(pat)) v = S0;
                }
            }
            acc[e] += v;
        }
        __syncthreads();
    }
    for (int e = tid; e < NA; e += kObsThreads) p.partials[size_t(blockIdx.x) * NA + e] = acc[e];
}

// Adds the per-CTA rows in CTA order.
__global__ void meq_obs_reduce(const double *partials, int rows, int na, double *out) {
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < na; e += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int r = 0; r < rows; ++r) s += partials[size_t(r) * na + e];
        out[e] = s;
    }
}

inline size_t obs_smem_bytes(int n) {
    const int C = n < kObsBits ? n : kObsBits;
    const int nq = 1 + C * (C + 1) / 2 + (C >= 4 ? (C - 3) * 16 : 0) + 14;
    return sizeof(double) * ((size_t(1) << C) + obs_count(n) + nq);
}

}  // namespace tasep
