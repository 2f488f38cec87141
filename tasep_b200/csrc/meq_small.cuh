// meq_small.cuh - whole-lattice kernel for n <= kSmallMaxN.
//
// The full state space (at most 2^11 states) and every stage vector live in
// one CTA's shared memory, and the whole integration loop - stages, L1 norm
// and the exit rule of src/masterEquation.c:670-679 - runs inside a single
// launch.  Rows are evaluated in the reference's entry order
// (src/lib/solv.c:81-135) with separate multiply and add.
#pragma once

#include "meq_common.cuh"

namespace tasep {

constexpr int kSmallMaxN = 11;
constexpr int kSmallThreads = 512;

enum SmallMode : int { SM_RUN = 0, SM_APPLY = 1 };
enum SmallIntegrator : int { SI_REF = 0, SI_HORNER = 1, SI_UFORM = 2 };

struct SmallParams {
    int n;
    int mode;        // SM_RUN or SM_APPLY
    int integrator;  // SI_*
    const double *x_in;
    double *x_out;
    double h, t0;
    unsigned long long max_steps;
    unsigned long long step0;  // index of the first step (exit bookkeeping)
    double thresh;
    int stop_count;
    int exit_rule;
    ExitState *ex;
    RateSpec rs;
};

// One generator row applied to x (shared memory), reference order.
template <typename T>
__device__ __forceinline__ T small_row(int n, uint32_t i, const T *__restrict__ r, const T *__restrict__ x) {
    using A = Ar<T, true>;
    T acc = T(0);
    const uint32_t hi = 1u << (n - 1);
    const bool top = (i & hi) != 0;
    if (top) acc = A::madd(acc, r[0], x[i - hi]);
    T d = T(0);
    if (i & 1u) d = A::sub(d, r[n]);
    if (!top) d = A::sub(d, r[0]);
    const uint32_t lm = hi - 1u;
    uint32_t m = ~i & (i >> 1) & lm;
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        d = A::sub(d, r[n - 1 - j]);
    }
    acc = A::madd(acc, d, x[i]);
    if (!(i & 1u)) acc = A::madd(acc, r[n], x[i + 1]);
    uint32_t hm = i & ~(i >> 1) & lm;
    while (hm) {
        const int k = __ffs(hm) - 1;
        hm &= hm - 1;
        acc = A::madd(acc, r[n - 1 - k], x[i + (1u << k)]);
    }
    return acc;
}

// Deterministic block sum over kSmallThreads threads.
__device__ __forceinline__ double small_block_sum(double v, double *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    v = warp_sum(v);
    if (lane == 0) red[warp] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int w = 0; w < kSmallThreads / 32; ++w) s += red[w];
    return s;
}

// E: type of the Horner stage vectors (double or float).
template <typename E>
__global__ void __launch_bounds__(kSmallThreads, 1) meq_small_kernel(const __grid_constant__ SmallParams p) {
    extern __shared__ __align__(16) unsigned char small_smem[];
    const int n = p.n;
    const uint32_t N = 1u << n;
    double *rd = reinterpret_cast<double *>(small_smem);     // 4 rate sets (double)
    float *rf = reinterpret_cast<float *>(rd + 4 * kMaxR);  // rate set 0 (float)
    double *red = reinterpret_cast<double *>(rf + 2 * kMaxR);
    int *flag = reinterpret_cast<int *>(red + kSmallThreads / 32);
    double *X = reinterpret_cast<double *>(small_smem + 2048);
    double *V1 = X + N;  // REF: next state; UFORM: U2; HORNER: A (as E)
    double *V2 = V1 + N;
    double *V3 = V2 + N;
    const int tid = threadIdx.x;
    // a run whose exit rule already fired in an earlier launch (the host
    // enqueues ahead of the exit state it has read) leaves the state as it is
    if (p.mode == SM_RUN && *reinterpret_cast<volatile int *>(&p.ex->done)) return;

    for (uint32_t i = tid; i < N; i += kSmallThreads) X[i] = p.x_in[i];
    if (tid == 0) *flag = 0;

    if (p.mode == SM_APPLY) {
        if (tid <= n) rd[tid] = rate_at(p.rs, tid, p.t0);
        __syncthreads();
        for (uint32_t i = tid; i < N; i += kSmallThreads) p.x_out[i] = small_row<double>(n, i, rd, X);
        return;
    }

    const double h = p.h;
    double t = p.t0;
    int early_stop = p.ex->early_stop;
    unsigned long long steps_at_stop = p.ex->steps_at_stop, done_steps = 0;
    double cs_last = 0.0;
    int converged = 0;
    E *A = reinterpret_cast<E *>(V1);
    E *B = A + N;
    E *C = B + N;
    const E hc4 = E(h / 4), hc3 = E(h / 3);
    const double hc2 = h / 2;

    for (unsigned long long s = 0; s < p.max_steps; ++s) {
        if (tid <= n) {
            if (p.integrator == SI_UFORM) {
                rd[0 * kMaxR + tid] = rate_at(p.rs, tid, t);
                rd[1 * kMaxR + tid] = rate_at(p.rs, tid, t + h / 2);
                rd[2 * kMaxR + tid] = rate_at(p.rs, tid, t + h / 2);
                rd[3 * kMaxR + tid] = rate_at(p.rs, tid, t + h);
            } else {
                const double r = rate_at(p.rs, tid, t);
                rd[tid] = r;
                rf[tid] = float(r);
            }
        }
        __syncthreads();
        double cs = 0.0;
        if (p.integrator == SI_REF) {
            for (uint32_t i = tid; i < N; i += kSmallThreads) {
                const double kv = __dmul_rn(h, small_row<double>(n, i, rd, X));
                const double k2 = __dmul_rn(2.0, kv);
                const double D = div6_rn(__dadd_rn(__dadd_rn(__dadd_rn(kv, k2), k2), kv));
                V1[i] = __dadd_rn(X[i], D);
                cs += fabs(D);
            }
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads) X[i] = V1[i];
        } else if (p.integrator == SI_HORNER) {
            const E *rE = sizeof(E) == 8 ? reinterpret_cast<const E *>(rd) : reinterpret_cast<const E *>(rf);
            for (uint32_t i = tid; i < N; i += kSmallThreads) A[i] = E(h * small_row<double>(n, i, rd, X));
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads) B[i] = A[i] + hc4 * small_row<E>(n, i, rE, A);
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads) C[i] = A[i] + hc3 * small_row<E>(n, i, rE, B);
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads) {
                const double D = double(A[i]) + hc2 * double(small_row<E>(n, i, rE, C));
                X[i] = X[i] + D;
                cs += fabs(D);
            }
        } else {  // SI_UFORM: classical RK4 with stage inputs, rates at stage times
            const double hh = 0.5 * h;
            for (uint32_t i = tid; i < N; i += kSmallThreads)
                V1[i] = __dadd_rn(__dmul_rn(hh, small_row<double>(n, i, rd, X)), X[i]);
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads)
                V2[i] = __dadd_rn(__dmul_rn(hh, small_row<double>(n, i, rd + kMaxR, V1)), X[i]);
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads)
                V3[i] = __dadd_rn(__dmul_rn(h, small_row<double>(n, i, rd + 2 * kMaxR, V2)), X[i]);
            __syncthreads();
            for (uint32_t i = tid; i < N; i += kSmallThreads) {
                const double x = X[i];
                const double k1 = 2.0 * (V1[i] - x), k2 = 2.0 * (V2[i] - x), k3 = V3[i] - x;
                const double k4 = __dmul_rn(h, small_row<double>(n, i, rd + 3 * kMaxR, V3));
                const double D = div6_rn(__dadd_rn(__dadd_rn(__dadd_rn(k1, 2.0 * k2), 2.0 * k3), k4));
                X[i] = __dadd_rn(x, D);
                cs += fabs(D);
            }
        }
        __syncthreads();
        const double tot = small_block_sum(cs, red);
        t += h;
        if (tid == 0) {
            cs_last = tot;
            done_steps = s + 1;
            if (p.exit_rule) {
                if (tot < p.thresh) {
                    ++early_stop;
                    steps_at_stop = p.step0 + s;
                } else {
                    early_stop = 0;
                }
                if (early_stop > p.stop_count) {
                    converged = 1;
                    *flag = 1;
                }
            }
        }
        __syncthreads();
        if (*flag) break;
    }
    for (uint32_t i = tid; i < N; i += kSmallThreads) p.x_out[i] = X[i];
    if (tid == 0) {
        ExitState *ex = p.ex;
        ex->early_stop = early_stop;
        ex->steps_at_stop = steps_at_stop;
        ex->steps_done = p.step0 + done_steps;
        ex->last_checksum = cs_last;
        ex->converged = converged;
        ex->done = converged;
    }
}

inline size_t small_smem_bytes(int n) { return 2048 + 4 * sizeof(double) * (size_t(1) << n); }

}  // namespace tasep
