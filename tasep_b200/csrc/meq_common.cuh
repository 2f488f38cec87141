// meq_common.cuh - shared types and sm_100a PTX helpers for the TASEP
// master-equation kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include <utility>

namespace tasep {

constexpr int kMaxN = 33;
constexpr int kMaxR = kMaxN + 1;

// Kernel flavours.  REF is the reference step; H1..H4 the four sweeps of
// classical RK4 for constant rates (the factored form of Rk4Factors in the
// tile and batched sweeps, a Horner scheme in the small and cluster-resident
// kernels); U1..U4 the four
// stages of classical RK4 with materialised stage inputs (time-variant
// rates); APPLY is y = M x.
enum Stage : int {
    ST_REF = 0, ST_H1, ST_H2, ST_H3, ST_H4, ST_U1, ST_U2, ST_U3, ST_U4, ST_APPLY, ST_COUNT
};

// Exit-rule state kept on the device so that steps can be enqueued ahead of
// the host (src/masterEquation.c:670-679).
struct ExitState {
    int done;
    int converged;
    int early_stop;
    int error;  // 0 ok, 1 = a bounded wait expired
    unsigned long long steps_at_stop;
    unsigned long long steps_done;
    double last_checksum;
    double pad;
};

// Classical RK4 for constant rates.  With z = hM the step is the degree-4
// Taylor polynomial x' = x + z x + z^2 x/2 + z^3 x/6 + z^4 x/24, i.e.
// x' = x + z Q(z) x with 24 Q(z) = z^3 + 4 z^2 + 12 z + 24 = (z - r)(z^2 + p z + q),
// r the real root, p = 4 + r, q = -24/r.  The sweeps evaluate it as
//   v1 = z x,  v2 = (z - r) v1,  w = (z + p) v2,  x' = x + (z w + q v2) / 24,
// four generator applications of which only the last reads an operand besides
// its gathered vector and the state: 80 B per state per step in FP64 (a
// Horner scheme needs 88: its third sweep also reads z x).  The intermediate
// vectors stay within a small factor of v1 (|r| < 3, p, q > 0): no cancellation.
struct Rk4Factors {
    double r, p, q;
};
inline Rk4Factors rk4_factors() {
    double r = -2.9;  // Newton's method on z^3 + 4 z^2 + 12 z + 24 (one real root near -2.9)
    for (int i = 0; i < 60; ++i) {
        const double f = ((r + 4.0) * r + 12.0) * r + 24.0;
        const double d = (3.0 * r + 8.0) * r + 12.0;
        const double nr = r - f / d;
        if (nr == r) break;
        r = nr;
    }
    return {r, 4.0 + r, -24.0 / r};
}

// Rates for one launch: constant, or the time-variant functions of
// src/lib/matvec.c:44-68 evaluated at the stage time.
struct RateSpec {
    double r[kMaxR];
    double amp[kMaxR], per[kMaxR], off[kMaxR], cst[kMaxR];
    int type[kMaxR];
    int timevar;
};

// One rate at time t, with the reference's separate roundings
// (amplitude*sin(t*period + offset) + constant, clamped at 0).
__device__ __forceinline__ double rate_at(const RateSpec &rs, int i, double t) {
    if (!rs.timevar) return rs.r[i];
    double v;
    switch (rs.type[i]) {
    case 0: v = __dadd_rn(__dmul_rn(rs.amp[i], sin(__dadd_rn(__dmul_rn(t, rs.per[i]), rs.off[i]))), rs.cst[i]); break;
    case 1: v = __dadd_rn(__dmul_rn(rs.amp[i], cos(__dadd_rn(__dmul_rn(t, rs.per[i]), rs.off[i]))), rs.cst[i]); break;
    case 2: v = __dadd_rn(__dmul_rn(rs.amp[i], t), rs.cst[i]); break;
    default: return rs.r[i];
    }
    return v < 0.0 ? 0.0 : v;
}

// Arithmetic with or without contraction.  EXACT keeps every multiply and add
// separately rounded, as the reference's C (ISO mode, no contraction).
template <typename T, bool EXACT> struct Ar;
template <> struct Ar<double, true> {
    static __device__ __forceinline__ double madd(double acc, double a, double b) { return __dadd_rn(acc, __dmul_rn(a, b)); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
};
template <> struct Ar<double, false> {
    static __device__ __forceinline__ double madd(double acc, double a, double b) { return fma(a, b, acc); }
    static __device__ __forceinline__ double sub(double a, double b) { return a - b; }
};
template <> struct Ar<float, true> {
    static __device__ __forceinline__ float madd(float acc, float a, float b) { return __fadd_rn(acc, __fmul_rn(a, b)); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <> struct Ar<float, false> {
    static __device__ __forceinline__ float madd(float acc, float a, float b) { return fmaf(a, b, acc); }
    static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
};

// ---- PTX helpers (mbarrier, bulk async copies, cache policies) ----------

__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// RN(s / 6), the last operation of the reference's (k1 + 2 k2 + 2 k3 + k4) / 6
// (src/lib/solv.c:44-52), without a division instruction sequence.  Markstein's
// correction step (P. Markstein, IBM J. Res. Dev. 34(1), 1990): with
// z = RN(1/6), q = RN(s z) is within one ulp of v = s/6 (z is within 2^-56 of
// 1/6), the remainder r = s - 6q is exactly representable, so fma gives it
// exactly, and q' = RN(q + r z) differs from RN(q + r/6) = RN(v) only if
// q + r z and v straddle a rounding midpoint.  They cannot: |q + r z - v| =
// |r| |z - 1/6| < 12 ulp(v) 2^-56, while for a 53-bit s = S 2^E the distance
// from S 2^E / 6 to any midpoint of its binade is |8S - 3(2k+1)| 2^E / 48 or
// |4S - 3(2k+1)| 2^E / 24, an odd multiple of at least 2^E / 48 >= ulp(v) / 12.
// The argument needs s, q and r normal: 2^-900 <= |s| <= 2^1000.  +0 (most
// states early in a run from a pure state) also comes out exact; the rest
// (-0, subnormals, infinities, NaN) take the IEEE division.
__device__ __forceinline__ double div6_fast(double s) {
    constexpr double z = 1.0 / 6.0;  // RN(1/6), folded by the compiler
    const double q = __dmul_rn(s, z);
    const double r = __fma_rn(-q, 6.0, s);
    return __fma_rn(r, z, q);
}
// s for which div6_fast is the IEEE quotient: the normal range above and +0
// (q = r = +0); -0 would come out as +0.
__device__ __forceinline__ bool div6_fast_ok(double s) {
    const double a = fabs(s);
    return (a >= 0x1p-900 && a <= 0x1p+1000) || __double_as_longlong(s) == 0;
}
__device__ __forceinline__ double div6_rn(double s) {
    if (div6_fast_ok(s)) return div6_fast(s);
    return __ddiv_rn(s, 6.0);
}
// Four quotients per thread with one warp vote: the branch-free fast path
// unless some value in the warp needs the division.
__device__ __forceinline__ void div6_rn4(const double (&s)[4], double (&d)[4]) {
    const bool ok = div6_fast_ok(s[0]) && div6_fast_ok(s[1]) && div6_fast_ok(s[2]) && div6_fast_ok(s[3]);
    if (__all_sync(__activemask(), ok)) {
#pragma unroll
        for (int j = 0; j < 4; ++j) d[j] = div6_fast(s[j]);
    } else {
#pragma unroll
        for (int j = 0; j < 4; ++j) d[j] = div6_rn(s[j]);
    }
}

// Programmatic dependent launch (sweeps launched with the programmatic
// stream-serialization attribute): grid_dep_launch lets the next sweep's CTAs
// be scheduled, onto SMs this grid has left, while this grid finishes;
// grid_dep_wait blocks until the previous grid has completed and its memory
// is visible.  Nothing before the wait may touch device memory that the
// previous grid writes or reads.  Both are no-ops for a normal launch.
__device__ __forceinline__ void grid_dep_launch() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void grid_dep_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// Host side: launch with programmatic stream serialization, so that the
// kernel's CTAs may start (and run up to grid_dep_wait) while the previous
// kernel on the stream finishes.  Also valid inside stream capture.
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st,
                              Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Bounded wait: gives up after limit_ns (~2 s by default; or as soon as
// another thread has flagged an error), records the error and returns false.
constexpr uint64_t kWaitLimitNs = 2000000000ull;

__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, volatile int *err_flag,
                                          uint64_t limit_ns = kWaitLimitNs) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t it = 0;; ++it) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (*err_flag) return false;
            if (global_timer_ns() - t0 > limit_ns) {
                *err_flag = 1;
                return false;
            }
        }
    }
}

// Hands a shared-memory buffer back to the bulk-copy producer.  The reads of
// the buffer were generic-proxy loads and the producer's next bulk copy into
// it is an async-proxy write: every reading thread fences the two proxies
// before the warp arrives, otherwise the copy can overwrite data a lane has
// not finished reading (seen as stale partner tiles under load).
__device__ __forceinline__ void consumer_release(uint64_t *bar, int lane) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncwarp();
    if (lane == 0) mbar_arrive(bar);
}

// Bounded wait that ignores the error flag: used on the error path to let
// copies already issued land before the CTA exits.
__device__ __forceinline__ void mbar_drain(uint64_t *bar, uint32_t parity, uint64_t limit_ns) {
    const uint64_t t0 = global_timer_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_timer_ns() - t0 > limit_ns) return;
}

__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_normal() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_normal.b64 %0, 1.0;" : "=l"(p));
    return p;
}
__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Lowers the L2 eviction priority of one 128-byte line (if it is cached) to
// evict_normal; a hint, no effect on the data.
__device__ __forceinline__ void l2_demote_line(const void *p) {
    asm volatile("applypriority.global.L2::evict_normal [%0], 128;" ::"l"(p) : "memory");
}

// Bulk global -> shared copy completing on an mbarrier (no multicast).
// dst, src 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *bar,
                                         uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar)), "l"(policy)
        : "memory");
}

// 4-element vector load from shared memory.
template <typename T> struct V4;
template <> struct V4<double> {
    static __device__ __forceinline__ void lds(const double *p, double &a, double &b, double &c, double &d) {
        const double2 u = reinterpret_cast<const double2 *>(p)[0];
        const double2 v = reinterpret_cast<const double2 *>(p)[1];
        a = u.x; b = u.y; c = v.x; d = v.y;
    }
    static __device__ __forceinline__ void lds2(const double *p, double &a, double &b) {
        const double2 u = reinterpret_cast<const double2 *>(p)[0];
        a = u.x; b = u.y;
    }
    // read-once coherent global load (no L1 allocation, evict-first in L2).  Not
    // the .nc path: the stage that reads the state also rewrites it in place.
    static __device__ __forceinline__ void ldg(const double *p, double &a, double &b, double &c, double &d,
                                               uint64_t pol) {
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                     : "=d"(a), "=d"(b)
                     : "l"(p), "l"(pol));
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                     : "=d"(c), "=d"(d)
                     : "l"(p + 2), "l"(pol));
    }
    static __device__ __forceinline__ void stg(double *p, double a, double b, double c, double d, uint64_t pol) {
        asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(a), "d"(b),
                     "l"(pol)
                     : "memory");
        asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p + 2), "d"(c),
                     "d"(d), "l"(pol)
                     : "memory");
    }
};
template <> struct V4<float> {
    static __device__ __forceinline__ void lds(const float *p, float &a, float &b, float &c, float &d) {
        const float4 u = reinterpret_cast<const float4 *>(p)[0];
        a = u.x; b = u.y; c = u.z; d = u.w;
    }
    static __device__ __forceinline__ void lds2(const float *p, float &a, float &b) {
        const float2 u = reinterpret_cast<const float2 *>(p)[0];
        a = u.x; b = u.y;
    }
    static __device__ __forceinline__ void ldg(const float *p, float &a, float &b, float &c, float &d, uint64_t pol) {
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v4.f32 {%0, %1, %2, %3}, [%4], %5;"
                     : "=f"(a), "=f"(b), "=f"(c), "=f"(d)
                     : "l"(p), "l"(pol));
    }
    static __device__ __forceinline__ void stg(float *p, float a, float b, float c, float d, uint64_t pol) {
        asm volatile("st.global.L1::no_allocate.L2::cache_hint.v4.f32 [%0], {%1, %2, %3, %4}, %5;" ::"l"(p), "f"(a),
                     "f"(b), "f"(c), "f"(d), "l"(pol)
                     : "memory");
    }
};

// 2-element vector accesses (one 16-byte / 8-byte access per lane, so a
// warp covers a contiguous span: bank-conflict free in shared memory and
// fully coalesced in global memory).
template <typename T> struct V2;
template <> struct V2<double> {
    static __device__ __forceinline__ void lds(const double *p, double &a, double &b) {
        const double2 u = *reinterpret_cast<const double2 *>(p);
        a = u.x; b = u.y;
    }
    static __device__ __forceinline__ void ldg(const double *p, double &a, double &b, uint64_t pol) {
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f64 {%0, %1}, [%2], %3;"
                     : "=d"(a), "=d"(b)
                     : "l"(p), "l"(pol));
    }
    static __device__ __forceinline__ void stg(double *p, double a, double b, uint64_t pol) {
        asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;" ::"l"(p), "d"(a), "d"(b),
                     "l"(pol)
                     : "memory");
    }
};
template <> struct V2<float> {
    static __device__ __forceinline__ void lds(const float *p, float &a, float &b) {
        const float2 u = *reinterpret_cast<const float2 *>(p);
        a = u.x; b = u.y;
    }
    static __device__ __forceinline__ void ldg(const float *p, float &a, float &b, uint64_t pol) {
        asm volatile("ld.global.L1::no_allocate.L2::cache_hint.v2.f32 {%0, %1}, [%2], %3;"
                     : "=f"(a), "=f"(b)
                     : "l"(p), "l"(pol));
    }
    static __device__ __forceinline__ void stg(float *p, float a, float b, uint64_t pol) {
        asm volatile("st.global.L1::no_allocate.L2::cache_hint.v2.f32 [%0], {%1, %2}, %3;" ::"l"(p), "f"(a), "f"(b),
                     "l"(pol)
                     : "memory");
    }
};

// Deterministic warp sum (fixed xor tree).
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

}  // namespace tasep
