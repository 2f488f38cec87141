// meq_cluster.cuh - batched sweeps with each system resident in one
// thread-block cluster (n <= 17).
//
// A system of n <= 17 sites needs 24 B per state for the classical-RK4
// Horner scheme in FP64 (state x, stage vectors a and b/c; 16 B in mixed
// precision), at most 3 MB - less than the shared memory of a cluster of 16
// SMs.  So a cluster keeps one system entirely on chip and runs it to its own
// exit rule with no HBM traffic at all: CTA r of a cluster of C = 2^cs_log2
// CTAs holds states [r*S, (r+1)*S), S = 2^(n - cs_log2), of every vector in
// its shared memory; a gather whose partner lives in another CTA (the high
// state bits are the CTA rank) reads that CTA's shared memory through the
// cluster's distributed shared memory (ld.shared::cluster).  Between stages
// the cluster synchronises through mbarriers with bounded waits (every CTA
// arrives on every CTA's barrier; each waits on its own).  Clusters are
// persistent: when a system converges (or reaches the step limit) the
// cluster writes it back and takes the next one from a global queue, so
// converged systems retire without costing the others anything.
//
// One RK4 step (constant rates, Horner form; the tile sweeps use the factored form):
//   H1 a = h M x          (gathers x)
//   H2 b = a + h/4 M a    (gathers a)
//   H3 c = a + h/3 M b    (gathers b; c kept in registers until every CTA
//                          has finished gathering b, then stored over b)
//   H4 D = a + h/2 M c, x' = x + D, L1 norm of D  (gathers c)
// Rows are summed in the reference's order (entry, diagonal, exit, hops by
// ascending bit, src/lib/solv.c:81-135); the diagonal comes from two tables
// (state bits 0..7 and 8..n-1) plus the term straddling them, a
// reassociation the RK4 stages allow.  The exit rule is the reference's
// (src/masterEquation.c:670-679) per system: every CTA reads all CTAs' partial
// norms in rank order, so all of them take the same decision.
#pragma once

#include <type_traits>

#include "meq_batch.cuh"

namespace tasep {

constexpr int kClThreads = 512;
constexpr int kClMaxN = 17;
constexpr int kClMaxRanks = 16;

struct ClusterParams {
    int n, nsys;
    int cs_log2;                 // log2 CTAs per cluster
    int sbits;                   // log2 states per CTA (n - cs_log2)
    double h;
    const double *rates;         // [nsys][n+1]
    double *X;                   // [nsys][2^n], initial and final states
    BatchExit *ex;               // [nsys]
    unsigned int *queue;         // next system to take (0 at launch)
    int *error;                  // set when a bounded wait expired
    double thresh;
    int stop_count;
    int exit_rule;
    unsigned long long max_steps;
    unsigned long long wait_ns;  // 0: kWaitLimitNs
    int sys_limit;               // systems taken from the queue (nsys for a run)
};

struct ClCtrl {
    uint64_t cbar[2];            // cluster barriers, used alternately (count = CTAs per cluster)
    int sys;                     // rank 0: the cluster's current system
    int err;
    int done;
    int pad;
    double partial;              // this CTA's L1 norm of the step
    double wsum[kClThreads / 32];
    double rates_d[kClMaxN + 1];
    float rates_f[kClMaxN + 1];
    uint32_t cl_bar[2][kClMaxRanks];  // cluster addresses of every rank's cbar[0], cbar[1]
    uint32_t cl_ctrl[kClMaxRanks];  // ... of every rank's control block
    uint32_t cl_buf[3][kClMaxRanks];  // ... of every rank's X, A, B buffers
};
constexpr int kClCtrlBytes = 1024;
static_assert(sizeof(ClCtrl) <= kClCtrlBytes, "cluster control block");

template <typename E> struct ClLayout {
    static constexpr int dlo = 256;                        // entries, bits 0..7
    static constexpr int dhi = 1 << (kClMaxN - 8);         // entries, bits 8..n-1
    static size_t bytes(int sbits) {
        const size_t S = size_t(1) << sbits;
        return kClCtrlBytes + (dlo + dhi) * sizeof(double) * 2 + S * (sizeof(double) + 2 * sizeof(E));
    }
};

__device__ __forceinline__ uint32_t cl_rank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_id() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
__device__ __forceinline__ uint32_t cl_count() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
// address of the same shared-memory location in CTA `rank` of the cluster
__device__ __forceinline__ uint32_t cl_map(const void *p, uint32_t rank) {
    uint32_t a;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(a) : "r"(smem_u32(p)), "r"(rank));
    return a;
}
__device__ __forceinline__ void cl_hw_sync() {  // hardware cluster barrier (start and end of the kernel only)
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ bool mbar_try_wait_cluster(uint64_t *bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

template <typename T> struct ClLoad;
template <> struct ClLoad<double> {
    static __device__ __forceinline__ void pair(uint32_t a, double &x, double &y) {
        asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(a) : "memory");
    }
    static __device__ __forceinline__ double one(uint32_t a) {
        double x;
        asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(x) : "r"(a) : "memory");
        return x;
    }
};
template <> struct ClLoad<float> {
    static __device__ __forceinline__ void pair(uint32_t a, float &x, float &y) {
        asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(a) : "memory");
    }
    static __device__ __forceinline__ float one(uint32_t a) {
        float x;
        asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(x) : "r"(a) : "memory");
        return x;
    }
};

// Bounded cluster barrier number k: every thread orders its shared-memory
// writes at cluster scope, thread r < C arrives on rank r's barrier
// cbar[k & 1], thread 0 waits (acquire) on its own.  The two barriers
// alternate, so an arrival for barrier k+1 from a CTA that is already past
// barrier k can never count towards barrier k of a slower CTA.  Returns false
// once a wait has expired in this CTA (the error is also raised globally).
__device__ __forceinline__ bool cl_barrier(ClCtrl &c, uint32_t &k, int ranks, uint64_t limit, int *gerr) {
    const int which = k & 1;
    const uint32_t parity = (k >> 1) & 1;
    asm volatile("fence.acq_rel.cluster;" ::: "memory");
    __syncthreads();
    if (int(threadIdx.x) < ranks && !c.err)
        asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(c.cl_bar[which][threadIdx.x])
                     : "memory");
    if (threadIdx.x == 0 && !c.err) {
        bool ok = mbar_try_wait_cluster(&c.cbar[which], parity);
        if (!ok) {
            const uint64_t t0 = global_timer_ns();
            while (!(ok = mbar_try_wait_cluster(&c.cbar[which], parity)))
                if (global_timer_ns() - t0 > limit) break;
        }
        if (!ok) {
            c.err = 1;
            atomicExch(gerr, 1);
        }
    }
    __syncthreads();
    ++k;
    return !c.err;
}

// Row sums of all pairs a thread owns, for a gathered vector with local part
// `loc` and per-rank cluster addresses `cbase`.  Thread t owns the NP pairs
// (i, i+1), i = rank*S + 2t + 1024q, q = 0..NP-1 (S = 1024 NP states per CTA).
// The loops run over the terms in the reference's row order (entry,
// diagonal, exit, hops by ascending bit) with the pairs innermost: the loads
// of one term for all NP pairs are independent and in flight together, and
// whether a hop's partner lives in another CTA depends only on its bit.
template <typename G, int NP>
__device__ __forceinline__ void cl_gather(const ClCtrl &c, const uint32_t *cbase, const G *loc, int n, int sbits,
                                          uint32_t rank, const G *dlo, const G *dhi, G (&t)[2 * NP]) {
    using A = Ar<G, false>;
    using V2T = typename std::conditional<sizeof(G) == 8, double2, float2>::type;
    const uint32_t smask = (1u << sbits) - 1;
    const uint32_t i0 = (rank << sbits) + 2 * threadIdx.x;
    auto rate = [&](int k) -> G { return sizeof(G) == 8 ? G(c.rates_d[k]) : G(c.rates_f[k]); };
    auto pair_at = [&](uint32_t j, G &u, G &v) {  // pair starting at even global index j
        const uint32_t rj = j >> sbits, lj = j & smask;
        if (rj == rank) {
            const V2T w = *reinterpret_cast<const V2T *>(loc + lj);
            u = w.x;
            v = w.y;
        } else {
            ClLoad<G>::pair(cbase[rj] + lj * uint32_t(sizeof(G)), u, v);
        }
    };
    G x[2 * NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) {
        const V2T w = *reinterpret_cast<const V2T *>(loc + ((i0 + 1024u * q) & smask));
        x[2 * q] = w.x;
        x[2 * q + 1] = w.y;
        t[2 * q] = G(0);
        t[2 * q + 1] = G(0);
    }
    {  // 1. entry from i - 2^(n-1)
        const G r0 = rate(0);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const uint32_t i = i0 + 1024u * q;
            if ((i >> (n - 1)) & 1) {
                G e0, e1;
                pair_at(i - (1u << (n - 1)), e0, e1);
                t[2 * q] = A::madd(t[2 * q], r0, e0);
                t[2 * q + 1] = A::madd(t[2 * q + 1], r0, e1);
            }
        }
    }
    {  // 2. diagonal (bits 0..7 and the pair (7, 8) are the thread's), 3. exit
        const G lo0 = dlo[i0 & 255], lo1 = dlo[(i0 + 1) & 255];
        const G r7 = (!((i0 >> 7) & 1) && ((i0 >> 8) & 1)) ? rate(n - 8) : G(0);
        const G rn = rate(n);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const uint32_t i = i0 + 1024u * q;
            const G hi = dhi[i >> 8];
            const G d0 = (lo0 + hi) - r7, d1 = (lo1 + hi) - r7;
            t[2 * q] = A::madd(t[2 * q], d0, x[2 * q]);
            t[2 * q + 1] = A::madd(t[2 * q + 1], d1, x[2 * q + 1]);
            t[2 * q] = A::madd(t[2 * q], rn, x[2 * q + 1]);
        }
    }
    if (!((i0 >> 1) & 1)) {  // 4. hop k = 0 into the odd state, from i+2 (same CTA, same q)
        const G r = rate(n - 1);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const G p = loc[((i0 + 1024u * q) & smask) + 2];
            t[2 * q + 1] = A::madd(t[2 * q + 1], r, p);
        }
    }
    for (int k = 1; k < n - 1; ++k) {  // hops k >= 1 into both states, from the pair at i + 2^k
        const G r = rate(n - 1 - k);
        const bool remote = k + 1 >= sbits;
#pragma unroll
        for (int q = 0; q < NP; ++q) {
            const uint32_t i = i0 + 1024u * q;
            if (((i >> k) & 3u) == 1u) {
                const uint32_t j = i + (1u << k);
                G p0, p1;
                if (remote) {
                    ClLoad<G>::pair(cbase[j >> sbits] + (j & smask) * uint32_t(sizeof(G)), p0, p1);
                } else {
                    const V2T w = *reinterpret_cast<const V2T *>(loc + (j & smask));
                    p0 = w.x;
                    p1 = w.y;
                }
                t[2 * q] = A::madd(t[2 * q], r, p0);
                t[2 * q + 1] = A::madd(t[2 * q + 1], r, p1);
            }
        }
    }
}

template <typename E, int NP>
__global__ void __launch_bounds__(kClThreads, 1) meq_cluster_kernel(const __grid_constant__ ClusterParams p) {
    extern __shared__ __align__(128) unsigned char cl_smem[];
    ClCtrl &c = *reinterpret_cast<ClCtrl *>(cl_smem);
    const int n = p.n, sbits = p.sbits;
    const int ranks = 1 << p.cs_log2;
    const uint32_t S = 1u << sbits;
    double *dlo_d = reinterpret_cast<double *>(cl_smem + kClCtrlBytes);
    double *dhi_d = dlo_d + ClLayout<E>::dlo;
    E *dlo_e = reinterpret_cast<E *>(dhi_d + ClLayout<E>::dhi);
    E *dhi_e = dlo_e + ClLayout<E>::dlo;
    double *X = reinterpret_cast<double *>(cl_smem + kClCtrlBytes + (ClLayout<E>::dlo + ClLayout<E>::dhi) * 2 *
                                                                         sizeof(double));
    E *Av = reinterpret_cast<E *>(X + S);
    E *Bv = Av + S;
    const uint32_t rank = cl_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const uint64_t limit = p.wait_ns ? p.wait_ns : kWaitLimitNs;

    if (tid == 0) {
        mbar_init(&c.cbar[0], ranks);
        mbar_init(&c.cbar[1], ranks);
        fence_mbar_init();
        c.err = 0;
        c.sys = -1;
    }
    if (tid < ranks) {
        c.cl_bar[0][tid] = cl_map(&c.cbar[0], tid);
        c.cl_bar[1][tid] = cl_map(&c.cbar[1], tid);
        c.cl_ctrl[tid] = cl_map(&c, tid);
        c.cl_buf[0][tid] = cl_map(X, tid);
        c.cl_buf[1][tid] = cl_map(Av, tid);
        c.cl_buf[2][tid] = cl_map(Bv, tid);
    }
    cl_hw_sync();  // every CTA's barrier is initialised before anyone arrives on it
    uint32_t bk = 0;  // cluster barriers passed
    const unsigned long long N = 1ull << n;
    const double h = p.h;

    while (!c.err) {
        // ---- take the next system (rank 0 draws it, the others read it) ----
        if (rank == 0 && tid == 0) {
            const unsigned s = atomicAdd(p.queue, 1u);
            c.sys = s < unsigned(p.sys_limit) ? int(s) : -1;
        }
        if (!cl_barrier(c, bk, ranks, limit, p.error)) break;
        int sys;
        {
            uint32_t a = c.cl_ctrl[0] + uint32_t(offsetof(ClCtrl, sys));
            asm volatile("ld.shared::cluster.s32 %0, [%1];" : "=r"(sys) : "r"(a) : "memory");
        }
        if (sys < 0) break;
        // ---- load the system: rates, diagonal tables, this CTA's part of x ----
        const double *rs = p.rates + size_t(sys) * (n + 1);
        if (tid <= n) {
            c.rates_d[tid] = rs[tid];
            c.rates_f[tid] = float(rs[tid]);
        }
        __syncthreads();
        for (int l = tid; l < 256; l += kClThreads) {  // bits 0..7: -r[n] b0, pairs j = 0..6
            double d = 0.0;
            if (l & 1) d -= c.rates_d[n];
            for (int j = 0; j < 7; ++j)
                if (!((l >> j) & 1) && ((l >> (j + 1)) & 1)) d -= c.rates_d[n - 1 - j];
            dlo_d[l] = d;
            E de = E(0);
            if (l & 1) de -= E(c.rates_d[n]);
            for (int j = 0; j < 7; ++j)
                if (!((l >> j) & 1) && ((l >> (j + 1)) & 1)) de -= E(c.rates_d[n - 1 - j]);
            dlo_e[l] = de;
        }
        for (int hh = tid; hh < (1 << (n - 8)); hh += kClThreads) {  // bits 8..n-1: -r[0] !b(n-1), pairs j >= 8
            double d = 0.0;
            E de = E(0);
            if (!((hh >> (n - 9)) & 1)) {
                d -= c.rates_d[0];
                de -= E(c.rates_d[0]);
            }
            for (int j = 8; j < n - 1; ++j)
                if (!((hh >> (j - 8)) & 1) && ((hh >> (j - 7)) & 1)) {
                    d -= c.rates_d[n - 1 - j];
                    de -= E(c.rates_d[n - 1 - j]);
                }
            dhi_d[hh] = d;
            dhi_e[hh] = de;
        }
        {
            const double *xs = p.X + size_t(sys) * N + size_t(rank) * S;
            for (uint32_t l = 2 * tid; l < S; l += 2 * kClThreads)
                *reinterpret_cast<double2 *>(X + l) = *reinterpret_cast<const double2 *>(xs + l);
        }
        if (!cl_barrier(c, bk, ranks, limit, p.error)) break;

        int early = 0, converged = 0;
        unsigned long long step = 0, at_stop = 0;
        double last = 0.0;
        bool failed = false;
        while (step < p.max_steps) {
            // H1: a = h M x
            {
                double t[2 * NP];
                cl_gather<double, NP>(c, c.cl_buf[0], X, n, sbits, rank, dlo_d, dhi_d, t);
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const uint32_t l = 2 * tid + 1024u * q;
                    Av[l] = E(h * t[2 * q]);
                    Av[l + 1] = E(h * t[2 * q + 1]);
                }
            }
            if (!cl_barrier(c, bk, ranks, limit, p.error)) { failed = true; break; }
            const E h4 = E(h / 4), h3 = E(h / 3);
            const double h2 = h / 2;
            {  // H2: b = a + h/4 M a
                E t[2 * NP];
                cl_gather<E, NP>(c, c.cl_buf[1], Av, n, sbits, rank, dlo_e, dhi_e, t);
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const uint32_t l = 2 * tid + 1024u * q;
                    Bv[l] = Av[l] + h4 * t[2 * q];
                    Bv[l + 1] = Av[l + 1] + h4 * t[2 * q + 1];
                }
            }
            if (!cl_barrier(c, bk, ranks, limit, p.error)) { failed = true; break; }
            {  // H3: c = a + h/3 M b, held in registers until b is no longer gathered
                E t[2 * NP];
                cl_gather<E, NP>(c, c.cl_buf[2], Bv, n, sbits, rank, dlo_e, dhi_e, t);
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const uint32_t l = 2 * tid + 1024u * q;
                    t[2 * q] = Av[l] + h3 * t[2 * q];
                    t[2 * q + 1] = Av[l + 1] + h3 * t[2 * q + 1];
                }
                if (!cl_barrier(c, bk, ranks, limit, p.error)) { failed = true; break; }
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const uint32_t l = 2 * tid + 1024u * q;
                    Bv[l] = t[2 * q];
                    Bv[l + 1] = t[2 * q + 1];
                }
            }
            if (!cl_barrier(c, bk, ranks, limit, p.error)) { failed = true; break; }
            // H4: D = a + h/2 M c, x += D, L1 norm
            double cs = 0.0;
            {
                E t[2 * NP];
                cl_gather<E, NP>(c, c.cl_buf[2], Bv, n, sbits, rank, dlo_e, dhi_e, t);
#pragma unroll
                for (int q = 0; q < NP; ++q) {
                    const uint32_t l = 2 * tid + 1024u * q;
                    const double D0 = double(Av[l]) + h2 * double(t[2 * q]);
                    const double D1 = double(Av[l + 1]) + h2 * double(t[2 * q + 1]);
                    X[l] += D0;
                    X[l + 1] += D1;
                    cs += fabs(D0) + fabs(D1);
                }
            }
            {
                const double ws = warp_sum(cs);
                if (lane == 0) c.wsum[warp] = ws;
                __syncthreads();
                if (tid == 0) {
                    double s = 0.0;
                    for (int w = 0; w < kClThreads / 32; ++w) s += c.wsum[w];
                    c.partial = s;
                }
            }
            if (!cl_barrier(c, bk, ranks, limit, p.error)) { failed = true; break; }
            // exit rule on the system's norm: the same sum, in rank order, in every CTA
            if (tid == 0) {
                double s = 0.0;
                for (int r = 0; r < ranks; ++r) {
                    double v;
                    asm volatile("ld.shared::cluster.f64 %0, [%1];"
                                 : "=d"(v)
                                 : "r"(c.cl_ctrl[r] + uint32_t(offsetof(ClCtrl, partial)))
                                 : "memory");
                    s += v;
                }
                last = s;
                int done = 0;
                if (p.exit_rule) {
                    if (s < p.thresh) {
                        early += 1;
                        at_stop = step;
                    } else {
                        early = 0;
                    }
                    if (early > p.stop_count) {
                        converged = 1;
                        done = 1;
                    }
                }
                c.done = done;
            }
            __syncthreads();
            ++step;
            if (c.done) break;
        }
        // ---- write back, record the result ----
        if (!failed) {
            double *xs = p.X + size_t(sys) * N + size_t(rank) * S;
            for (uint32_t l = 2 * tid; l < S; l += 2 * kClThreads)
                *reinterpret_cast<double2 *>(xs + l) = *reinterpret_cast<const double2 *>(X + l);
            if (rank == 0 && tid == 0) {
                BatchExit &e = p.ex[sys];
                e.steps_done = step;
                e.steps_at_stop = at_stop;
                e.early_stop = early;
                e.converged = converged;
                e.last_checksum = last;
                e.done = 1;
            }
        }
        // the partial norms and the queue slot are read remotely: keep them
        // until every CTA is past this system
        if (failed || !cl_barrier(c, bk, ranks, limit, p.error)) break;
    }
    cl_hw_sync();  // no CTA leaves while another may still read its shared memory
}

}  // namespace tasep
