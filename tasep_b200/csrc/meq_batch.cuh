// meq_batch.cuh - many independent systems of the same length in one sweep.
//
// The batch is one array of nsys * 2^n states; system s owns states
// [s*2^n, (s+1)*2^n).  A launch applies one classical-RK4 sweep (factored
// form, Rk4Factors) to every system that has not converged yet: tiles of
// 2^kTileBits states, a producer warp streaming each tile and its partner
// tiles (partners never leave their system) into shared memory with
// cp.async.bulk, 16 consumer warps in the pair layout of meq_tile.cuh.  What
// differs from the single-system kernel:
//   * rates are per system: each consumer warp copies its system's rates into
//     a shared-memory row when its next tile belongs to another system, and
//     each thread forms the diagonal of its four states from its fixed
//     low-bit pairs and those rates;
//   * the L1 norm and the exit rule are per system: each warp stores its
//     partial sum in a fixed slot, a per-system ticket finds the last warp,
//     which adds the system's slots in order and updates that system's exit
//     state (src/masterEquation.c:670-679);
//   * a converged system (or one that reached the step limit) is skipped by
//     every later launch - it retires from the sweep - and its step count is
//     kept on the device, so a chunk of steps can be captured once in a CUDA
//     graph and replayed until every system has converged.
#pragma once

#include "meq_tile.cuh"

namespace tasep {

struct BatchExit {
    int done;
    int converged;
    int early_stop;
    int pad;
    unsigned long long steps_done;
    unsigned long long steps_at_stop;
    double last_checksum;
};

struct BatchParams {
    int n;                    // lattice length of every system (> kTileBits)
    int tps_bits;             // log2 tiles per system
    int nsys;
    const void *g;            // gathered vector (batched)
    const void *s0, *s1;      // per-state extras (batched)
    void *out;
    double h, hc;
    double cx;  // RK4 sweeps 2, 3: coefficient of the own gathered value; 4: of v2
    const double *rates;      // [nsys][n+1]
    double *partials;         // [nsys][tiles per system][kConsumerWarps]
    unsigned int *counters;   // [nsys]
    BatchExit *ex;            // [nsys]
    int *active;              // systems still running
    const int *list;          // ids of the systems that were running when the step started
    const int *count;         // number of entries in list
    int *error;               // set when a bounded wait expired
    int sys_major;            // 0: tiles interleaved over the CTAs; 1: whole systems per CTA
    double thresh;
    int stop_count;
    int exit_rule;
    unsigned long long max_steps;
};

// Rebuilds the list of running systems (ascending ids) after a step, so the
// next step's launches visit only their tiles.  One CTA; ballot-based scan.
__global__ void batch_compact_kernel(const BatchExit *ex, int nsys, int *list, int *count) {
    __shared__ int wtot[32];
    __shared__ int base;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nw = blockDim.x >> 5;
    grid_dep_launch();
    grid_dep_wait();  // the exit flags of the step's last sweep
    if (tid == 0) base = 0;
    __syncthreads();
    for (int s0 = 0; s0 < nsys; s0 += blockDim.x) {
        const int s = s0 + tid;
        const bool a = s < nsys && !*reinterpret_cast<const volatile int *>(&ex[s].done);
        const unsigned m = __ballot_sync(0xffffffffu, a);
        const int before = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) wtot[warp] = __popc(m);
        __syncthreads();
        int off = base;
        for (int w = 0; w < warp; ++w) off += wtot[w];
        if (a) list[off + before] = s;
        __syncthreads();
        if (tid == 0)
            for (int w = 0; w < nw; ++w) base += wtot[w];
        __syncthreads();
    }
    if (tid == 0) *count = base;
}

// k-th tile of this CTA's sequence, as a global tile index (ntiles when past
// the end).  Only systems on the running list are visited.
// Tile indices are 32-bit (the host keeps nsys * tiles per system below 2^31).
__device__ __forceinline__ uint32_t batch_tile(const BatchParams &p, uint32_t k, int ntb, uint32_t ntiles, int na) {
    const uint32_t mask = (1u << ntb) - 1;
    uint32_t e, t;
    if (!p.sys_major) {
        const uint32_t l = blockIdx.x + k * gridDim.x;
        e = l >> ntb;
        t = l & mask;
    } else {
        e = blockIdx.x + (k >> ntb) * gridDim.x;
        t = k & mask;
    }
    if (e >= uint32_t(na)) return ntiles;
    return (uint32_t(p.list[e]) << ntb) | t;
}

constexpr int kWarpRates = 32;  // per-warp row of one system's rates (n + 1 <= 25)

template <typename G> __device__ __forceinline__ G batch_rate(const double *r, int i) {
    return static_cast<G>(__ldg(r + i));
}

template <int S, typename E>
__global__ void __launch_bounds__(kTileThreads, 1) meq_batch_kernel(const __grid_constant__ BatchParams p) {
    using Tr = StageT<S, E>;
    using G = typename Tr::G;
    using O = typename Tr::O;
    using X0 = typename Tr::X0;
    using X1 = typename Tr::X1;
    static_assert(!Tr::EXACT && Tr::NX <= 2, "batched sweeps run the constant-rate RK4 sweeps");
    using LYB = TileLayout<S, E>;
    constexpr int gb = LYB::gb;
    // no diagonal table in shared memory here; each consumer warp keeps the
    // rates of the system it works on in a row of its own (kWarpRates)
    constexpr int RS0 = (kSmemMax - kCtrlBytes - 2 * gb - kConsumerWarps * kWarpRates * int(sizeof(G))) / gb;
    constexpr int RS = RS0 < kMaxRing ? RS0 : kMaxRing;

    extern __shared__ __align__(128) unsigned char batch_smem[];
    TileCtrl &c = *reinterpret_cast<TileCtrl *>(batch_smem);
    unsigned char *stage_base = batch_smem + kCtrlBytes;
    unsigned char *ring_base = stage_base + 2 * gb;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = p.n;
    const int ntb = p.tps_bits;  // tile bits inside a system (>= 1)
    const uint32_t tps = 1u << ntb;
    const uint32_t ntiles = uint32_t(p.nsys) << ntb;
    const int R = n + 1;
    grid_dep_launch();
    if (tid == 0) {
        c.err = 0;
        for (int b = 0; b < 2; ++b) {
            mbar_init(&c.full[b], 1);
            mbar_init(&c.empty[b], kConsumerWarps);
        }
        for (int s = 0; s < RS; ++s) {
            mbar_init(&c.rfull[s], 1);
            mbar_init(&c.rempty[s], kConsumerWarps);
        }
        fence_mbar_init();
    }
    // up to here only parameters and shared memory: the previous launch may
    // still be running
    grid_dep_wait();
    const int na = *p.count;  // running systems this step (set before the launch)
    __syncthreads();
    volatile int *errf = &c.err;
    const uint32_t lowmask = ntb >= 2 ? ((1u << (ntb - 1)) - 1) : 0u;
    const G *__restrict__ g = static_cast<const G *>(p.g);

    if (warp == kConsumerWarps) {
        // ---------------- producer ----------------
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();
            const uint64_t normal = policy_evict_normal();
            uint32_t it = 0;
            int pslot = 0;
            uint32_t plap = 0;
            bool ok = true;
            for (uint32_t k = 0; ok; ++k) {
                const uint32_t T = batch_tile(p, k, ntb, ntiles, na);
                if (T >= ntiles) break;
                const uint32_t t = T & (tps - 1), base = T - t;
                const int b = it & 1;
                if (it >= 2 && !mbar_wait(&c.empty[b], ((it >> 1) - 1) & 1, errf)) break;
                unsigned char *st = stage_base + b * gb;
                mbar_arrive_expect_tx(&c.full[b], gb);
                bulk_g2s(st, g + (unsigned long long)T * kTile, gb, &c.full[b], normal);
                const bool top = (t >> (ntb - 1)) & 1;
                const bool strad = !(t & 1);
                const uint32_t hmask = t & ~(t >> 1) & lowmask;
                const int np = int(top) + int(strad) + __popc(hmask);
                uint32_t hm = hmask;
                for (int q = 0; q < np; ++q) {
                    unsigned long long src;
                    uint32_t bytes = gb;
                    if (q == 0 && top) {
                        src = t - (1ull << (ntb - 1));
                    } else if (q == int(top) && strad) {
                        src = t + 1;
                        bytes = gb / 2;
                    } else {
                        const int u = __ffs(hm) - 1;
                        hm &= hm - 1;
                        src = t + (1ull << u);
                    }
                    if (plap > 0 && !mbar_wait(&c.rempty[pslot], (plap - 1) & 1, errf)) {
                        ok = false;
                        break;
                    }
                    mbar_arrive_expect_tx(&c.rfull[pslot], bytes);
                    bulk_g2s(ring_base + pslot * gb, g + (base + src) * kTile, bytes, &c.rfull[pslot], keep);
                    if (++pslot == RS) {
                        pslot = 0;
                        ++plap;
                    }
                }
                ++it;
            }
            if (!ok || *errf) {
                atomicExch(p.error, 1);
                for (int b = 0; b < 2; ++b) {
                    const uint32_t uses = (it + 1 - b) / 2;
                    if (uses) mbar_drain(&c.full[b], (uses - 1) & 1, 100000000ull);
                }
                for (int s = 0; s < RS; ++s) {
                    const uint32_t uses = plap + (s < pslot ? 1u : 0u);
                    if (uses) mbar_drain(&c.rfull[s], (uses - 1) & 1, 100000000ull);
                }
            }
        }
        return;
    }

    // ---------------- consumers (pair layout of meq_tile.cuh) ----------------
    const uint64_t once = policy_evict_first();
    O *__restrict__ out = static_cast<O *>(p.out);
    const uint32_t t9 = tid;
    const int pb0 = 2 * tid, pb1 = 2 * tid + kTile / 2;
    const bool b9 = (t9 >> 8) & 1;
    const bool b1clear = !(t9 & 1);
    int qcnt = 0, qoff[4], qidx[4];  // this thread's in-tile hops k = q+1, ascending
    {
        uint32_t hq = t9 & ~(t9 >> 1) & 0xFFu;
        qcnt = __popc(hq);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int q = hq ? __ffs(hq) - 1 : 0;
            hq &= hq - 1;
            qoff[k] = 2 << q;
            qidx[k] = n - 2 - q;
        }
    }
    // This thread's part of the diagonal below the tile level, in terms of the
    // system's rates: the pairs j = 1..8 (state bits j, j+1 = t bits j-1, j)
    // with b_j = 0, b_(j+1) = 1 are the same for its four states; j = 0 adds
    // r[n-1] to the first state of each pair if t bit 0 is set; j = 9 adds
    // r[n-10] to the P1 states (bit 10 set) if t bit 8 is clear; the exit term
    // r[n] goes to the second state of each pair (b0 set).
    int dcnt = 0, didx[4];
    {
        uint32_t dq = ~t9 & (t9 >> 1) & 0xFFu;
        dcnt = __popc(dq);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int q = dq ? __ffs(dq) - 1 : 0;
            dq &= dq - 1;
            didx[k] = n - 2 - q;
        }
    }
    const bool t0set = t9 & 1;
    uint32_t it = 0;
    int cslot = 0;
    uint32_t cph = 0;
    bool ok = true;
    G *wr = reinterpret_cast<G *>(ring_base + RS * gb) + warp * kWarpRates;  // this warp's rates row
    uint32_t cur_sys = 0xffffffffu;

    for (uint32_t k = 0;; ++k) {
        const uint32_t T = batch_tile(p, k, ntb, ntiles, na);
        if (T >= ntiles) break;
        const uint32_t sys = T >> ntb, t = T & (tps - 1);
        const int b = it & 1;
        const bool top = (t >> (ntb - 1)) & 1;
        const bool strad = !(t & 1);
        const uint32_t hmask = t & ~(t >> 1) & lowmask;
        const uint32_t dhmask = ~t & (t >> 1) & lowmask;
        const unsigned long long gT = (unsigned long long)T * kTile;
        if (sys != cur_sys) {  // warp-uniform: one coalesced load of the system's rates
            __syncwarp();
            if (lane < R) wr[lane] = batch_rate<G>(p.rates + size_t(sys) * R, lane);
            __syncwarp();
            cur_sys = sys;
        }
        const G rn = wr[n], r0 = wr[0], rn1 = wr[n - 1];
        const G r9 = wr[n - 10], rnL = wr[n - kTileBits];

        X0 xa[4];
        X1 xb[4];
        if constexpr (Tr::NX > 0) {
            const X0 *s = static_cast<const X0 *>(p.s0) + gT;
            V2<X0>::ldg(s + pb0, xa[0], xa[1], once);
            V2<X0>::ldg(s + pb1, xa[2], xa[3], once);
        }
        if constexpr (Tr::NX > 1) {
            const X1 *s = static_cast<const X1 *>(p.s1) + gT;
            V2<X1>::ldg(s + pb0, xb[0], xb[1], once);
            V2<X1>::ldg(s + pb1, xb[2], xb[3], once);
        }
        // diagonal below the tile level (reassociated: these stages may)
        G d0, d1, d2, d3;
        {
            G sd = top ? G(0) : r0;
#pragma unroll
            for (int k = 0; k < 4; ++k)
                if (k < dcnt) sd += wr[didx[k]];
            const G e0 = t0set ? -(sd + rn1) : -sd;  // first state of a pair (b0 clear)
            const G e1 = -(sd + rn);                 // second state (b0 set)
            d0 = e0; d1 = e1;
            d2 = b9 ? e0 : e0 - r9;
            d3 = b9 ? e1 : e1 - r9;
        }
        G a0 = G(0), a1 = G(0), a2 = G(0), a3 = G(0);
        int eslot = 0;
        if (top) {
            eslot = cslot;
            if (!mbar_wait(&c.rfull[cslot], cph, errf)) { ok = false; break; }
            const G *ent = reinterpret_cast<const G *>(ring_base + cslot * gb);
            G e0, e1, e2, e3;
            V2<G>::lds(ent + pb0, e0, e1);
            V2<G>::lds(ent + pb1, e2, e3);
            a0 = fma(r0, e0, a0); a1 = fma(r0, e1, a1); a2 = fma(r0, e2, a2); a3 = fma(r0, e3, a3);
            if (++cslot == RS) { cslot = 0; cph ^= 1; }
        }
        if (!mbar_wait(&c.full[b], (it >> 1) & 1, errf)) { ok = false; break; }
        const G *xs = reinterpret_cast<const G *>(stage_base + b * gb);
        G x0, x1, x2, x3;
        V2<G>::lds(xs + pb0, x0, x1);
        V2<G>::lds(xs + pb1, x2, x3);
        if (!strad) { d0 -= rnL; d1 -= rnL; }
        {
            G ds = G(0);
            for (uint32_t mh = dhmask; mh; mh &= mh - 1)
                ds += wr[n - 1 - kTileBits - (__ffs(mh) - 1)];
            d0 -= ds; d1 -= ds; d2 -= ds; d3 -= ds;
        }
        a0 = fma(d0, x0, a0); a1 = fma(d1, x1, a1); a2 = fma(d2, x2, a2); a3 = fma(d3, x3, a3);
        a0 = fma(rn, x1, a0);
        a2 = fma(rn, x3, a2);
        {
            const G n0 = __shfl_down_sync(0xffffffffu, x0, 1);
            const G n2 = __shfl_down_sync(0xffffffffu, x2, 1);
            if (b1clear) {
                a1 = fma(rn1, n0, a1);
                a3 = fma(rn1, n2, a3);
            }
        }
        G c0 = G(0), c1 = G(0), c2 = G(0), c3 = G(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < qcnt) {
                const G rq = wr[qidx[k]];
                G p0, p1, p2, p3;
                V2<G>::lds(xs + pb0 + qoff[k], p0, p1);
                V2<G>::lds(xs + pb1 + qoff[k], p2, p3);
                c0 = fma(rq, p0, c0); c1 = fma(rq, p1, c1); c2 = fma(rq, p2, c2); c3 = fma(rq, p3, c3);
            }
        }
        a0 += c0; a1 += c1; a2 += c2; a3 += c3;
        if (b9) {
            G p0, p1;
            V2<G>::lds(xs + pb0 + kTile / 4, p0, p1);
            a0 = fma(r9, p0, a0);
            a1 = fma(r9, p1, a1);
        }
        if (top) consumer_release(&c.rempty[eslot], lane);
        if (strad) {
            if (!mbar_wait(&c.rfull[cslot], cph, errf)) { ok = false; break; }
            const G *hp = reinterpret_cast<const G *>(ring_base + cslot * gb);
            G p2, p3;
            V2<G>::lds(hp + pb0, p2, p3);
            a2 = fma(rnL, p2, a2);
            a3 = fma(rnL, p3, a3);
            consumer_release(&c.rempty[cslot], lane);
            if (++cslot == RS) { cslot = 0; cph ^= 1; }
        }
        for (uint32_t mh = hmask; mh; mh &= mh - 1) {
            if (!mbar_wait(&c.rfull[cslot], cph, errf)) { ok = false; break; }
            const G *pp = reinterpret_cast<const G *>(ring_base + cslot * gb);
            const G rr = wr[n - 1 - kTileBits - (__ffs(mh) - 1)];
            G p0, p1, p2, p3;
            V2<G>::lds(pp + pb0, p0, p1);
            V2<G>::lds(pp + pb1, p2, p3);
            a0 = fma(rr, p0, a0); a1 = fma(rr, p1, a1); a2 = fma(rr, p2, a2); a3 = fma(rr, p3, a3);
            consumer_release(&c.rempty[cslot], lane);
            if (++cslot == RS) { cslot = 0; cph ^= 1; }
        }
        if (!ok) break;

        const G acc[4] = {a0, a1, a2, a3};
        const G xv[4] = {x0, x1, x2, x3};
        O o[4];
        double cs = 0.0;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const G Tv = acc[j];
            if constexpr (S == ST_H1) {
                o[j] = static_cast<O>(p.h * Tv);
            } else if constexpr (S == ST_H2 || S == ST_H3) {
                o[j] = static_cast<O>(static_cast<G>(p.cx) * xv[j] + static_cast<G>(p.hc) * Tv);
            } else {
                const double D = p.cx * static_cast<double>(xa[j]) + p.hc * static_cast<double>(Tv);
                o[j] = xb[j] + D;
                cs += fabs(D);
            }
        }
        V2<O>::stg(out + gT + pb0, o[0], o[1], once);
        V2<O>::stg(out + gT + pb1, o[2], o[3], once);
        consumer_release(&c.empty[b], lane);
        ++it;

        if constexpr (Tr::FINAL) {
            // this warp's share of the system's L1 norm goes to a fixed slot; the
            // system's last warp adds the slots in order and applies the exit rule
            const double ws = warp_sum(cs);
            double *slots = p.partials + size_t(sys) * (tps * kConsumerWarps);
            unsigned tk = 0;
            if (lane == 0) {
                slots[t * kConsumerWarps + warp] = ws;
                __threadfence();
                tk = atomicAdd(p.counters + sys, 1u);
            }
            tk = __shfl_sync(0xffffffffu, tk, 0);
            if (tk == unsigned(tps * kConsumerWarps) - 1u) {
                __threadfence();
                double s = 0.0;
                for (unsigned long long i = lane; i < tps * kConsumerWarps; i += 32) s += __ldcg(slots + i);
                s = warp_sum(s);
                if (lane == 0) {
                    BatchExit &ex = p.ex[sys];
                    const unsigned long long step = ex.steps_done;
                    ex.last_checksum = s;
                    ex.steps_done = step + 1;
                    if (p.exit_rule) {
                        if (s < p.thresh) {
                            ex.early_stop += 1;
                            ex.steps_at_stop = step;
                        } else {
                            ex.early_stop = 0;
                        }
                        if (ex.early_stop > p.stop_count) ex.converged = 1;
                    }
                    if (ex.converged || step + 1 >= p.max_steps) {
                        __threadfence();
                        *reinterpret_cast<volatile int *>(&ex.done) = 1;
                        atomicSub(p.active, 1);
                    }
                    p.counters[sys] = 0u;
                    __threadfence();
                }
            }
        }
    }
    if (!ok || *errf) atomicExch(p.error, 1);
}

template <int S, typename E> constexpr int batch_smem_bytes() {
    using G = typename StageT<S, E>::G;
    constexpr int gb = TileLayout<S, E>::gb;
    constexpr int wr = kConsumerWarps * kWarpRates * int(sizeof(G));
    constexpr int RS0 = (kSmemMax - kCtrlBytes - 2 * gb - wr) / gb;
    constexpr int RS = RS0 < kMaxRing ? RS0 : kMaxRing;
    return kCtrlBytes + 2 * gb + RS * gb + wr;
}

}  // namespace tasep
