// meq_tile.cuh - matrix-free generator sweep for n > kTileBits.
//
// One launch applies the TASEP generator M once to a "gathered" vector g and
// fuses the stage's epilogue (axpy, RK4 combination, L1 norm of the
// increment, exit rule).  M is never stored: each state i gathers its
// in-flows (entry, diagonal, exit, hops) from bit-flipped neighbours, in the
// reference's row order (src/lib/solv.c:81-135; src/lib/matgen.c:29-67):
//   1. entry from i - 2^(n-1) if bit n-1 of i is set, rate r[0];
//   2. diagonal -(r[n][b0] + r[0][!b(n-1)] + sum_j r[n-1-j][!b_j & b_(j+1)]),
//      subtracted in that order;
//   3. exit from i+1 if bit 0 is clear, rate r[n];
//   4. hops from i + 2^k for k ascending where b_k & !b_(k+1), rate r[n-1-k].
//
// Layout: the state vector is one flat array in reference index order.  A
// tile is 2^kTileBits consecutive states; tile T's index holds the state's
// bits >= kTileBits.  Per CTA (one per SM, persistent over tiles):
//   * a producer warp streams, with cp.async.bulk (no multicast), the tile of
//     g into a double-buffered stage, then every partner tile this tile
//     needs - the entry tile, the lower half of tile T+1 (the hop straddling
//     the tile edge) and one tile per active high hop - into a ring of
//     shared-memory slots; per-state extra inputs go straight to registers;
//   * 16 consumer warps; thread t owns the state pairs {2t, 2t+1} and
//     {2t+1024, 2t+1025}.  The hop inside a pair is a register move, the one
//     between neighbouring pairs a shuffle, other in-tile hops read the staged
//     tile (a per-thread list of partner offsets), high hops read the ring
//     slots in ascending bit order.  The diagonal's low part (everything up to
//     bit 9, which precedes the tile-level terms in the reference's
//     subtraction order) comes from a table built once per launch; the exact
//     stages subtract the tile-level terms in order, so the reference's
//     rounding sequence is kept exactly, while the reassociating RK4 sweeps
//     look their sum up in five-bit window tables.
// All CTAs sweep the tiles together (natural order, except that the entry bit
// toggles fastest: sweep_tile), so partner tiles up to a few tens of MB ahead
// are still in L2 when they are gathered.
#pragma once

#include "meq_common.cuh"

namespace tasep {

constexpr int kTileBits = 11;
constexpr int kTile = 1 << kTileBits;               // states per tile
constexpr int kConsumerWarps = 16;
constexpr int kConsumers = kConsumerWarps * 32;      // 512: one group of 4 states each
constexpr int kTileThreads = kConsumers + 32;        // + producer warp
constexpr int kMaxRing = 16;                       // partner ring slots (upper bound)
constexpr int kSmemMax = 232448;                   // dynamic shared memory per CTA on sm_100
static_assert(kTile / 4 == kConsumers, "one group of four states per consumer thread");

// L2 cache policy of the tile sweep (TileParams::l2_near, l2_flags).
//
// In the sweep order a tile is first read as a hop partner of an earlier tile
// (T needs T + 2^u, 2^(u+1) tiles ahead) and last read as its own tile; after
// that no later tile needs it (the entry partner, one tile later, excepted).
// So the lines worth keeping are those of partner reads whose own read comes
// within the L2 window: hop bits u < l2_near are read evict_last; the others
// (partners whose own read is further away than L2 can hold) and, with
// L2F_OWN_FIRST, the own-tile reads are evict_first, so they do not push the
// useful lines out.  With L2F_DEMOTE the consumers lower the lines of a tile
// they have just received to evict_normal, so a tile that was kept as a
// partner stops occupying the evict_last class once it is no longer needed.
enum : int { L2F_OWN_FIRST = 1, L2F_DEMOTE = 2, L2F_FAR_FIRST = 4 };

struct TileParams {
    int n;
    int l2_near;   // hop bits (tile-index bits) read evict_last as partners
    int l2_flags;  // L2F_*
    unsigned long long ntiles;
    const void *g;             // gathered vector
    const void *s0, *s1, *s2;  // per-state extra inputs
    void *out;
    double h, hc;              // step and stage coefficient
    double cx;                 // RK4 sweeps 2, 3: coefficient of the own gathered value; 4: of v2
    double t;                  // stage time
    double *partials;          // per-CTA L1 partial sums (final stages)
    unsigned int *counter;     // last-CTA ticket
    ExitState *ex;
    unsigned long long step;   // step index (exit rule)
    double thresh;             // stop_tol * h
    int stop_count;
    int exit_rule;
    int skip_if_done;
    // Bounded waits: limit in ns (0 = kWaitLimitNs).  skip_copy_plus1 = k+1
    // makes CTA 0's producer leave out its k-th partner copy, so the consumers'
    // wait for it expires (tests of the error path; 0 = off).
    unsigned long long wait_ns;
    int skip_copy_plus1;
    RateSpec rs;
};

// Per-stage types: G gathered, O output, X0..X2 extras (NX used).
template <int S, typename E> struct StageT;
template <typename E> struct StageT<ST_APPLY, E> {
    using G = double; using O = double; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 0; static constexpr bool FINAL = false; static constexpr bool EXACT = true;
};
template <typename E> struct StageT<ST_REF, E> {
    using G = double; using O = double; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 0; static constexpr bool FINAL = true; static constexpr bool EXACT = true;
};
template <typename E> struct StageT<ST_H1, E> {
    using G = double; using O = E; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 0; static constexpr bool FINAL = false; static constexpr bool EXACT = false;
};
template <typename E> struct StageT<ST_H2, E> {
    using G = E; using O = E; using X0 = E; using X1 = E; using X2 = E;
    static constexpr int NX = 0; static constexpr bool FINAL = false; static constexpr bool EXACT = false;
};
template <typename E> struct StageT<ST_H3, E> {
    using G = E; using O = E; using X0 = E; using X1 = E; using X2 = E;
    static constexpr int NX = 0; static constexpr bool FINAL = false; static constexpr bool EXACT = false;
};
template <typename E> struct StageT<ST_H4, E> {
    using G = E; using O = double; using X0 = E; using X1 = double; using X2 = double;
    static constexpr int NX = 2; static constexpr bool FINAL = true; static constexpr bool EXACT = false;
};
template <typename E> struct StageT<ST_U1, E> {
    using G = double; using O = double; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 0; static constexpr bool FINAL = false; static constexpr bool EXACT = true;
};
template <typename E> struct StageT<ST_U2, E> {
    using G = double; using O = double; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 1; static constexpr bool FINAL = false; static constexpr bool EXACT = true;
};
template <typename E> struct StageT<ST_U3, E> : StageT<ST_U2, E> {};
template <typename E> struct StageT<ST_U4, E> {
    using G = double; using O = double; using X0 = double; using X1 = double; using X2 = double;
    static constexpr int NX = 3; static constexpr bool FINAL = true; static constexpr bool EXACT = true;
};

struct TileCtrl {
    uint64_t full[2], empty[2];
    uint64_t rfull[kMaxRing], rempty[kMaxRing];
    double wsum[kConsumerWarps];
    double rates_d[kMaxR + 1];
    float rates_f[kMaxR + 3];
    int skip;
    int err;
    int is_last;
    int pad;
};
constexpr int kCtrlBytes = 1024;
static_assert(sizeof(TileCtrl) <= kCtrlBytes, "control block");

template <int S, typename E> struct TileLayout {
    using Tr = StageT<S, E>;
    static constexpr int gb = kTile * sizeof(typename Tr::G);
    static constexpr int x0b = Tr::NX > 0 ? kTile * sizeof(typename Tr::X0) : 0;
    static constexpr int x1b = Tr::NX > 1 ? kTile * sizeof(typename Tr::X1) : 0;
    static constexpr int x2b = Tr::NX > 2 ? kTile * sizeof(typename Tr::X2) : 0;
    static constexpr int stage = gb;     // the gathered tile; extras go straight to registers
    static constexpr int dtab = 2 * gb;  // low diagonal prefixes, for top bit clear / set
    // tile-level diagonal sums of the reassociating stages: 6 windows x 32 entries
    static constexpr int dst = Tr::EXACT ? 0 : int(6 * 32 * sizeof(typename Tr::G));
    // as many partner slots as shared memory holds
    static constexpr int RS0 = (kSmemMax - kCtrlBytes - 2 * stage - dtab - dst) / gb;
    static constexpr int RS = RS0 < kMaxRing ? RS0 : kMaxRing;
    static constexpr int bytes = kCtrlBytes + 2 * stage + RS * gb + dtab + dst;
    static_assert(RS >= 4, "partner ring too shallow");
};

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }

// Sweep order of the tiles.  A partner tile is read from DRAM unless it is
// still in L2 from a recent read, and L2 holds about 2^23 doubles, so only
// partners a limited sweep distance away hit.  The entry partner (the top
// tile-index bit, half of all tiles) is the most frequent far partner; letting
// that bit toggle fastest puts every tile next to its entry partner.  The
// other partners' sweep distances double, which moves one hop pair out of
// the L2 window (a quarter of the tiles): 1.5 instead of 1.75 far-partner
// reads per tile at n = 28.
__device__ __forceinline__ uint32_t sweep_tile(uint32_t o, int ntb) {
    return ntb >= 2 ? ((o >> 1) | ((o & 1u) << (ntb - 1))) : o;
}

template <typename G> __device__ __forceinline__ G rate_of(const TileCtrl &c, int i);
template <> __device__ __forceinline__ double rate_of<double>(const TileCtrl &c, int i) { return c.rates_d[i]; }
template <> __device__ __forceinline__ float rate_of<float>(const TileCtrl &c, int i) { return c.rates_f[i]; }

// kTuned: the instantiation that honours a non-default L2 policy and the
// wait-expiry test hook.  The default launch uses the lean one: the producer
// thread that issues the bulk copies is on the sweep's critical path, and the
// per-copy policy selection alone cost 2-3 % of the step time.
template <int S, typename E, bool kTuned>
__global__ void __launch_bounds__(kTileThreads, 1) meq_tile_kernel(const __grid_constant__ TileParams p) {
    using Tr = StageT<S, E>;
    using G = typename Tr::G;
    using O = typename Tr::O;
    using X0 = typename Tr::X0;
    using X1 = typename Tr::X1;
    using X2 = typename Tr::X2;
    using A = Ar<G, Tr::EXACT>;
    using LY = TileLayout<S, E>;

    extern __shared__ __align__(128) unsigned char tile_smem[];
    TileCtrl &c = *reinterpret_cast<TileCtrl *>(tile_smem);
    unsigned char *stage_base = tile_smem + kCtrlBytes;
    unsigned char *ring_base = stage_base + 2 * LY::stage;
    G *dtab = reinterpret_cast<G *>(ring_base + LY::RS * LY::gb);
    G *dst = dtab + 2 * kTile;  // reassociating stages only
    constexpr int RS = LY::RS;

    const int tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int n = p.n;
    const int ntb = n - kTileBits;  // tile-index bits (>= 1)
    // tile indices fit 32 bits (at most 2^22 tiles for n <= 33); 32-bit masks
    // and bit scans cost half the integer instructions of 64-bit ones
    const uint32_t ntiles = uint32_t(p.ntiles);

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
    if (tid <= n) {
        const double r = rate_at(p.rs, tid, p.t);
        c.rates_d[tid] = r;
        c.rates_f[tid] = static_cast<float>(r);
    }
    // up to here only parameters and shared memory: the previous sweep may
    // still be running
    grid_dep_wait();
    if (tid == 0) c.skip = (p.skip_if_done && p.ex) ? *reinterpret_cast<volatile int *>(&p.ex->done) : 0;
    __syncthreads();
    if (c.skip) return;
    volatile int *errf = &c.err;
    const uint64_t wait_ns = p.wait_ns ? p.wait_ns : kWaitLimitNs;

    const G *__restrict__ g = static_cast<const G *>(p.g);

    if (warp == kConsumerWarps) {
        // ---------------- producer ----------------
        if (lane == 0) {
            const uint64_t keep = policy_evict_last();    // near partners: read again as own tile soon
            const uint64_t normal = policy_evict_normal();
            const uint64_t first = policy_evict_first();
            const uint64_t own_pol = (kTuned && (p.l2_flags & L2F_OWN_FIRST)) ? first : normal;
            const uint64_t far_pol = (kTuned && (p.l2_flags & L2F_FAR_FIRST)) ? first : keep;
            const uint64_t ent_pol = (kTuned && (p.l2_flags & L2F_DEMOTE)) ? normal : keep;
            const int near = p.l2_near;
            const bool skip_copy = kTuned && p.skip_copy_plus1 > 0 && blockIdx.x == 0;
            uint32_t it = 0, cur = 0;
            bool ok = true;
            for (uint32_t ord = blockIdx.x; ord < ntiles && ok; ord += gridDim.x, ++it) {
                const uint32_t T = sweep_tile(ord, ntb);
                const int b = it & 1;
                if (it >= 2 && !mbar_wait(&c.empty[b], ((it >> 1) - 1) & 1, errf, wait_ns)) break;
                unsigned char *st = stage_base + b * LY::stage;
                mbar_arrive_expect_tx(&c.full[b], LY::stage);
                bulk_g2s(st, g + (unsigned long long)T * kTile, LY::gb, &c.full[b], own_pol);  // read again only as a far partner
                // partner tiles, in the order the consumers add them
                const bool top = (T >> (ntb - 1)) & 1;
                const bool strad = !(T & 1);
                const uint32_t hmask = ntb >= 2 ? (T & ~(T >> 1) & ((1u << (ntb - 1)) - 1)) : 0u;
                const int np = int(top) + int(strad) + __popc(hmask);
                uint32_t hm = hmask;
                for (int q = 0; q < np; ++q) {
                    unsigned long long src;
                    uint32_t bytes = LY::gb;
                    uint64_t pol = keep;
                    if (q == 0 && top) {
                        src = T - (1ull << (ntb - 1));
                        if constexpr (kTuned) pol = ent_pol;
                    } else if (q == int(top) && strad) {
                        src = T + 1;
                        bytes = LY::gb / 2;
                    } else {
                        const int u = __ffs(hm) - 1;
                        hm &= hm - 1;
                        src = T + (1ull << u);
                        if constexpr (kTuned)
                            if (u >= near) pol = far_pol;
                    }
                    const int slot = cur % RS;
                    if (cur >= RS && !mbar_wait(&c.rempty[slot], ((cur / RS) - 1) & 1, errf, wait_ns)) {
                        ok = false;
                        break;
                    }
                    if (!(kTuned && skip_copy && cur + 1 == uint32_t(p.skip_copy_plus1))) {
                        mbar_arrive_expect_tx(&c.rfull[slot], bytes);
                        bulk_g2s(ring_base + slot * LY::gb, g + src * kTile, bytes, &c.rfull[slot], pol);
                    }
                    ++cur;
                }
            }
            if (!ok || *errf) {
                atomicExch(&p.ex->error, 1);
                // let every copy issued so far complete before the CTA can exit
                for (int b = 0; b < 2; ++b) {
                    const uint32_t uses = (it + 1 - b) / 2;  // tiles started on buffer b
                    if (uses) mbar_drain(&c.full[b], (uses - 1) & 1, 100000000ull);
                }
                for (int s = 0; s < RS; ++s) {
                    const uint32_t uses = cur > uint32_t(s) ? (cur - 1 - s) / RS + 1 : 0;
                    if (uses) mbar_drain(&c.rfull[s], (uses - 1) & 1, 100000000ull);
                }
            }
        }
        return;
    }

    // ---------------- consumers ----------------
    // Thread t owns two pairs of states: P0 = {2t, 2t+1} and P1 = {2t+1024,
    // 2t+1025} (local indices).  State bit 0 lies inside a pair, bits 1..9 are
    // t, bit 10 selects the pair.  A warp's 16-byte accesses to a pair array
    // cover 512 contiguous bytes, so shared-memory reads are conflict free.
    //
    // Low diagonal prefixes: d = 0; -r[n] if b0; -r[0] if top clear; then
    // -r[n-1-j] for j = 0..9 where b_j = 0, b_(j+1) = 1 (src/lib/solv.c:103-116).
    for (int l = tid; l < kTile; l += kConsumers) {
        for (int tp = 0; tp < 2; ++tp) {
            G d = G(0);
            if (l & 1) d = A::sub(d, rate_of<G>(c, n));
            if (!tp) d = A::sub(d, rate_of<G>(c, 0));
            for (int j = 0; j < kTileBits - 1; ++j)
                if (!((l >> j) & 1) && ((l >> (j + 1)) & 1)) d = A::sub(d, rate_of<G>(c, n - 1 - j));
            dtab[tp * kTile + l] = d;
        }
    }
    if constexpr (!Tr::EXACT) {
        // Tile-level diagonal: the sum of r[n-1-11-u] over the tile-index
        // pairs u with bit u clear and bit u+1 set, looked up in windows of
        // five tile-index bits: window w covers u = 4w..4w+3, entry e holds
        // the sum over those pairs that e's bits select.  Stages that must
        // keep the reference's subtraction order run the loop below instead.
        for (int l = tid; l < 6 * 32; l += kConsumers) {
            const int w = l >> 5, e = l & 31;
            G v = G(0);
            for (int j = 0; j < 4; ++j) {
                const int u = 4 * w + j;
                if (u <= ntb - 2 && !((e >> j) & 1) && ((e >> (j + 1)) & 1)) v += rate_of<G>(c, n - 1 - kTileBits - u);
            }
            dst[l] = v;
        }
    }
    const int nwin = (ntb + 2) / 4;  // windows holding a pair u <= ntb - 2
    const G rn = rate_of<G>(c, n), r0 = rate_of<G>(c, 0), rn1 = rate_of<G>(c, n - 1);
    const G r9 = rate_of<G>(c, n - 10), rnL = rate_of<G>(c, n - kTileBits);
    consumer_sync();

    const uint64_t once = policy_evict_first();
    const bool demote = kTuned && (p.l2_flags & L2F_DEMOTE) != 0;
    O *__restrict__ out = static_cast<O *>(p.out);
    const uint32_t t9 = tid;              // state bits 1..9
    const int pb0 = 2 * tid;              // local index of P0
    const int pb1 = 2 * tid + kTile / 2;  // local index of P1
    const bool b9 = (t9 >> 8) & 1;        // state bit 9 (warp-uniform)
    const bool b1clear = !(t9 & 1);       // state bit 1 clear
    // In-tile hops k = q+1 (q = 0..7) need t bit q set and bit q+1 clear: a
    // per-thread constant.  At most 4 such q; keep their partner offsets and
    // rates in registers, in ascending q (the reference's order).
    int qcnt = 0;
    int qoff[4];
    G qrate[4];
    {
        uint32_t hq = t9 & ~(t9 >> 1) & 0xFFu;
        qcnt = __popc(hq);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int q = hq ? __ffs(hq) - 1 : 0;
            hq &= hq - 1;
            qoff[k] = 2 << q;
            qrate[k] = rate_of<G>(c, n - 2 - q);
        }
    }
    double cs = 0.0;
    uint32_t it = 0;
    int cslot = 0;     // next ring slot to consume
    uint32_t cph = 0;  // its fill parity
    bool ok = true;

    for (uint32_t ord = blockIdx.x; ord < ntiles; ord += gridDim.x, ++it) {
        const uint32_t T = sweep_tile(ord, ntb);
        const int b = it & 1;
        const bool top = (T >> (ntb - 1)) & 1;
        const bool strad = !(T & 1);
        const uint32_t lowmask = ntb >= 2 ? ((1u << (ntb - 1)) - 1) : 0u;
        const uint32_t hmask = T & ~(T >> 1) & lowmask;
        const uint32_t dhmask = ~T & (T >> 1) & lowmask;
        const unsigned long long gT = (unsigned long long)T * kTile;

        // per-state extra inputs, read once straight into registers; they are
        // only needed in the epilogue, so their latency hides behind the sweep
        X0 xa[4];
        X1 xb[4];
        X2 xc[4];
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
        if constexpr (Tr::NX > 2) {
            const X2 *s = static_cast<const X2 *>(p.s2) + gT;
            V2<X2>::ldg(s + pb0, xc[0], xc[1], once);
            V2<X2>::ldg(s + pb1, xc[2], xc[3], once);
        }
        G a0 = G(0), a1 = G(0), a2 = G(0), a3 = G(0);
        int eslot = 0;
        if (top) {  // 1. entry
            eslot = cslot;
            if (!mbar_wait(&c.rfull[eslot], cph, errf, wait_ns)) { ok = false; break; }
            const G *ent = reinterpret_cast<const G *>(ring_base + eslot * LY::gb);
            G e0, e1, e2, e3;
            V2<G>::lds(ent + pb0, e0, e1);
            V2<G>::lds(ent + pb1, e2, e3);
            a0 = A::madd(a0, r0, e0); a1 = A::madd(a1, r0, e1);
            a2 = A::madd(a2, r0, e2); a3 = A::madd(a3, r0, e3);
            if (++cslot == RS) { cslot = 0; cph ^= 1; }  // released after the in-tile terms below
        }
        if (!mbar_wait(&c.full[b], (it >> 1) & 1, errf, wait_ns)) { ok = false; break; }
        const G *xs = reinterpret_cast<const G *>(stage_base + b * LY::stage);
        // this was the tile's last read of the sweep: its lines leave the evict_last class
        if (demote && tid < LY::gb / 128) l2_demote_line(reinterpret_cast<const unsigned char *>(g + gT) + tid * 128);

        G x0, x1, x2, x3;
        V2<G>::lds(xs + pb0, x0, x1);
        V2<G>::lds(xs + pb1, x2, x3);
        // 2. diagonal: low prefix from the table, then j = 10 and j >= 11
        const G *dt = dtab + (top ? kTile : 0);
        G d0, d1, d2, d3;
        V2<G>::lds(dt + pb0, d0, d1);
        V2<G>::lds(dt + pb1, d2, d3);
        if (!strad) {  // j = 10: b10 = 0 (P0), b11 = 1
            d0 = A::sub(d0, rnL); d1 = A::sub(d1, rnL);
        }
        if constexpr (Tr::EXACT) {  // the reference's subtraction order
            uint32_t mh = dhmask;
            while (mh) {
                const int u = __ffs(mh) - 1;
                mh &= mh - 1;
                const G rr = rate_of<G>(c, n - 1 - kTileBits - u);
                d0 = A::sub(d0, rr); d1 = A::sub(d1, rr); d2 = A::sub(d2, rr); d3 = A::sub(d3, rr);
            }
        } else {  // reassociation allowed: one sum of the tile-level rates, from the windows
            G ds = dst[T & 31];
#pragma unroll
            for (int w = 1; w < 6; ++w)
                if (w < nwin) ds += dst[w * 32 + ((T >> (4 * w)) & 31)];
            d0 -= ds; d1 -= ds; d2 -= ds; d3 -= ds;
        }
        a0 = A::madd(a0, d0, x0); a1 = A::madd(a1, d1, x1);
        a2 = A::madd(a2, d2, x2); a3 = A::madd(a3, d3, x3);
        // 3. exit (b0 clear: the first state of each pair)
        a0 = A::madd(a0, rn, x1);
        a2 = A::madd(a2, rn, x3);
        // 4. hops, ascending bit
        {  // k = 0: second state of a pair with bit 1 clear <- first state of the next pair (next lane)
            const G n0 = __shfl_down_sync(0xffffffffu, x0, 1);
            const G n2 = __shfl_down_sync(0xffffffffu, x2, 1);
            if (b1clear) {
                a1 = A::madd(a1, rn1, n0);
                a3 = A::madd(a3, rn1, n2);
            }
        }
        // k = 1..8: partner pair t + 2^q for this thread's active q (ascending).
        // Stages that may reassociate collect them in a second accumulator so
        // the two dependency chains interleave.
        G c0 = G(0), c1 = G(0), c2 = G(0), c3 = G(0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (k < qcnt) {
                G p0, p1, p2, p3;
                V2<G>::lds(xs + pb0 + qoff[k], p0, p1);
                V2<G>::lds(xs + pb1 + qoff[k], p2, p3);
                if constexpr (Tr::EXACT) {
                    a0 = A::madd(a0, qrate[k], p0); a1 = A::madd(a1, qrate[k], p1);
                    a2 = A::madd(a2, qrate[k], p2); a3 = A::madd(a3, qrate[k], p3);
                } else {
                    c0 = A::madd(c0, qrate[k], p0); c1 = A::madd(c1, qrate[k], p1);
                    c2 = A::madd(c2, qrate[k], p2); c3 = A::madd(c3, qrate[k], p3);
                }
            }
        }
        if constexpr (!Tr::EXACT) {
            a0 += c0; a1 += c1; a2 += c2; a3 += c3;
        }
        if (b9) {  // k = 9: P0 states with b9 set <- pair t + 256 (bit 9 clear, bit 10 set)
            G p0, p1;
            V2<G>::lds(xs + pb0 + kTile / 4, p0, p1);
            a0 = A::madd(a0, r9, p0);
            a1 = A::madd(a1, r9, p1);
        }
        if (top) {
            consumer_release(&c.rempty[eslot], lane);
        }
        if (strad) {  // k = 10: P1 <- lower half of tile T+1
            const int slot = cslot;
            if (!mbar_wait(&c.rfull[slot], cph, errf, wait_ns)) { ok = false; break; }
            const G *hp = reinterpret_cast<const G *>(ring_base + slot * LY::gb);
            G p2, p3;
            V2<G>::lds(hp + pb0, p2, p3);
            a2 = A::madd(a2, rnL, p2);
            a3 = A::madd(a3, rnL, p3);
            consumer_release(&c.rempty[slot], lane);
            if (++cslot == RS) { cslot = 0; cph ^= 1; }
        }
        {
            uint32_t mh = hmask;  // k >= 11
            while (mh) {
                const int u = __ffs(mh) - 1;
                mh &= mh - 1;
                const int slot = cslot;
                if (!mbar_wait(&c.rfull[slot], cph, errf, wait_ns)) { ok = false; break; }
                const G *pp = reinterpret_cast<const G *>(ring_base + slot * LY::gb);
                const G rr = rate_of<G>(c, n - 1 - kTileBits - u);
                G p0, p1, p2, p3;
                V2<G>::lds(pp + pb0, p0, p1);
                V2<G>::lds(pp + pb1, p2, p3);
                a0 = A::madd(a0, rr, p0); a1 = A::madd(a1, rr, p1);
                a2 = A::madd(a2, rr, p2); a3 = A::madd(a3, rr, p3);
                consumer_release(&c.rempty[slot], lane);
                if (++cslot == RS) { cslot = 0; cph ^= 1; }
            }
            if (!ok) break;
        }

        // ---- epilogue ----
        const G acc[4] = {a0, a1, a2, a3};
        const G xv[4] = {x0, x1, x2, x3};
        O o[4];
        double s6[4];  // REF, U4: (k1 + 2 k2 + 2 k3 + k4), to be divided by 6
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const G Tv = acc[j];
            if constexpr (S == ST_APPLY) {
                o[j] = Tv;
            } else if constexpr (S == ST_REF) {
                const double kv = __dmul_rn(p.h, Tv);
                const double k2 = __dmul_rn(2.0, kv);
                s6[j] = __dadd_rn(__dadd_rn(__dadd_rn(kv, k2), k2), kv);
            } else if constexpr (S == ST_H1) {
                o[j] = static_cast<O>(p.h * Tv);
            } else if constexpr (S == ST_H2 || S == ST_H3) {  // v2 = (z - r) v1, w = (z + p) v2
                o[j] = static_cast<O>(static_cast<G>(p.cx) * xv[j] + static_cast<G>(p.hc) * Tv);
            } else if constexpr (S == ST_H4) {  // x' = x + (z w + q v2) / 24
                const double D = p.cx * static_cast<double>(xa[j]) + p.hc * static_cast<double>(Tv);
                o[j] = xb[j] + D;
                cs += fabs(D);
            } else if constexpr (S == ST_U1) {
                o[j] = __dadd_rn(__dmul_rn(p.hc, Tv), xv[j]);
            } else if constexpr (S == ST_U2 || S == ST_U3) {
                o[j] = __dadd_rn(__dmul_rn(p.hc, Tv), xa[j]);
            } else if constexpr (S == ST_U4) {
                const double x = xa[j];
                const double k1 = 2.0 * (xb[j] - x);
                const double k2 = 2.0 * (xc[j] - x);
                const double k3 = xv[j] - x;
                const double k4 = __dmul_rn(p.h, Tv);
                s6[j] = __dadd_rn(__dadd_rn(__dadd_rn(k1, 2.0 * k2), 2.0 * k3), k4);
            }
        }
        if constexpr (S == ST_REF || S == ST_U4) {
            double D[4];
            div6_rn4(s6, D);
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                o[j] = __dadd_rn(S == ST_REF ? double(xv[j]) : double(xa[j]), D[j]);
                cs += fabs(D[j]);
            }
        }
        V2<O>::stg(out + gT + pb0, o[0], o[1], once);
        V2<O>::stg(out + gT + pb1, o[2], o[3], once);
        consumer_release(&c.empty[b], lane);
    }
    if (!ok || *errf) {
        atomicExch(&p.ex->error, 1);
        __threadfence();
    }

    if constexpr (Tr::FINAL) {
        // deterministic CTA sum, then the last CTA reduces all partials in
        // CTA order and applies the exit rule (src/masterEquation.c:670-679)
        const double ws = warp_sum(cs);
        if (lane == 0) c.wsum[warp] = ws;
        consumer_sync();
        if (tid == 0) {
            double s = 0.0;
            for (int w = 0; w < kConsumerWarps; ++w) s += c.wsum[w];
            p.partials[blockIdx.x] = s;
            __threadfence();
            const unsigned t = atomicAdd(p.counter, 1u);
            c.is_last = (t == gridDim.x - 1);
        }
        consumer_sync();
        if (c.is_last && warp == 0) {
            __threadfence();
            double s = 0.0;
            for (unsigned i = lane; i < gridDim.x; i += 32) s += __ldcg(p.partials + i);
            s = warp_sum(s);
            if (lane == 0) {
                ExitState *ex = p.ex;
                // a step with an expired wait has no valid norm: NaN marks it
                // for callers that only read the norm (the status stays set)
                const bool failed = *reinterpret_cast<volatile int *>(&ex->error) != 0;
                ex->last_checksum = failed ? __longlong_as_double(0x7ff8000000000000ll) : s;
                ex->steps_done = p.step + 1;
                if (p.exit_rule) {
                    if (s < p.thresh) {
                        ex->early_stop += 1;
                        ex->steps_at_stop = p.step;
                    } else {
                        ex->early_stop = 0;
                    }
                    if (ex->early_stop > p.stop_count) {
                        ex->done = 1;
                        ex->converged = 1;
                    }
                }
                *p.counter = 0u;
                __threadfence();
            }
        }
    }
}

}  // namespace tasep
