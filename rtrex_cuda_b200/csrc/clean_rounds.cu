// Round-parallel replay of a large clean unit, order-faithful to initialClean +
// deleteAndClean (RTRex_Sequential/Escape/Decomposition.h:302-460, :147-283).
//
// The reference pops one edge at a time from a LIFO stack; a pop reads and
// writes only the records of its own edge and of the other two edges of each
// of its live triangles ("cells"), and the perVertex weights of the
// triangles' vertices -- which no pop ever reads.  So two pops whose cell
// sets are disjoint commute on everything a later pop can see, and the
// perVertex subtractions can be replayed afterwards if their order is known.
// One thread block replays one unit in rounds over the pending list (the
// stack, top first, then the unloaded seeds):
//
//  1. the first W pending items (the window, W = kRoundWarps; one warp each)
//     load their records and reserve their cells in a shared-memory hash table
//     (owner = the smallest window position that claims the cell; every claim
//     also adds its triangle weight to the cell's `acc`);
//  2. an item that owns all its cells is a winner: no earlier pending item
//     touches them, so its values are final and its pop is computed exactly;
//  3. winners commit unless an earlier pending item could change the sequence
//     in front of them: a winner that pushes (its pushes go right after it),
//     or a loser that might push when it pops.  A loser cannot push if none of
//     its live-triangle edges can fall below threshold even after every
//     claim in the window is subtracted (pe - acc >= thr, with a relative
//     margin of 1e-9 far above the rounding of those few subtractions) -- its
//     pop then inserts nothing, and later winners, disjoint from its cells,
//     may pass it;
//  4. the next window is the pending order after the round: the uncommitted
//     items, the pusher's pushes (last pushed first) right after the pusher,
//     then the rest of the list.
//
// The committed pops are those of the reference, each seeing the values it
// sees there; the order differs only between pops with disjoint cells.  The
// reference's pop order is kept as a linked list (`nx`, next pop; seeds
// chained in pop order, a pusher's pushes spliced in after it), ranked after
// the replay by pointer jumping.  Each pop logs its live triangle weights and
// third vertices in triangle order at its own triangle-list offset; the
// (vertex, rank) pairs of those subtractions, sorted, are folded into
// perVertex in the reference's order.
//
// An item whose list is longer than 32 entries ends the commits before it; at
// the front of the window it is popped alone by one warp, in 32-entry chunks.
#include "clean_units.cuh"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>

namespace rtr {

namespace {

constexpr int kRoundWarps = 16;
constexpr int kRoundBlock = 32 * kRoundWarps;
constexpr int kHashBits = 12;
constexpr int kHashSlots = 1 << kHashBits;  // a full window claims at most 16 x 65 cells
constexpr int kPend = 1024;                 // pending items held in shared memory
constexpr int kRefill = 512;                // items moved per refill from global memory
constexpr unsigned kNoCell = 0xffffffffu;
constexpr unsigned kNoOwner = 0xffffffffu;
constexpr unsigned kFull = 0xffffffffu;

// Per-round control words, double-buffered by round parity: a round's words
// are read by every thread after its commit barrier, and reset one round
// later (after a barrier that every reader has passed).
struct RoundCtl {
    int cut;             // a loser at this position might push: nothing after it commits
    int p1;              // first winner that pushes
    int npush;           // its pushes, in S.push
    unsigned committed;  // window positions that committed
};

struct RoundSmem {
    StackEntry pend[kPend];          // pending items after the window; pend[np-1] is the next in order
    StackEntry win[2][kRoundWarps];  // the window of a round (by parity), position k = warp k
    StackEntry push[64];             // the committing pusher's pushes, in push order
    unsigned hkey[kHashSlots];       // claimed cell (forward rank)
    unsigned hown[kHashSlots];       // smallest claiming window position
    double hacc[kHashSlots];         // sum of the claiming triangles' weights
    RoundCtl ctl[2];
    int wcnt[kRoundWarps];           // per-warp counts of a refill's kept seeds
    int np_solo;                     // pend count after a solo pop
    long long gtop_solo;
    int stop;
};

struct RoundArgs {
    const TriEntry* tl;
    EdgeRec* rec;
    double inv_n;
    const StackEntry* seeds;
    const UnitDesc* units;
    const uint64_t* order;
    StackEntry* stacks;
    int32_t* nx;        // [m] next pop in the reference's order (self at the tail)
    double* wbuf;       // [tl_len] a pop's live triangle weights, at its list offset, triangle order
    int32_t* zbuf;      // [tl_len] their third vertices
    int32_t* pop_wcnt;  // [m] live triangles a pop removed (0: none logged)
    unsigned* err;
    unsigned long long* total;
    unsigned long long* diag;
};

__device__ __forceinline__ int h_insert(RoundSmem& S, unsigned cell, unsigned owner, double w, bool add)
{
    unsigned slot = (cell * 2654435761u) >> (32 - kHashBits);
    for (int probe = 0; probe < kHashSlots; ++probe) {
        const unsigned k = atomicCAS(&S.hkey[slot], kNoCell, cell);
        if (k == kNoCell || k == cell) {
            atomicMin(&S.hown[slot], owner);
            if (add) atomicAdd(&S.hacc[slot], w);
            return (int)slot;
        }
        slot = (slot + 1) & (kHashSlots - 1);
    }
    return -1;
}

// Claims of one triangle's two other edges, both probes issued before either
// is resolved (the edges differ).
__device__ __forceinline__ void h_insert2(RoundSmem& S, unsigned c1, unsigned c2, unsigned owner, double w, int& s1,
                                          int& s2)
{
    unsigned a = (c1 * 2654435761u) >> (32 - kHashBits), b = (c2 * 2654435761u) >> (32 - kHashBits);
    unsigned ka = atomicCAS(&S.hkey[a], kNoCell, c1);
    unsigned kb = atomicCAS(&S.hkey[b], kNoCell, c2);
    s1 = s2 = -1;
    for (int probe = 0; probe < kHashSlots; ++probe) {
        if (ka == kNoCell || ka == c1) {
            s1 = (int)a;
            break;
        }
        a = (a + 1) & (kHashSlots - 1);
        ka = atomicCAS(&S.hkey[a], kNoCell, c1);
    }
    for (int probe = 0; probe < kHashSlots; ++probe) {
        if (kb == kNoCell || kb == c2) {
            s2 = (int)b;
            break;
        }
        b = (b + 1) & (kHashSlots - 1);
        kb = atomicCAS(&S.hkey[b], kNoCell, c2);
    }
    if (s1 >= 0) atomicMin(&S.hown[s1], owner);
    if (s2 >= 0) atomicMin(&S.hown[s2], owner);
    if (s1 >= 0) atomicAdd(&S.hacc[s1], w);
    if (s2 >= 0) atomicAdd(&S.hacc[s2], w);
}

__device__ __forceinline__ void h_clear(RoundSmem& S, int slot)
{
    if (slot >= 0) {
        S.hkey[slot] = kNoCell;
        S.hown[slot] = kNoOwner;
        S.hacc[slot] = 0.0;
    }
}

// Warp 0: move the oldest pending items (the bottom of pend) to the unit's
// global region so that `need` more fit.  False when that region is full.
__device__ bool pend_spill(RoundSmem& S, StackEntry* gm, int64_t cap, int& np, int64_t& gtop, int need)
{
    const int lane = threadIdx.x & 31;
    int s = kPend / 2;
    if (np + need - s > kPend) s = np + need - kPend;
    if (s > np) s = np;
    if (gtop + s > cap) return false;
    for (int j = lane; j < s; j += 32) gm[gtop + j] = S.pend[j];
    __syncwarp();
    for (int base = 0; base < np - s; base += 32) {
        const int j = base + lane;
        StackEntry tmp{};
        if (j < np - s) tmp = S.pend[s + j];
        __syncwarp();
        if (j < np - s) S.pend[j] = tmp;
        __syncwarp();
    }
    gtop += s;
    np -= s;
    return true;
}

// Item k (warp-uniform) of the pending order after a round: the uncommitted
// window items before the pusher P, the pushes (last pushed first), the
// uncommitted items after P, then pend from its top.
__device__ __forceinline__ StackEntry pending_item(const RoundSmem& S, int prev, unsigned U, int P, int npush, int nU,
                                                   int np, int k)
{
    const int lane = threadIdx.x & 31;
    const bool mine = (U >> lane) & 1u;
    const int pos = __popc(U & ((1u << lane) - 1u)) + (P >= 0 && lane > P ? npush : 0);
    const unsigned hit = __ballot_sync(kFull, mine && pos == k);
    if (hit) return S.win[prev][__ffs(hit) - 1];
    const int below = P >= 0 ? __popc(U & ((1u << P) - 1u)) : nU;
    if (k >= below && k < below + npush) return S.push[npush - 1 - (k - below)];
    return S.pend[np - 1 - (k - nU - npush)];
}

// Warp 0: the pop of an item with a list longer than 32 entries, alone in its
// round (deleteAndClean's loop body, Decomposition.h:152-281, 32 triangles at
// a time).  Its pushes go straight onto pend.
__device__ void solo_pop(const RoundArgs& a, RoundSmem& S, const StackEntry& c, StackEntry* gm, int64_t cap, int& np,
                         int64_t& gtop, unsigned long long& removed)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const PairSide ps = pair_side(c);
    const EdgeRec* r = a.rec + c.e;
    const unsigned long long ow = *reinterpret_cast<const unsigned long long*>(&r->cnt);
    const double pe_e = r->pe;
    const uint32_t s_e = (uint32_t)(ow >> 32) & SS_SUP;
    int nl_total = 0;
    if (s_e > 0) {
        const int32_t old = a.nx[c.e];
        int32_t prev = -1;  // the previous push of this pop
        for (int base = 0; base < c.cnt; base += 32) {
            const bool valid = base + lane < c.cnt;
            TriEntry t{};
            EdgeRec r1{}, r2{};
            r1.ss = SS_N;
            r2.ss = SS_N;
            if (valid) t = ld_entry(a.tl + c.t0 + base + lane);
            const int32_t rlw = ps.lower_is_a ? t.raz : t.rbz;
            const int32_t rhw = ps.lower_is_a ? t.rbz : t.raz;
            if (valid) {
                r1 = a.rec[rlw];
                r2 = a.rec[rhw];
            }
            const uint32_t c1 = r1.ss & SS_CODE, c2 = r2.ss & SS_CODE;
            const bool live = valid && c1 != SS_N && c2 != SS_N;
            bool f1 = false, f2 = false;
            if (live) {
                const double x1 = r1.pe - t.wgt, x2 = r2.pe - t.wgt;
                f1 = c1 != SS_S && x1 < r1.thr;
                f2 = c2 != SS_S && x2 < r2.thr;
                a.rec[rlw].pe = x1;
                a.rec[rhw].pe = x2;
                a.rec[rlw].ss = ((r1.ss & SS_SUP) - 1u) | (f1 ? SS_S : c1);
                a.rec[rhw].ss = ((r2.ss & SS_SUP) - 1u) | (f2 ? SS_S : c2);
            }
            const unsigned lm = __ballot_sync(kFull, live);
            const unsigned b1 = __ballot_sync(kFull, f1), b2 = __ballot_sync(kFull, f2);
            if (live) {
                const int k = __popc(lm & lt);
                a.wbuf[c.t0 + nl_total + k] = t.wgt;
                a.zbuf[c.t0 + nl_total + k] = t.z;
            }
            const int nl = __popc(lm);
            const int npc = __popc(b1) + __popc(b2);
            if (npc) {
                if (np + npc > kPend && !pend_spill(S, gm, cap, np, gtop, npc)) {
                    if (lane == 0) {
                        atomicOr(a.err, (unsigned)DEV_ERR_STACK_OVERFLOW);
                        S.stop = 1;
                    }
                    return;
                }
                const int before = __popc(b1 & lt) + __popc(b2 & lt);
                if (f1) S.pend[np + before] = StackEntry{rlw, ps.lower, t.z, ps.dlow, t.dz, (int32_t)r1.cnt, r1.t0};
                if (f2)
                    S.pend[np + before + (f1 ? 1 : 0)] =
                        StackEntry{rhw, ps.higher, t.z, ps.dhigh, t.dz, (int32_t)r2.cnt, r2.t0};
                __syncwarp();
                // sequence list: each push follows the previous one, the first the old successor
                for (int j = lane; j < npc; j += 32) {
                    const int32_t x = S.pend[np + j].e;
                    const int32_t pred = j > 0 ? S.pend[np + j - 1].e : (prev >= 0 ? prev : (old == c.e ? x : old));
                    a.nx[x] = pred;
                }
                prev = S.pend[np + npc - 1].e;
                np += npc;
            }
            nl_total += nl;
            __syncwarp();
        }
        if (prev >= 0 && lane == 0) a.nx[c.e] = prev;
        if (lane == 0) a.pop_wcnt[c.e] = nl_total;
    }
    // the own perEdge as in the windowed commit: k_pop_pe folds the logged weights
    a.rec[c.e].ss = (s_e - (uint32_t)nl_total) | SS_N;
    if (lane == 0) {
        if (nl_total == 0 && fabs(pe_e) > a.inv_n) atomicAdd(a.diag, 1ull);
        removed += (unsigned long long)nl_total;
    }
    __syncwarp();
}

__global__ void __launch_bounds__(kRoundBlock, 1) k_clean_rounds(RoundArgs a)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    RoundSmem& S = *reinterpret_cast<RoundSmem*>(smem_raw);
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const UnitDesc ud = a.units[(uint32_t)a.order[blockIdx.x]];
    StackEntry* gm = a.stacks + ud.stack_base;
    for (int i = tid; i < kHashSlots; i += kRoundBlock) {
        S.hkey[i] = kNoCell;
        S.hown[i] = kNoOwner;
        S.hacc[i] = 0.0;
    }
    if (tid == 0) {
        S.stop = 0;
        for (int q = 0; q < 2; ++q) S.ctl[q] = RoundCtl{kRoundWarps, kRoundWarps, 0, 0u};
    }
    // The pending list, identical in every thread: pend[0, np) (top = next),
    // the unit's global region gm[0, gtop) (top = next), seeds [seed_begin, sp).
    int np = 0;
    int64_t gtop = 0, sp = ud.seed_end;
    unsigned long long removed = 0;
    // this warp's item of the coming round (position wid of wn), window parity
    int cur = 1, wn = 0;
    bool solo = false;
    StackEntry c{};
    // the previous round's outcome (none before the first round)
    unsigned U = 0;
    int npush = 0, P = -1;
    __syncthreads();
    while (true) {
        // ---- next window (every warp, from the previous round's outcome)
        {
            const int nU = __popc(U);
            const int T = nU + npush;  // items in front of pend
            while (np < kRoundWarps && (gtop > 0 || sp > ud.seed_begin)) {
                // refill pend from below: the global region first, then the seeds
                StackEntry keep{};
                if (tid < np) keep = S.pend[tid];
                if (gtop > 0) {
                    const int k = (int)(gtop < kRefill ? gtop : kRefill);
                    __syncthreads();
                    if (tid < np) S.pend[k + tid] = keep;
                    for (int j = tid; j < k; j += kRoundBlock) S.pend[j] = gm[gtop - k + j];
                    gtop -= k;
                    np += k;
                } else {
                    // Seeds whose support is already 0 are retired here without a
                    // pop (support only decreases; such a pop touches no cell but
                    // its own and pushes nothing) and take no window slot.
                    static_assert(kRefill <= kRoundBlock, "one refill candidate per thread");
                    const int k = (int)(sp - ud.seed_begin < kRefill ? sp - ud.seed_begin : kRefill);
                    StackEntry se{};
                    bool kept = false;
                    if (tid < k) {
                        se = a.seeds[sp - k + tid];
                        const EdgeRec* r = a.rec + se.e;
                        kept = (r->ss & SS_SUP) > 0;
                        if (!kept) {
                            if (fabs(r->pe) > a.inv_n) atomicAdd(a.diag, 1ull);
                            a.rec[se.e].ss = SS_N;
                        }
                    }
                    const unsigned bal = __ballot_sync(kFull, kept);
                    if (lane == 0) S.wcnt[wid] = __popc(bal);
                    __syncthreads();
                    int below = 0, kk = 0;
                    for (int w = 0; w < kRoundWarps; ++w) {
                        const int cw = S.wcnt[w];
                        below += w < wid ? cw : 0;
                        kk += cw;
                    }
                    if (tid < np) S.pend[kk + tid] = keep;
                    if (kept) S.pend[below + __popc(bal & lt)] = se;  // seed order kept
                    sp -= k;
                    np += kk;
                }
                __syncthreads();
            }
            const int avail = T + np;
            solo = avail > 0 && pending_item(S, cur, U, P, npush, nU, np, 0).cnt > 32;
            const int nwn = solo ? 1 : (avail < kRoundWarps ? avail : kRoundWarps);
            const int tk = nwn > T ? nwn - T : 0;  // taken from pend
            const int ov = T > nwn ? T - nwn : 0;  // back onto pend
            const int nxt = cur ^ 1;
            if (wid < nwn) {
                c = pending_item(S, cur, U, P, npush, nU, np, wid);
                if (lane == 0) S.win[nxt][wid] = c;
            }
            int np1 = np - tk;
            if (np1 + ov > kPend) {  // move the oldest pending items to the global region
                const int sn = kPend / 2 < np1 ? kPend / 2 : np1;
                if (gtop + sn > ud.stack_cap) {
                    if (tid == 0) atomicOr(a.err, (unsigned)DEV_ERR_STACK_OVERFLOW);
                    break;
                }
                StackEntry keep{};
                for (int j = tid; j < sn; j += kRoundBlock) gm[gtop + j] = S.pend[j];
                if (sn + tid < np1) keep = S.pend[sn + tid];
                __syncthreads();
                if (sn + tid < np1) S.pend[tid] = keep;
                gtop += sn;
                np1 -= sn;
                __syncthreads();
            }
            // items nwn .. T-1 go back on top of pend (item nwn at the top)
            for (int k = nwn + wid; k < T; k += kRoundWarps) {
                const StackEntry x = pending_item(S, cur, U, P, npush, nU, np, k);
                if (lane == 0) S.pend[np1 + (T - 1 - k)] = x;
            }
            np = np1 + ov;
            wn = nwn;
            cur = nxt;
        }
        if (wn == 0) break;
        const int par = cur;  // control words of this round
        if (solo) {
            // an item with a longer list: popped alone by warp 0
            if (wid == 0) {
                solo_pop(a, S, c, gm, ud.stack_cap, np, gtop, removed);
                if (lane == 0) {
                    S.np_solo = np;
                    S.gtop_solo = gtop;
                }
            }
            __syncthreads();
            if (tid == 0) S.ctl[par ^ 1] = RoundCtl{kRoundWarps, kRoundWarps, 0, 0u};
            np = S.np_solo;
            gtop = S.gtop_solo;
            const bool stop = S.stop != 0;
            __syncthreads();  // S.np_solo is rewritten by the next solo round only after this
            if (stop) break;
            U = 0;
            npush = 0;
            P = -1;
            continue;
        }
        // ---- load: own record and sequence successor, entries, the two other records of each triangle
        const bool active = wid < wn;
        const bool lng = active && c.cnt > 32;  // ends the commits before it; takes no cells
        PairSide ps{};
        TriEntry t{};
        unsigned long long ow = 0;
        double ope = 0.0;
        int32_t succ = 0;
        bool valid = false;
        if (active && !lng) {
            ps = pair_side(c);
            valid = lane < c.cnt;
            const EdgeRec* r = a.rec + c.e;
            ow = *reinterpret_cast<const unsigned long long*>(&r->cnt);
            ope = r->pe;
            succ = a.nx[c.e];
            if (valid) t = ld_entry(a.tl + c.t0 + lane);
        }
        EdgeRec r1{}, r2{};
        r1.ss = SS_N;
        r2.ss = SS_N;
        const int32_t rlw = ps.lower_is_a ? t.raz : t.rbz;
        const int32_t rhw = ps.lower_is_a ? t.rbz : t.raz;
        if (valid) {
            r1 = a.rec[rlw];
            r2 = a.rec[rhw];
        }
        const uint32_t c1 = r1.ss & SS_CODE, c2 = r2.ss & SS_CODE;
        const bool live = valid && c1 != SS_N && c2 != SS_N;
        // ---- reserve (the own cell by the first lane without a triangle, lane 31 for a full list)
        const int ol = c.cnt < 32 ? c.cnt : 31;
        int so = -1, s1 = -1, s2 = -1;
        if (active && !lng && lane == ol) so = h_insert(S, (unsigned)c.e, (unsigned)wid, 0.0, false);
        if (live) h_insert2(S, (unsigned)rlw, (unsigned)rhw, (unsigned)wid, t.wgt, s1, s2);
        __syncthreads();
        // ---- decide
        RoundCtl& ctl = S.ctl[par];
        if (tid == 0) S.ctl[par ^ 1] = RoundCtl{kRoundWarps, kRoundWarps, 0, 0u};
        bool mine = !lng, may = lng;
        if (active && !lng && lane == ol) mine = so >= 0 && S.hown[so] == (unsigned)wid;
        if (live) mine = mine && s1 >= 0 && s2 >= 0 && S.hown[s1] == (unsigned)wid && S.hown[s2] == (unsigned)wid;
        const bool winner = __all_sync(kFull, mine) && active;
        double x1 = 0.0, x2 = 0.0;
        bool f1 = false, f2 = false;
        unsigned lm = 0, b1 = 0, b2 = 0;
        if (winner) {
            if (live) {
                x1 = r1.pe - t.wgt;
                x2 = r2.pe - t.wgt;
                f1 = c1 != SS_S && x1 < r1.thr;
                f2 = c2 != SS_S && x2 < r2.thr;
            }
            lm = __ballot_sync(kFull, live);
            b1 = __ballot_sync(kFull, f1);
            b2 = __ballot_sync(kFull, f2);
            if (lane == 0 && (b1 | b2)) atomicMin(&ctl.p1, wid);
        } else if (active) {
            if (live) {
                if (s1 < 0 || s2 < 0) {
                    may = true;
                } else {
                    if (c1 != SS_S) {
                        const double q = S.hacc[s1];
                        may = may || (r1.pe - q) - r1.thr < 1e-9 * (fabs(r1.pe) + q);
                    }
                    if (c2 != SS_S) {
                        const double q = S.hacc[s2];
                        may = may || (r2.pe - q) - r2.thr < 1e-9 * (fabs(r2.pe) + q);
                    }
                }
            }
            if (lane == ol && !lng && so < 0) may = true;
            if (__any_sync(kFull, may) && lane == 0) atomicMin(&ctl.cut, wid);
        }
        __syncthreads();
        // ---- commit
        const int p1 = ctl.p1;
        const int cutoff = ctl.cut < p1 + 1 ? ctl.cut : p1 + 1;
        if (winner && wid < cutoff) {
            const uint32_t s_e = (uint32_t)(ow >> 32) & SS_SUP;
            const int nl = __popc(lm);
            if (live) {
                a.rec[rlw].pe = x1;
                a.rec[rhw].pe = x2;
                a.rec[rlw].ss = ((r1.ss & SS_SUP) - 1u) | (f1 ? SS_S : c1);
                a.rec[rhw].ss = ((r2.ss & SS_SUP) - 1u) | (f2 ? SS_S : c2);
                const int k = __popc(lm & lt);
                a.wbuf[c.t0 + k] = t.wgt;
                a.zbuf[c.t0 + k] = t.z;
            }
            // every lane holds the same values: the same stores from all lanes.  The popped
            // edge's own perEdge keeps the value it has at the pop; k_pop_pe subtracts the
            // logged live weights (in triangle order) after the replay, off the round's path.
            a.rec[c.e].ss = (s_e - (uint32_t)nl) | SS_N;
            a.pop_wcnt[c.e] = nl;
            if (lane == 0) {
                if (nl == 0 && fabs(ope) > a.inv_n) atomicAdd(a.diag, 1ull);
                removed += (unsigned long long)nl;
                atomicOr(&ctl.committed, 1u << wid);
            }
            if (wid == p1) {
                // the pushes in the reference's order (triangle order, (lower,w)
                // before (higher,w)), spliced into the sequence list after this pop
                const int npu = __popc(b1) + __popc(b2);
                const int before = __popc(b1 & lt) + __popc(b2 & lt);
                if (f1) S.push[before] = StackEntry{rlw, ps.lower, t.z, ps.dlow, t.dz, (int32_t)r1.cnt, r1.t0};
                if (f2)
                    S.push[before + (f1 ? 1 : 0)] =
                        StackEntry{rhw, ps.higher, t.z, ps.dhigh, t.dz, (int32_t)r2.cnt, r2.t0};
                __syncwarp();
                for (int j = lane; j < npu; j += 32) {
                    const int32_t x = S.push[j].e;
                    a.nx[x] = j > 0 ? S.push[j - 1].e : (succ == c.e ? x : succ);
                }
                if (lane == 0) {
                    a.nx[c.e] = S.push[npu - 1].e;
                    ctl.npush = npu;
                }
            }
        }
        // every reader of the table is past the barrier above
        h_clear(S, so);
        h_clear(S, s1);
        h_clear(S, s2);
        __syncthreads();
        // ---- this round's outcome, for the next window
        const unsigned wmask = wn >= 32 ? kFull : (1u << wn) - 1u;
        U = wmask & ~ctl.committed;
        npush = ctl.npush;
        P = npush ? p1 : -1;
    }
    if (lane == 0 && removed) atomicAdd(a.total, (unsigned long long)(-(long long)removed));
}

__global__ void k_seq_self(int32_t* __restrict__ nx, int64_t m)
{
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < m; x += (int64_t)gridDim.x * blockDim.x)
        nx[x] = (int32_t)x;
}

// Seeds chained in pop order (highest slot first); the last one is the tail.
__global__ void k_seq_seeds(const UnitDesc* __restrict__ units, const uint64_t* __restrict__ order,
                            const StackEntry* __restrict__ seeds, int32_t* __restrict__ nx)
{
    const UnitDesc ud = units[(uint32_t)order[blockIdx.x]];
    for (int64_t j = ud.seed_begin + threadIdx.x; j < ud.seed_end; j += blockDim.x)
        nx[seeds[j].e] = j > ud.seed_begin ? seeds[j - 1].e : seeds[j].e;
}

__global__ void k_rank_init(const int32_t* __restrict__ nx, int32_t* __restrict__ dd, int64_t m)
{
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < m; x += (int64_t)gridDim.x * blockDim.x)
        dd[x] = nx[x] == (int32_t)x ? 0 : 1;
}

// One pointer-jumping step (Wyllie): distance to the tail.
__global__ void k_rank_step(const int32_t* __restrict__ nx, const int32_t* __restrict__ dd, int32_t* __restrict__ nx2,
                            int32_t* __restrict__ dd2, int64_t m)
{
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < m; x += (int64_t)gridDim.x * blockDim.x) {
        const int32_t y = nx[x];
        dd2[x] = y == (int32_t)x ? dd[x] : dd[x] + dd[y];
        nx2[x] = nx[y];
    }
}

__global__ void k_round_lens(const UnitDesc* __restrict__ units, const uint64_t* __restrict__ order, int64_t nbig,
                             const StackEntry* __restrict__ seeds, const int32_t* __restrict__ dd,
                             int64_t* __restrict__ len)
{
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nbig; b += (int64_t)gridDim.x * blockDim.x) {
        const UnitDesc ud = units[(uint32_t)order[b]];
        len[b] = (int64_t)dd[seeds[ud.seed_end - 1].e] + 1;
    }
}

// tpos[tail of unit b] = rank of that tail among all units' pops.
__global__ void k_round_tails(const UnitDesc* __restrict__ units, const uint64_t* __restrict__ order, int64_t nbig,
                              const StackEntry* __restrict__ seeds, const int32_t* __restrict__ nx,
                              const int64_t* __restrict__ len, const int64_t* __restrict__ base,
                              int32_t* __restrict__ tpos)
{
    for (int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; b < nbig; b += (int64_t)gridDim.x * blockDim.x) {
        const UnitDesc ud = units[(uint32_t)order[b]];
        tpos[nx[seeds[ud.seed_end - 1].e]] = (int32_t)(base[b] + len[b] - 1);
    }
}

// Entries of the vertex log per pop: its two endpoints and each logged third vertex.
__global__ void k_log_count(const int32_t* __restrict__ pop_wcnt, int64_t m, uint32_t* __restrict__ cnt)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
        cnt[e] = pop_wcnt[e] > 0 ? 2u + (uint32_t)pop_wcnt[e] : 0u;
}

// Sort keys (vertex, rank of the pop) of every logged subtraction.
__global__ void k_log_keys(const int32_t* __restrict__ pop_wcnt, const uint32_t* __restrict__ off, int64_t m,
                           const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                           const int32_t* __restrict__ nb, const EdgeRec* __restrict__ rec,
                           const int32_t* __restrict__ zbuf, const int32_t* __restrict__ nx,
                           const int32_t* __restrict__ dd, const int32_t* __restrict__ tpos, int pb,
                           uint64_t* __restrict__ keys, int32_t* __restrict__ inv, unsigned* __restrict__ err)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t wc = pop_wcnt[e];
        if (wc <= 0) continue;
        const int32_t tp = tpos[nx[e]];
        const int32_t pos = tp - dd[e];
        uint64_t* k = keys + off[e];
        if (tp < 0 || pos < 0 || (int64_t)pos >= m) {  // a pop outside every ranked list
            atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
            for (int32_t j = 0; j < wc + 2; ++j) k[j] = ~0ull;
            continue;
        }
        inv[pos] = (int32_t)e;
        const int64_t s = fwd[e];
        const int64_t t0 = rec[e].t0;
        k[0] = ((uint64_t)esrc[s] << pb) | (uint64_t)pos;
        k[1] = ((uint64_t)nb[s] << pb) | (uint64_t)pos;
        for (int32_t j = 0; j < wc; ++j) k[2 + j] = ((uint64_t)zbuf[t0 + j] << pb) | (uint64_t)pos;
    }
}

// perEdge of the edges that k_clean_rounds popped with live triangles: the
// record kept the value it had at the pop, and the pop's live weights are
// logged in triangle order at the edge's list offset; they are subtracted now
// in that order -- the popped edge's own fold in deleteAndClean
// (RTRex_Sequential/Escape/Decomposition.h:152-281) -- followed by the
// reference's residual check.  No pop reads a popped edge's perEdge (its
// triangles are no longer live), so moving the fold here changes no bit.
__global__ void k_pop_pe(EdgeRec* __restrict__ rec, const int32_t* __restrict__ pop_wcnt,
                         const double* __restrict__ wbuf, int64_t m, double inv_n, unsigned long long* __restrict__ diag)
{
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x) {
        const int32_t wc = pop_wcnt[e];
        if (wc <= 0) continue;
        const int64_t wo = rec[e].t0;
        double x = rec[e].pe;
        for (int32_t k = 0; k < wc; ++k) x -= wbuf[wo + k];
        rec[e].pe = x;
        if (fabs(x) > inv_n) atomicAdd(diag, 1ull);
    }
}

// perVertex of the round-replayed units: the logged subtractions of each
// vertex in the reference's pop order (within a pop, triangle order).
__global__ void k_pv_fold(const uint64_t* __restrict__ keys, int64_t cnt, int pb, const int32_t* __restrict__ inv,
                          const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                          const int32_t* __restrict__ nb, const EdgeRec* __restrict__ rec,
                          const int32_t* __restrict__ pop_wcnt, const double* __restrict__ wbuf,
                          const int32_t* __restrict__ zbuf, double* __restrict__ pv, unsigned* __restrict__ err)
{
    const uint64_t pmask = (1ull << pb) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < cnt; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t v = keys[i] >> pb;
        if (keys[i] == ~0ull || (i > 0 && (keys[i - 1] >> pb) == v)) continue;
        double x = pv[v];
        for (int64_t j = i; j < cnt && (keys[j] >> pb) == v; ++j) {
            const int32_t e = inv[keys[j] & pmask];
            if (e < 0) {
                atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
                continue;
            }
            const int64_t s = fwd[e];
            const int64_t wo = rec[e].t0;
            const int32_t wc = pop_wcnt[e];
            if ((uint64_t)esrc[s] == v || (uint64_t)nb[s] == v) {
                for (int32_t k = 0; k < wc; ++k) x -= wbuf[wo + k];
            } else {  // third vertex of one triangle: the run is ascending in z
                int32_t lo = 0, hi = wc - 1;
                while (lo < hi) {
                    const int32_t mid = (lo + hi) >> 1;
                    if ((uint64_t)zbuf[wo + mid] < v) lo = mid + 1;
                    else hi = mid;
                }
                x -= wbuf[wo + lo];
            }
        }
        pv[v] = x;
    }
}

}  // namespace

int clean_rounds_launch(rtr_graph* g, Scratch& sc, cudaStream_t side, EdgeRec* rec, const StackEntry* seeds,
                        const UnitDesc* units, const uint64_t* order, int64_t nbig, StackEntry* stacks,
                        RoundReplay* rr)
{
    const int64_t m = g->m;
    rr->nbig = nbig;
    rr->rec = rec;
    rr->seeds = seeds;
    rr->units = units;
    rr->order = order;
    rr->nx = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->nx2 = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->dd = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->dd2 = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->inv = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->pop_wcnt = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    rr->logcnt = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    rr->logoff = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    rr->logtmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(m + 1));
    rr->wbuf = (double*)sc.get(sizeof(double) * (g->tl_len + 1));
    rr->zbuf = (int32_t*)sc.get(sizeof(int32_t) * (g->tl_len + 1));
    const size_t nb8 = sizeof(int64_t) * (nbig + 1);
    rr->len = (int64_t*)sc.get(nb8);
    rr->ubase = (int64_t*)sc.get(nb8);
    rr->tmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nbig + 1));
    if (!rr->nx || !rr->nx2 || !rr->dd || !rr->dd2 || !rr->inv || !rr->pop_wcnt || !rr->logcnt || !rr->logoff ||
        !rr->logtmp ||
        !rr->wbuf || !rr->zbuf || !rr->len || !rr->ubase || !rr->tmp) {
        set_error("device allocation failed (clean rounds)");
        return RTR_ERR_CUDA;
    }
    cudaStream_t s = g->stream;
    const int kB = 256;
    RTR_CUDA_TRY(cudaMemsetAsync(rr->pop_wcnt, 0, sizeof(int32_t) * (m + 1), s));
    k_seq_self<<<grid_for(m, kB), kB, 0, s>>>(rr->nx, m);
    k_seq_seeds<<<(unsigned)nbig, kB, 0, s>>>(units, order, seeds, rr->nx);
    g->launches += 2;
    RTR_CUDA_TRY(cudaGetLastError());
    // the replay itself runs on the side stream, after everything above
    cudaEvent_t ready;
    RTR_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    cudaEventRecord(ready, s);
    cudaStreamWaitEvent(side, ready, 0);
    cudaEventDestroy(ready);
    RoundArgs ra{g->tl,   rec,      1 / (double)g->n, seeds,        units,
                 order,   stacks,   rr->nx,           rr->wbuf,     rr->zbuf,
                 rr->pop_wcnt, (unsigned*)(g->ctr + 1), g->ctr, g->ctr + 2};
    const size_t smem = sizeof(RoundSmem);
    RTR_CUDA_TRY(cudaFuncSetAttribute(k_clean_rounds, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_clean_rounds<<<(unsigned)nbig, kRoundBlock, smem, side>>>(ra);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    return RTR_OK;
}

int clean_rounds_finish(rtr_graph* g, Scratch& sc, RoundReplay* rr)
{
    cudaStream_t s = g->stream;
    const int64_t m = g->m, nbig = rr->nbig;
    const int kB = 256;
    const int gb = grid_for(nbig, kB), gm = grid_for(m, kB);
    k_pop_pe<<<gm, kB, 0, s>>>(rr->rec, rr->pop_wcnt, rr->wbuf, m, 1 / (double)g->n, g->ctr + 2);
    // rank every pop in the reference's order
    k_rank_init<<<gm, kB, 0, s>>>(rr->nx, rr->dd, m);
    const int steps = bits_for((uint64_t)m) + 1;
    for (int k = 0; k < steps; ++k) {
        k_rank_step<<<gm, kB, 0, s>>>(rr->nx, rr->dd, rr->nx2, rr->dd2, m);
        std::swap(rr->nx, rr->nx2);
        std::swap(rr->dd, rr->dd2);
    }
    k_round_lens<<<gb, kB, 0, s>>>(rr->units, rr->order, nbig, rr->seeds, rr->dd, rr->len);
    exclusive_scan_i64(rr->len, rr->ubase, nbig, rr->ubase + nbig, rr->tmp, s);
    int32_t* tpos = rr->nx2;  // free after the last step
    RTR_CUDA_TRY(cudaMemsetAsync(tpos, 0xff, sizeof(int32_t) * (m + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(rr->inv, 0xff, sizeof(int32_t) * (m + 1), s));
    k_round_tails<<<gb, kB, 0, s>>>(rr->units, rr->order, nbig, rr->seeds, rr->nx, rr->len, rr->ubase, tpos);
    k_log_count<<<gm, kB, 0, s>>>(rr->pop_wcnt, m, rr->logcnt);
    exclusive_scan_u32(rr->logcnt, rr->logoff, m, rr->logoff + m, rr->logtmp, s);
    g->launches += 2 + steps + 4 + 2 * 2;
    uint32_t nlog = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nlog, rr->logoff + m, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    if (nlog == 0) return RTR_OK;
    const int pb = bits_for((uint64_t)m);
    uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * ((size_t)nlog + 1));
    uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * ((size_t)nlog + 1));
    void* rtmp = sc.get(radix_temp_bytes(nlog));
    if (!keys || !alt || !rtmp) {
        set_error("device allocation failed (clean rounds log)");
        return RTR_ERR_CUDA;
    }
    unsigned* err = (unsigned*)(g->ctr + 1);
    k_log_keys<<<gm, kB, 0, s>>>(rr->pop_wcnt, rr->logoff, m, g->fwd, g->esrc, g->nbors, rr->rec, rr->zbuf, rr->nx,
                                 rr->dd, tpos, pb, keys, rr->inv, err);
    const int nbits = bits_for((uint64_t)g->n) + pb;
    uint64_t* sorted = radix_sort_u64(keys, alt, nlog, nbits, rtmp, s);
    k_pv_fold<<<grid_for(nlog, kB), kB, 0, s>>>(sorted, nlog, pb, rr->inv, g->fwd, g->esrc, g->nbors, rr->rec,
                                                 rr->pop_wcnt, rr->wbuf, rr->zbuf, g->pv, err);
    g->launches += 2 + 3 * ((nbits + 7) / 8);
    RTR_CUDA_TRY(cudaGetLastError());
    return RTR_OK;
}

}  // namespace rtr
