// Cascading clean, order-faithful to initialClean + deleteAndClean
// (RTRex_Sequential/Escape/Decomposition.h:302-460 and :147-283).
//
// The reference seeds every u<v edge below eps * 1/(du*dv) in slot order onto a
// LIFO stack and then pops: a popped edge removes each of its live triangles
// (no 'N' edge), subtracting the triangle weight from the two other edges and
// the three vertices, and pushes the other edges that fall below threshold.
// Floating-point sums make the survivor set depend on that exact order (a
// bulk-synchronous peel differs on order-sensitive inputs), so the device
// replays the same order -- but only where order can matter:
//
//  * a seed with no triangles is a no-op pop: it is marked 'N' directly;
//  * edges with triangles split into vertex-disjoint units (connected
//    components of the graph of triangle-carrying edges, by union-find with
//    hooking to the smaller root).  Every cell a pop touches (the popped edge,
//    the two other edges of each triangle, the three vertices) lies in the
//    popped edge's unit, and a cascade never leaves its unit, so each unit can
//    replay its own seeds (in slot order, popped last-first) and cascades
//    independently and still perform the reference's operations, in the
//    reference's order, on every cell;
//  * one warp replays one unit.  A pop is latency-bound, so its data is laid
//    out for two dependent round trips: (1) the popped edge's 32-byte record
//    and its triangle-list entries (which carry the triangle weight), then
//    (2) the records of the two other edges of every triangle and the third
//    vertex's weight.  Lists longer than 32 entries are taken 64 at a time
//    with the next window's entries fetched during the current window's
//    records (pop_edge); shorter ones take the single-window path (pop_short).
//    A window seed's first 32 entries are staged in shared memory by one TMA
//    bulk copy per seed (cp.async.bulk, completing on a per-warp mbarrier).
//    Entries are read evict-first (each list is read once), so streaming the
//    lists does not displace the edge records from L2.  (Warming the next
//    pop's lines with prefetch instructions was measured and costs more on
//    the single warp's critical path than it saves.)
//    The lanes take 32 triangles at a time, update the
//    distinct per-triangle cells in parallel, fold the shared cells (the
//    popped edge, its two endpoints) in triangle order, and append pushes in
//    the reference's push order (triangle order, (lower,w) before (higher,w)).
//    Seeds are loaded 32 at a time; support only decreases, so a seed whose
//    support is already 0 when loaded is retired without a pop.
#include "clean_units.cuh"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>
#include <vector>

namespace rtr {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ uint8_t status_char(uint32_t ss)
{
    const uint32_t c = ss & SS_CODE;
    return c == SS_N ? ST_N : (c == SS_S ? ST_S : ST_Y);
}

// Seeding pass over the forward edges (Decomposition.h:378-405) and the
// construction of the clean-time edge records.
__global__ void k_seed(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                       const int32_t* __restrict__ deg, const int32_t* __restrict__ fwd, int64_t m, double eps,
                       const double* __restrict__ pe, const uint32_t* __restrict__ sup,
                       const int64_t* __restrict__ tl_off, EdgeRec* __restrict__ rec, uint32_t* __restrict__ is_seed,
                       unsigned* __restrict__ err)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        const int64_t du = deg[esrc[i]], dv = deg[nb[i]];
        const double thr = eps * (1 / (double)(du * dv));
        const double p = pe[i];
        const uint32_t s = sup[i];
        if (s > SS_SUP) atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
        uint32_t code = SS_Y, seed = 0;
        if (p < thr) {
            if (s > 0) {
                code = SS_S;
                seed = 1;
            } else {
                code = SS_N;  // a pop with no triangle changes nothing but its own status
            }
        }
        EdgeRec r;
        r.pe = p;
        r.thr = thr;
        r.t0 = tl_off[i];
        r.cnt = (uint32_t)(tl_off[i + 1] - r.t0);
        r.ss = (s & SS_SUP) | code;
        rec[k] = r;
        is_seed[k] = seed;
    }
}

// Write the records back into the slot-indexed arrays the other stages use.
__global__ void k_clean_finish(const int32_t* __restrict__ fwd, int64_t m, const EdgeRec* __restrict__ rec,
                               double* __restrict__ pe, uint32_t* __restrict__ sup, uint8_t* __restrict__ st)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        const EdgeRec r = rec[k];
        pe[i] = r.pe;
        sup[i] = r.ss & SS_SUP;
        st[i] = status_char(r.ss);
    }
}

__device__ __forceinline__ int32_t uf_find(int32_t* p, int32_t x)
{
    while (true) {
        const int32_t px = p[x];
        if (px == x) return x;
        const int32_t ppx = p[px];
        if (ppx != px) atomicCAS(&p[x], px, ppx);
        x = px;
    }
}

__device__ __forceinline__ void uf_unite(int32_t* p, int32_t a, int32_t b)
{
    while (true) {
        a = uf_find(p, a);
        b = uf_find(p, b);
        if (a == b) return;
        if (a > b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        // hook the larger root under the smaller: the final root is the minimum id
        const int32_t old = atomicCAS(&p[b], b, a);
        if (old == b) return;
        b = old;
    }
}

__global__ void k_uf_init(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = (int32_t)v;
}

__global__ void k_uf_hook_support(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                                  const int32_t* __restrict__ fwd, int64_t m, const uint32_t* __restrict__ sup,
                                  int32_t* __restrict__ p)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (sup[i] > 0) uf_unite(p, esrc[i], nb[i]);
    }
}

__global__ void k_uf_flatten(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = uf_find(p, (int32_t)v);
}

// Per-unit capacity of the cascade stack (the unit's triangle-carrying edges)
// and the total length of their triangle lists.
__global__ void k_unit_edges(const int32_t* __restrict__ esrc, const int32_t* __restrict__ fwd, int64_t m,
                             const uint32_t* __restrict__ sup, const int32_t* __restrict__ root,
                             uint32_t* __restrict__ ecount, unsigned long long* __restrict__ tsum)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (sup[i] > 0) {
            const int32_t r = root[esrc[i]];
            atomicAdd(&ecount[r], 1u);
            atomicAdd(&tsum[r], (unsigned long long)sup[i]);
        }
    }
}

// Seed key = (unit root, forward rank): sorting groups seeds by unit and keeps
// slot order inside a unit (forward ranks ascend with slots).
__global__ void k_seed_keys(const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                            const uint32_t* __restrict__ is_seed, const uint32_t* __restrict__ pos, int64_t m,
                            const int32_t* __restrict__ root, int rbits, uint64_t* __restrict__ keys)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        if (is_seed[k]) keys[pos[k]] = ((uint64_t)root[esrc[fwd[k]]] << rbits) | (uint64_t)k;
}

__global__ void k_unit_heads(const uint64_t* __restrict__ keys, int64_t ns, int rbits, uint32_t* __restrict__ head)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x)
        head[j] = (j == 0 || (keys[j] >> rbits) != (keys[j - 1] >> rbits)) ? 1u : 0u;
}

__global__ void k_unit_desc(const uint64_t* __restrict__ keys, int64_t ns, int rbits,
                            const uint32_t* __restrict__ head, const uint32_t* __restrict__ hpos,
                            const uint32_t* __restrict__ ecount, UnitDesc* __restrict__ units,
                            int64_t* __restrict__ cap)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
        if (!head[j]) continue;
        const uint32_t u = hpos[j];
        units[u].seed_begin = j;
        units[u].root = (int64_t)(keys[j] >> rbits);
        cap[u] = ecount[(uint32_t)(keys[j] >> rbits)];
    }
}

// Unit bounds and the schedule: the units replayed in parallel rounds (many
// seeds, short lists: those are where disjoint pops are common) first, then
// the others; within each group the units with the most seeds first.
__global__ void k_unit_finish(UnitDesc* __restrict__ units, const int64_t* __restrict__ cap,
                              const int64_t* __restrict__ capoff, int64_t nu, int64_t ns,
                              const uint32_t* __restrict__ ecount, const unsigned long long* __restrict__ tsum,
                              int64_t round_min, double round_max_list, uint64_t* __restrict__ order_keys,
                              unsigned* __restrict__ nbig, int64_t stack_limit)
{
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < nu; u += (int64_t)gridDim.x * blockDim.x) {
        units[u].seed_end = (u + 1 < nu) ? units[u + 1].seed_begin : ns;
        units[u].stack_base = capoff[u];
        units[u].stack_cap = (stack_limit >= 0 && cap[u] > stack_limit) ? stack_limit : cap[u];
        const uint64_t work = (uint64_t)(units[u].seed_end - units[u].seed_begin);
        const int64_t r = units[u].root;
        const bool rounds = (int64_t)work >= round_min && (double)tsum[r] <= round_max_list * (double)ecount[r];
        if (rounds) atomicAdd(nbig, 1u);
        order_keys[u] = ((uint64_t)(rounds ? 0u : 1u) << 63) |
                        ((uint64_t)(0x7fffffffu - (uint32_t)(work < 0x7fffffffull ? work : 0x7fffffffull)) << 32) |
                        (uint64_t)u;
    }
}

// Seed descriptors, sorted seed j (unit-major, slot order within a unit).
__global__ void k_seed_info(const uint64_t* __restrict__ keys, int64_t ns, uint64_t rmask,
                            const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                            const int32_t* __restrict__ nb, const int32_t* __restrict__ deg,
                            const EdgeRec* __restrict__ rec, StackEntry* __restrict__ info)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = (int32_t)(keys[j] & rmask);
        const int64_t i = fwd[k];
        const int32_t u = esrc[i], v = nb[i];  // seeds are pushed as (u, v) with u < v
        info[j] = StackEntry{k, u, v, deg[u], deg[v], (int32_t)rec[k].cnt, rec[k].t0};
    }
}

struct CleanArgs {
    const TriEntry* tl;
    EdgeRec* rec;
    double* pv;
    double inv_n;
    const StackEntry* seeds;
    long wait_first;  // try_wait rounds of a window's first wait (kWaitLimit unless lowered to test the report)
    int64_t depth_limit;  // cascade-stack depth that counts as an overflow (-1: only the unit's region bounds it)
};

constexpr int kCleanBlock = 128;
constexpr int kCleanWarps = kCleanBlock / 32;
constexpr int kSmemStack = 256;  // newest stack entries of each warp live in shared memory

// Shared memory of one warp.
struct WarpSmem {
    StackEntry stack[kSmemStack];  // cascade stack, newest entries
    TriEntry went[32][32];         // first 32 triangles of each seed in the window
    StackEntry wseed[32];          // the window's seeds (lane k = k-th seed in pop order)
    double sw[32];                 // per-lane triangle weights of the current chunk
    uint64_t bar;                  // mbarrier completing the window's bulk copies
};

// Window staging by the TMA engine: one bulk global -> shared copy per seed
// (its first <= 32 entries, a contiguous run of 32-byte entries: source,
// destination and size are multiples of 16 bytes), all completing on the
// warp's mbarrier, which lane 0 arms with the window's byte total.  No
// multicast.  The wait is bounded.
__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(smem_u32(bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}

__device__ __forceinline__ void mbar_arm(uint64_t* bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void bulk_to_smem(void* dst, const void* src, unsigned bytes, uint64_t* bar)
{
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Non-blocking probe of the barrier phase (try_wait may suspend the thread for a
// while before it answers; test_wait answers at once).
__device__ __forceinline__ bool mbar_ready(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ bool mbar_done(uint64_t* bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

constexpr long kWaitLimit = 1l << 24;  // try_wait rounds before a wait is declared lost

// Per-warp cascade stack: the newest entries in shared memory, older ones
// spilled in order to the unit's global region (LIFO order is preserved).
struct WarpStack {
    StackEntry* sm;  // kSmemStack entries
    StackEntry* gm;  // unit's global region
    int64_t gtop;
    int64_t cap;
    int scount;
};

// 32 consecutive triangle-list entries of a pop (lane k holds entry base+k)
// with the records of their two other edges and their third vertex's weight.
struct Group {
    TriEntry t;
    EdgeRec r1, r2;  // (lower, z) and (higher, z)
    double pz;
    bool valid;
};

__device__ __forceinline__ void load_group(const CleanArgs& a, Group& g, bool lower_is_a)
{
    g.r1.ss = SS_N;
    g.r2.ss = SS_N;
    g.pz = 0.0;
    if (g.valid) {
        g.r1 = a.rec[lower_is_a ? g.t.raz : g.t.rbz];
        g.r2 = a.rec[lower_is_a ? g.t.rbz : g.t.raz];
        g.pz = a.pv[g.t.z];
    }
}

struct PopCtx {
    bool lower_is_a;
    int32_t lower, higher, dlow, dhigh;
    double acc_e, acc_u, acc_v;
    int removed;
};

// Remove the group's live triangles in list order: per-triangle cells in
// parallel, the popped edge and its endpoints folded in order, pushes appended
// in the reference's order.  False on stack overflow.
__device__ __forceinline__ bool apply_group(const CleanArgs& a, const Group& g, PopCtx& p, WarpStack& ws, double* sw,
                                            unsigned* err)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int32_t rlw = p.lower_is_a ? g.t.raz : g.t.rbz;
    const int32_t rhw = p.lower_is_a ? g.t.rbz : g.t.raz;
    const uint32_t c1 = g.r1.ss & SS_CODE, c2 = g.r2.ss & SS_CODE;
    const bool live = g.valid && c1 != SS_N && c2 != SS_N;
    const double wgt = live ? g.t.wgt : 0.0;
    bool p1 = false, p2 = false;
    if (live) {
        const double x1 = g.r1.pe - wgt;
        const double x2 = g.r2.pe - wgt;
        p1 = c1 != SS_S && x1 < g.r1.thr;
        p2 = c2 != SS_S && x2 < g.r2.thr;
        a.rec[rlw].pe = x1;
        a.rec[rhw].pe = x2;
        a.rec[rlw].ss = ((g.r1.ss & SS_SUP) - 1u) | (p1 ? SS_S : c1);
        a.rec[rhw].ss = ((g.r2.ss & SS_SUP) - 1u) | (p2 ? SS_S : c2);
        a.pv[g.t.z] = g.pz - wgt;
    }
    const unsigned lm = __ballot_sync(0xffffffffu, live);
    const unsigned b1 = __ballot_sync(0xffffffffu, p1);
    const unsigned b2 = __ballot_sync(0xffffffffu, p2);
    // live weights packed in lane (= triangle) order, so the fold below reads
    // fixed slots and only its floating-point chain is sequential
    if (live) sw[__popc(lm & lt)] = wgt;
    __syncwarp();
    // the popped edge and its endpoints accumulate in triangle order
    const int nl = __popc(lm);
#pragma unroll 4
    for (int k = 0; k < nl; ++k) {
        const double w = sw[k];
        p.acc_e -= w;
        p.acc_u -= w;
        p.acc_v -= w;
    }
    const int np = __popc(b1) + __popc(b2);
    if (np) {
        if (a.depth_limit >= 0 && ws.gtop + ws.scount + np > a.depth_limit) {  // a lowered bound (tests)
            if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_STACK_OVERFLOW);
            return false;
        }
        if (ws.scount + np > kSmemStack) {  // spill the shared part, oldest first
            if (ws.gtop + ws.scount > ws.cap) {
                if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_STACK_OVERFLOW);
                return false;
            }
            for (int k = lane; k < ws.scount; k += 32) ws.gm[ws.gtop + k] = ws.sm[k];
            ws.gtop += ws.scount;
            ws.scount = 0;
            __syncwarp();
        }
        const int before = ws.scount + __popc(b1 & lt) + __popc(b2 & lt);
        if (p1) ws.sm[before] = StackEntry{rlw, p.lower, g.t.z, p.dlow, g.t.dz, (int32_t)g.r1.cnt, g.r1.t0};
        if (p2)
            ws.sm[before + (p1 ? 1 : 0)] = StackEntry{rhw, p.higher, g.t.z, p.dhigh, g.t.dz, (int32_t)g.r2.cnt, g.r2.t0};
        ws.scount += np;
    }
    __syncwarp();
    p.removed += __popc(lm);
    return true;
}

__device__ __forceinline__ void pop_begin(const StackEntry& c, PopCtx& p)
{
    const int32_t u = c.first, v = c.second;
    const bool lo_is_u = c.dfirst < c.dsecond;
    p.lower = lo_is_u ? u : v;
    p.higher = lo_is_u ? v : u;
    p.dlow = lo_is_u ? c.dfirst : c.dsecond;
    p.dhigh = lo_is_u ? c.dsecond : c.dfirst;
    p.lower_is_a = p.lower == (u < v ? u : v);  // a = smaller endpoint of the forward edge
    p.removed = 0;
}

// The popped edge's own state, loaded by every lane from warp-uniform addresses
// (broadcast loads, no shuffles): the record's last word (list length |
// support word), its weight and its endpoints' weights.  Issued in the first
// round trip.
struct OwnState {
    unsigned long long w;  // cnt | ss << 32
    double pe, pu, pv;
};

__device__ __forceinline__ void pop_own_loads(const CleanArgs& a, const StackEntry& c, OwnState& o)
{
    const EdgeRec* r = a.rec + c.e;
    o.w = *reinterpret_cast<const unsigned long long*>(&r->cnt);
    o.pe = r->pe;
    o.pu = a.pv[c.first];
    o.pv = a.pv[c.second];
}

// False when the edge has no live triangle left (it is retired here).
__device__ __forceinline__ bool pop_own_state(const CleanArgs& a, const StackEntry& c, const OwnState& o,
                                              uint32_t& s_e, PopCtx& p, unsigned long long* diag)
{
    const int lane = threadIdx.x & 31;
    s_e = (uint32_t)(o.w >> 32) & SS_SUP;
    p.acc_e = o.pe;
    p.acc_u = o.pu;
    p.acc_v = o.pv;
    if (s_e == 0) {
        if (lane == 0) {
            if (fabs(p.acc_e) > a.inv_n) atomicAdd(&diag[0], 1ull);
            a.rec[c.e].ss = SS_N;
        }
        __syncwarp();
        return false;
    }
    return true;
}

__device__ __forceinline__ void pop_end(const CleanArgs& a, const StackEntry& c, uint32_t s_e, const PopCtx& p,
                                        unsigned long long* diag)
{
    // every lane holds the same values: the same stores from all lanes, no branch
    a.rec[c.e].pe = p.acc_e;
    a.rec[c.e].ss = (s_e - (uint32_t)p.removed) | SS_N;
    a.pv[c.first] = p.acc_u;
    a.pv[c.second] = p.acc_v;
    if ((threadIdx.x & 31) == 0 && fabs(p.acc_e) > a.inv_n) atomicAdd(&diag[0], 1ull);
    __syncwarp();
}

// Pop of an edge with at most 32 triangle-list entries: deleteAndClean's loop
// body (Decomposition.h:152-281) for the whole warp in two dependent round
// trips -- (1) the edge's record, its endpoints' weights and its entries (a
// window seed has them staged in shared memory, so its group's records come in
// this round trip too), then (2) the records of the two other edges of every
// triangle and the third vertex's weight.  Returns the number of triangles
// removed, or -1 on overflow.
__device__ __forceinline__ int pop_short(const CleanArgs& a, const StackEntry& c, const TriEntry* staged,
                                         WarpStack& ws, double* sw, unsigned* err, unsigned long long* diag)
{
    const int lane = threadIdx.x & 31;
    PopCtx p;
    pop_begin(c, p);
    uint32_t s_e;
    OwnState own;
    pop_own_loads(a, c, own);
    Group g;
    g.valid = lane < c.cnt;
    g.t = TriEntry{};
    if (g.valid) g.t = staged ? staged[lane] : ld_entry(a.tl + c.t0 + lane);
    if (staged) load_group(a, g, p.lower_is_a);
    if (!pop_own_state(a, c, own, s_e, p, diag)) return 0;
    if (!staged) load_group(a, g, p.lower_is_a);
    if (!apply_group(a, g, p, ws, sw, err)) return -1;
    pop_end(a, c, s_e, p, diag);
    return p.removed;
}

// Pop of an edge with a longer list.  Within a pop the liveness of every
// triangle is fixed (only the pop itself turns an edge 'N') and the
// per-triangle cells are distinct, so the list is taken 64 entries per window
// (two groups of 32): the window's records are loaded together, and the next
// window's entries (static data) are fetched while they are in flight.
__device__ __forceinline__ int pop_edge(const CleanArgs& a, const StackEntry& c, const TriEntry* staged, WarpStack& ws,
                                        double* sw, unsigned* err, unsigned long long* diag)
{
    const int lane = threadIdx.x & 31;
    PopCtx p;
    pop_begin(c, p);
    uint32_t s_e;
    OwnState own;
    pop_own_loads(a, c, own);
    Group g0, g1;
    g0.valid = lane < c.cnt;
    g1.valid = 32 + lane < c.cnt;
    g0.t = TriEntry{};
    g1.t = TriEntry{};
    if (g0.valid) g0.t = staged ? staged[lane] : ld_entry(a.tl + c.t0 + lane);
    if (g1.valid) g1.t = ld_entry(a.tl + c.t0 + 32 + lane);
    const bool seed_records = staged != nullptr;
    if (seed_records) load_group(a, g0, p.lower_is_a);
    if (!pop_own_state(a, c, own, s_e, p, diag)) return 0;
    TriEntry n0{}, n1{};
    for (int base = 0; base < c.cnt; base += 64) {
        if (base > 0) {
            g0.t = n0;
            g1.t = n1;
            g0.valid = base + lane < c.cnt;
            g1.valid = base + 32 + lane < c.cnt;
        }
        // next window's entries, fetched while this window's records load
        if (base + 64 + lane < c.cnt) n0 = ld_entry(a.tl + c.t0 + base + 64 + lane);
        if (base + 96 + lane < c.cnt) n1 = ld_entry(a.tl + c.t0 + base + 96 + lane);
        if (!(base == 0 && seed_records)) load_group(a, g0, p.lower_is_a);
        const bool second = base + 32 < c.cnt;
        if (second) load_group(a, g1, p.lower_is_a);
        if (!apply_group(a, g0, p, ws, sw, err)) return -1;
        if (second && !apply_group(a, g1, p, ws, sw, err)) return -1;
    }
    pop_end(a, c, s_e, p, diag);
    return p.removed;
}

__global__ void __launch_bounds__(kCleanBlock)
    k_clean_units(CleanArgs a, const UnitDesc* __restrict__ units, const uint64_t* __restrict__ order, int64_t first,
                  int64_t nu, StackEntry* __restrict__ stacks, unsigned* __restrict__ next_unit,
                  unsigned* __restrict__ err, unsigned long long* __restrict__ total,
                  unsigned long long* __restrict__ diag)
{
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem& sm = reinterpret_cast<WarpSmem*>(smem_raw)[wid];
    double* sw = sm.sw;
    if (lane == 0) mbar_init(&sm.bar);
    __syncwarp();
    unsigned bar_phase = 0;
    while (true) {
        unsigned ui = 0;
        if (lane == 0) ui = atomicAdd(next_unit, 1u);
        ui = __shfl_sync(0xffffffffu, ui, 0);
        if (first + (int64_t)ui >= nu) break;
        const UnitDesc ud = units[(uint32_t)order[first + ui]];
        WarpStack ws{sm.stack, stacks + ud.stack_base, 0, ud.stack_cap, 0};
        int64_t sp = ud.seed_end;  // seeds [seed_begin, sp) not yet loaded
        // Window of the next 32 seeds in pop order (lane k = seed sp_at_load-1-k).
        unsigned wmask = 0;
        StackEntry wseed{};
        unsigned long long removed = 0;
        while (true) {
            StackEntry cur;
            const TriEntry* staged = nullptr;
            if (ws.scount > 0) {
                cur = ws.sm[--ws.scount];
            } else if (ws.gtop > 0) {
                const int k = (int)(ws.gtop < kSmemStack ? ws.gtop : kSmemStack);
                for (int j = lane; j < k; j += 32) ws.sm[j] = ws.gm[ws.gtop - k + j];
                ws.gtop -= k;
                ws.scount = k;
                __syncwarp();
                cur = ws.sm[--ws.scount];
            } else {
                if (wmask == 0) {
                    if (sp <= ud.seed_begin) break;
                    const int64_t lo = (sp - 32 > ud.seed_begin) ? sp - 32 : ud.seed_begin;
                    const int wn = (int)(sp - lo);
                    bool live_seed = false;
                    if (lane < wn) {
                        wseed = a.seeds[sp - 1 - lane];
                        sm.wseed[lane] = wseed;
                        const EdgeRec r = a.rec[wseed.e];
                        // Support only decreases: a seed already at 0 is a no-op pop.
                        live_seed = (r.ss & SS_SUP) > 0;
                        if (!live_seed) {
                            if (fabs(r.pe) > a.inv_n) atomicAdd(&diag[0], 1ull);
                            a.rec[wseed.e].ss = SS_N;
                        }
                    }
                    wmask = __ballot_sync(0xffffffffu, live_seed);
                    sp = lo;
                    // stage the first 32 triangles of every live seed (static data):
                    // one bulk copy per seed, lane k copying seed k's run
                    const unsigned bytes = live_seed ? 32u * (unsigned)(wseed.cnt < 32 ? wseed.cnt : 32) : 0u;
                    const unsigned total = __reduce_add_sync(0xffffffffu, bytes);
                    if (total) {
                        // earlier generic reads of the staging area precede the async writes
                        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
                        if (lane == 0) mbar_arm(&sm.bar, total);
                        __syncwarp();
                        if (bytes) bulk_to_smem(&sm.went[lane][0], a.tl + wseed.t0, bytes, &sm.bar);
                        long it = 0;
                        if (a.wait_first < kWaitLimit) {  // a lowered bound (tests): probe without waiting
                            while (!mbar_ready(&sm.bar, bar_phase) && ++it < a.wait_first) {
                            }
                        } else {
                            while (!mbar_done(&sm.bar, bar_phase) && ++it < a.wait_first) {
                            }
                        }
                        if (it >= a.wait_first) {  // report, give the copies one more bounded wait, stop
                            if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_WAIT);
                            for (long j = 0; j < kWaitLimit && !mbar_done(&sm.bar, bar_phase); ++j) {
                            }
                            return;
                        }
                        bar_phase ^= 1u;
                    }
                    __syncwarp();
                    if (wmask == 0) continue;
                }
                const int k = __ffs(wmask) - 1;
                staged = sm.went[k];
                wmask &= wmask - 1;
                cur = sm.wseed[k];
            }
            __syncwarp();
            const int r = cur.cnt <= 32 ? pop_short(a, cur, staged, ws, sw, err, diag)
                                        : pop_edge(a, cur, staged, ws, sw, err, diag);
            if (r < 0) break;
            removed += (unsigned long long)r;
        }
        if (lane == 0 && removed) atomicAdd(total, (unsigned long long)(-(long long)removed));
    }
}

struct SideWait {
    cudaStream_t st = nullptr;
    ~SideWait()
    {
        if (st) cudaStreamSynchronize(st);
    }
};

}  // namespace

int initial_clean(rtr_graph* g, double eps)
{
    if (g->stage < 2) {
        set_error("clean called before count");
        return RTR_ERR_STATE;
    }
    if (!g->lists) {
        set_error("the graph was counted in the rows layout (its triangle lists did not fit in device memory, "
                  "or the count mode forbade them); the clean replays need the lists -- count again with "
                  "rtr_set_count_mode(g, 1, ...) on a device with room for them");
        return RTR_ERR_LIMIT;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m = g->m, m2 = g->m2;
    g->eps = eps;
    Scratch sc(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);

    uint32_t* is_seed = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    uint32_t* spos = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    uint32_t* stmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(m + 1));
    uint32_t* d_ns = (uint32_t*)sc.get(sizeof(uint32_t) * 2);
    int32_t* root = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    uint32_t* ecount = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    unsigned long long* tsum = (unsigned long long*)sc.get(sizeof(unsigned long long) * (n + 1));
    EdgeRec* rec = (EdgeRec*)sc.get(sizeof(EdgeRec) * (m + 1));
    if (!is_seed || !spos || !stmp || !d_ns || !root || !ecount || !tsum || !rec) {
        set_error("device allocation failed (clean)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr + 1, 0, 2 * sizeof(unsigned long long), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->st, ST_N, m2 + 16, s));  // backward slots are never read
    const int gm = grid_for(m, kBlock), gn = grid_for(n, kBlock);
    k_seed<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->deg, g->fwd, m, eps, g->pe, g->sup, g->tl_off, rec, is_seed,
                                 (unsigned*)(g->ctr + 1));
    k_uf_init<<<gn, kBlock, 0, s>>>(root, n);
    k_uf_hook_support<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->fwd, m, g->sup, root);
    k_uf_flatten<<<gn, kBlock, 0, s>>>(root, n);
    RTR_CUDA_TRY(cudaMemsetAsync(ecount, 0, sizeof(uint32_t) * (n + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(tsum, 0, sizeof(unsigned long long) * (n + 1), s));
    k_unit_edges<<<gm, kBlock, 0, s>>>(g->esrc, g->fwd, m, g->sup, root, ecount, tsum);
    exclusive_scan_u32(is_seed, spos, m, d_ns, stmp, s);
    g->launches += 8;
    RTR_CUDA_TRY(cudaGetLastError());
    uint32_t ns = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&ns, d_ns, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->kms[KT_CLEAN_UNITS] = 0;
    // an empty timer pair keeps the reading defined when no unit exists
    ktime_begin(g, KT_CLEAN_UNITS);
    ktime_end(g, KT_CLEAN_UNITS);

    if (ns > 0) {
        const int rbits = bits_for((uint64_t)m);
        const uint64_t rmask = (1ull << rbits) - 1;
        uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * (ns + 1));
        uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * (ns + 1));
        void* rtmp = sc.get(radix_temp_bytes(ns));
        uint32_t* head = (uint32_t*)sc.get(sizeof(uint32_t) * (ns + 1));
        uint32_t* hpos = (uint32_t*)sc.get(sizeof(uint32_t) * (ns + 1));
        uint32_t* htmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(ns + 1));
        StackEntry* seeds = (StackEntry*)sc.get(sizeof(StackEntry) * (ns + 1));
        if (!keys || !alt || !rtmp || !head || !hpos || !htmp || !seeds) {
            set_error("device allocation failed (clean seeds)");
            return RTR_ERR_CUDA;
        }
        k_seed_keys<<<gm, kBlock, 0, s>>>(g->fwd, g->esrc, is_seed, spos, m, root, rbits, keys);
        uint64_t* sorted = radix_sort_u64(keys, alt, ns, rbits + bits_for((uint64_t)n), rtmp, s);
        const int gs = grid_for(ns, kBlock);
        k_unit_heads<<<gs, kBlock, 0, s>>>(sorted, ns, rbits, head);
        exclusive_scan_u32(head, hpos, ns, d_ns + 1, htmp, s);
        k_seed_info<<<gs, kBlock, 0, s>>>(sorted, ns, rmask, g->fwd, g->esrc, g->nbors, g->deg, rec, seeds);
        g->launches += 4 + 3 * ((rbits + bits_for((uint64_t)n) + 7) / 8);
        uint32_t nu = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nu, d_ns + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        UnitDesc* units = (UnitDesc*)sc.get(sizeof(UnitDesc) * (nu + 1));
        int64_t* cap = (int64_t*)sc.get(sizeof(int64_t) * (nu + 1));
        int64_t* capoff = (int64_t*)sc.get(sizeof(int64_t) * (nu + 1));
        int64_t* ctmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nu + 1));
        int64_t* d_cap_total = (int64_t*)sc.get(sizeof(int64_t));
        uint64_t* okeys = (uint64_t*)sc.get(sizeof(uint64_t) * (nu + 1));
        uint64_t* oalt = (uint64_t*)sc.get(sizeof(uint64_t) * (nu + 1));
        void* otmp = sc.get(radix_temp_bytes(nu));
        unsigned* next_unit = (unsigned*)sc.get(sizeof(unsigned) * 4);
        if (!units || !cap || !capoff || !ctmp || !d_cap_total || !okeys || !oalt || !otmp || !next_unit) {
            set_error("device allocation failed (clean units)");
            return RTR_ERR_CUDA;
        }
        RTR_CUDA_TRY(cudaMemsetAsync(next_unit, 0, sizeof(unsigned) * 4, s));
        k_unit_desc<<<gs, kBlock, 0, s>>>(sorted, ns, rbits, head, hpos, ecount, units, cap);
        exclusive_scan_i64(cap, capoff, nu, d_cap_total, ctmp, s);
        k_unit_finish<<<grid_for(nu, kBlock), kBlock, 0, s>>>(units, cap, capoff, nu, ns, ecount, tsum,
                                                              g->clean_round_min, g->clean_round_list, okeys,
                                                              next_unit + 1, g->clean_stack_limit);
        uint64_t* order = radix_sort_u64(okeys, oalt, nu, 64, otmp, s);
        g->launches += 5 + 24;
        int64_t cap_total = 0;
        unsigned nbig = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&cap_total, d_cap_total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaMemcpyAsync(&nbig, next_unit + 1, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        StackEntry* stacks = (StackEntry*)sc.get(sizeof(StackEntry) * (cap_total + 1));
        if (!stacks) {
            set_error("device allocation failed (clean stacks)");
            return RTR_ERR_CUDA;
        }
        ktime_begin(g, KT_CLEAN_UNITS);
        // the largest units (order[0, nbig)) replay in parallel rounds on the
        // side stream while the others replay one warp per unit here
        RoundReplay rr;
        cudaEvent_t joined = nullptr;
        SideWait side_wait;  // an early return waits for the side stream before scratch is freed
        if (nbig > 0) {
            if (!g->side) RTR_CUDA_TRY(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
            side_wait.st = g->side;
            const int rc = clean_rounds_launch(g, sc, g->side, rec, seeds, units, order, nbig, stacks, &rr);
            if (rc) return rc;
            RTR_CUDA_TRY(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
            RTR_CUDA_TRY(cudaEventRecord(joined, g->side));
        }
        if ((int64_t)nbig < (int64_t)nu) {
            CleanArgs ca{g->tl, rec, g->pv, 1 / (double)n, seeds,
                         g->clean_wait_first > 0 ? (long)g->clean_wait_first : kWaitLimit, g->clean_stack_limit};
            // one warp per unit, persistent over the unit list (largest units first)
            const int64_t nsmall = (int64_t)nu - (int64_t)nbig;
            int blocks = (int)std::min<int64_t>((nsmall + kCleanWarps - 1) / kCleanWarps,
                                                (int64_t)grid_for(1 << 30, kCleanBlock, 8));
            blocks = std::max(blocks, 1);
            const size_t smem = sizeof(WarpSmem) * kCleanWarps;
            RTR_CUDA_TRY(cudaFuncSetAttribute(k_clean_units, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
            k_clean_units<<<blocks, kCleanBlock, smem, s>>>(ca, units, order, (int64_t)nbig, nu, stacks, next_unit,
                                                            (unsigned*)(g->ctr + 1), g->ctr, g->ctr + 2);
            g->launches += 1;
            RTR_CUDA_TRY(cudaGetLastError());
        }
        if (nbig > 0) {
            RTR_CUDA_TRY(cudaStreamWaitEvent(s, joined, 0));
            cudaEventDestroy(joined);
            const int rc = clean_rounds_finish(g, sc, &rr);
            if (rc) return rc;
        }
        ktime_end(g, KT_CLEAN_UNITS);
    }
    k_clean_finish<<<gm, kBlock, 0, s>>>(g->fwd, m, rec, g->pe, g->sup, g->st);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    cudaEventRecord(e1, s);
    RTR_CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&g->ms_clean, e0, e1);
    ktime_read(g, KT_CLEAN_UNITS);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    unsigned long long h[3];
    RTR_CUDA_TRY(cudaMemcpy(h, g->ctr, sizeof h, cudaMemcpyDeviceToHost));
    if (h[1] != 0) {
        set_error("device error word 0x%llx during the clean:%s%s%s%s%s", h[1],
                  (h[1] & DEV_ERR_STACK_OVERFLOW) ? " a unit's cascade stack overflowed its region;" : "",
                  (h[1] & DEV_ERR_BAD_STATUS) ? " an edge record held an impossible status;" : "",
                  (h[1] & DEV_ERR_SCRATCH) ? " a support count exceeded its field;" : "",
                  (h[1] & DEV_ERR_SORT) ? " a sort key left its range;" : "",
                  (h[1] & DEV_ERR_WAIT) ? " a bounded wait on an asynchronous copy ran out;" : "");
        return RTR_ERR_DEVICE;
    }
    g->diag_residual = (long long)h[2];
    g->stage = 3;
    return RTR_OK;
}

}  // namespace rtr
