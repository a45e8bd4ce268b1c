// Cluster extraction, order-faithful to disjointExtract's seed loop
// (RTRex_Sequential/Escape/Decomposition.h:566-919, populateStats :473-491).
//
// Seeds are visited in (degree, id) order (pairCompareSecond, Graph.cpp:40-45).
// Everything one seed does -- reading alive edges, the two-hop scan, writing
// triwgt / nbdBitMap / clustered, deleting the cluster's edges and the cascade
// that follows -- stays inside the seed's connected component of the current
// alive ('Y') graph, and the alive graph only shrinks.  So the components of
// the graph left by the initial clean are independent: each is replayed by one
// thread in the global seed order restricted to it, and performs the
// reference's floating-point operations in the reference's order.
//
// Per-component scratch mirrors the reference's containers:
//   std::unordered_set members  -> UsetOrder over (key, next, bucket) arrays
//   std::set two_hop            -> list + ascending sort
//   std::sort candidates        -> introsort restatement (stl_order.cuh)
//   std::stack deletion stack   -> array stack
// Cluster creation order is the global rank of each cluster's seed.
#include "primitives.cuh"
#include "rtr_graph.cuh"
#include "stl_order.cuh"

#include <algorithm>

namespace rtr {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int64_t fwd_slot(int32_t src, int64_t j, const int32_t* nb, const int32_t* partner)
{
    return (src < nb[j]) ? j : (int64_t)partner[j];
}

__device__ __forceinline__ int64_t find_slot(const int64_t* __restrict__ off, const int32_t* __restrict__ nb,
                                             int64_t v1, int32_t v2)
{
    int64_t lo = off[v1], hi = off[v1 + 1] - 1;
    while (lo <= hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int32_t x = nb[mid];
        if (x == v2) return mid;
        if (x > v2) hi = mid - 1;
        else lo = mid + 1;
    }
    return -1;
}

__global__ void k_iota_key_deg(const int32_t* __restrict__ deg, int64_t n, int B, uint64_t* __restrict__ keys)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)deg[v] << B) | (uint64_t)v;
}

__global__ void k_rank(const uint64_t* __restrict__ sorted, int64_t n, uint64_t mask, int32_t* __restrict__ rank,
                       int32_t* __restrict__ by_rank)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)(sorted[j] & mask);
        rank[v] = (int32_t)j;
        by_rank[j] = v;
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

__global__ void k_uf_init(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = (int32_t)v;
}

__global__ void k_uf_hook_alive(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                                const int32_t* __restrict__ fwd, int64_t m, const uint8_t* __restrict__ st,
                                int32_t* __restrict__ p)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (st[i] != ST_Y) continue;
        int32_t a = esrc[i], b = nb[i];
        while (true) {
            a = uf_find(p, a);
            b = uf_find(p, b);
            if (a == b) break;
            if (a > b) {
                const int32_t t = a;
                a = b;
                b = t;
            }
            const int32_t old = atomicCAS(&p[b], b, a);
            if (old == b) break;
            b = old;
        }
    }
}

__global__ void k_uf_flatten(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = uf_find(p, (int32_t)v);
}

__global__ void k_alive_count(const int32_t* __restrict__ esrc, const int32_t* __restrict__ fwd, int64_t m,
                              const uint8_t* __restrict__ st, const int32_t* __restrict__ root,
                              uint32_t* __restrict__ acount)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (st[i] == ST_Y) atomicAdd(&acount[root[esrc[i]]], 1u);
    }
}

__global__ void k_comp_keys(const int32_t* __restrict__ root, const int32_t* __restrict__ rank, int64_t n, int R,
                            uint64_t* __restrict__ keys)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)root[v] << R) | (uint64_t)rank[v];
}

__global__ void k_comp_heads(const uint64_t* __restrict__ keys, int64_t n, int R, const int32_t* __restrict__ by_rank,
                             uint32_t* __restrict__ head, int32_t* __restrict__ vlist)
{
    const uint64_t mask = (1ull << R) - 1;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        head[j] = (j == 0 || (keys[j] >> R) != (keys[j - 1] >> R)) ? 1u : 0u;
        vlist[j] = by_rank[keys[j] & mask];
    }
}

struct CompDesc {
    int64_t vbegin;   // into vlist / per-vertex scratch
    int64_t vcount;
    int64_t bbase;    // bucket scratch
    int64_t sbase;    // deletion-stack scratch
    int64_t scap;
};

__global__ void k_comp_begin(const uint64_t* __restrict__ keys, int64_t n, int R, const uint32_t* __restrict__ head,
                             const uint32_t* __restrict__ hpos, CompDesc* __restrict__ comps)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        if (head[j]) comps[hpos[j]].vbegin = j;
}

__global__ void k_comp_sizes(CompDesc* __restrict__ comps, int64_t nc, int64_t n, const uint64_t* __restrict__ keys,
                             int R, const uint32_t* __restrict__ acount, int64_t* __restrict__ bneed,
                             int64_t* __restrict__ sneed)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = comps[c].vbegin;
        const int64_t e = (c + 1 < nc) ? comps[c + 1].vbegin : n;
        comps[c].vcount = e - b;
        bneed[c] = (e - b > 1) ? uset_buckets_after(e - b) + 1 : 0;
        sneed[c] = acount[(uint32_t)(keys[b] >> R)];
    }
}

__global__ void k_comp_finish(CompDesc* __restrict__ comps, int64_t nc, const int64_t* __restrict__ boff,
                              const int64_t* __restrict__ soff, const int64_t* __restrict__ sneed,
                              uint64_t* __restrict__ order_keys, int64_t big_thr)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        comps[c].bbase = boff[c];
        comps[c].sbase = soff[c];
        comps[c].scap = sneed[c];
        // components for the block kernel (at least big_thr vertices) first, then
        // the others; largest first within each group
        const int64_t wr = comps[c].vcount + sneed[c];
        const uint64_t w = (uint64_t)(wr < 0x7fffffffll ? wr : 0x7fffffffll);
        const uint64_t small = comps[c].vcount >= big_thr ? 0u : 1u;
        order_keys[c] = (small << 63) | ((uint64_t)(0x7fffffffu - (uint32_t)w) << 32) | (uint64_t)c;
    }
}

struct Cand {
    int32_t vertex;
    int32_t pad;
    double wgt;
};

// A deletion-stack entry: the edge, the endpoint it was pushed from, the other
// endpoint, and its triangle list (offset, length), so that a pop's first
// entries are loaded together with its records.
struct DelEntry {
    int32_t e, first, second, cnt;
    int64_t t0;
};

struct ExtractArgs {
    const int32_t* vbase;  // per-vertex id base of its graph in a batch (null: a single graph)
    const int64_t* off;
    const int32_t* nb;
    const int32_t* esrc;
    const int32_t* partner;
    const int32_t* deg;
    const int64_t* tl_off;
    const TriEntry* tl;
    double* pe;
    double* pv;
    uint32_t* sup;
    uint8_t* st;
    double eps;
    double inv_n;
    const int32_t* vlist;
    uint8_t* clustered;
    uint8_t* nbd;
    uint8_t* in2hop;
    double* triwgt;
    int32_t* ukey;
    int32_t* unext;
    int32_t* ubucket;
    int32_t* twohop;
    Cand* cand;
    DelEntry* dstack;
    int32_t* hdr_seed;
    int64_t* hdr_start;
    int32_t* hdr_size;
    int32_t* out_vert;
    int32_t* ncl;
    unsigned* err;
    unsigned long long* total;
    unsigned long long* diag;
};

// deleteAndClean (Decomposition.h:147-283) after a cluster is cut out, for the
// whole warp (all lanes call it with the same arguments): a popped edge's
// triangle list is taken 32 entries at a time.
// Within one pop a triangle's liveness is fixed and its two other edges and
// third vertex are distinct from every other triangle's, so the lanes update
// those cells in parallel; the popped edge's weight and its endpoints' weights
// are folded in list order and pushes are appended in list order ((lower, z)
// before (higher, z)), as the sequential loop does.
__device__ void delete_and_clean_warp(const ExtractArgs& a, DelEntry* stack, int64_t top, int64_t cap, double* sw)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    long long removed = 0;
    while (top > 0) {
        __syncwarp();  // pushes and stores of the previous pop are visible
        const DelEntry d = stack[--top];
        const int32_t e = d.e, u = d.first, v = d.second;
        // the first 32 entries, issued with the edge's own records
        TriEntry t_first{};
        if (lane < d.cnt) t_first = a.tl[d.t0 + lane];
        const uint32_t s_e = a.sup[e];
        if (s_e == 0) {
            if (lane == 0) {
                if (fabs(a.pe[e]) > a.inv_n) atomicAdd(&a.diag[0], 1ull);
                a.st[e] = ST_N;
            }
            continue;
        }
        const int64_t du = a.deg[u], dv = a.deg[v];
        const bool lo_is_u = du < dv;
        const int32_t lower = lo_is_u ? u : v;
        const int32_t higher = lo_is_u ? v : u;
        const int64_t dlow = lo_is_u ? du : dv;
        const int64_t dhigh = lo_is_u ? dv : du;
        const bool lower_is_a = lower == a.esrc[e];
        double acc_e = a.pe[e], acc_u = a.pv[u], acc_v = a.pv[v];
        uint32_t rem = 0;
        const int64_t p1end = d.t0 + d.cnt;
        bool overflow = false;
        for (int64_t pb = d.t0; pb < p1end; pb += 32) {
            const int64_t p = pb + lane;
            const bool valid = p < p1end;
            TriEntry t{};
            if (pb == d.t0) t = t_first;
            else if (valid) t = a.tl[p];
            const int32_t elw = lower_is_a ? t.eaz : t.ebz;
            const int32_t ehw = lower_is_a ? t.ebz : t.eaz;
            // statuses, weights and supports of the triangle's other cells in one
            // round trip (the weights are only used when the triangle is live)
            uint8_t slw = ST_N, shw = ST_N;
            double pel = 0.0, peh = 0.0, pz = 0.0;
            uint32_t sul = 0, suh = 0;
            int64_t tlw0 = 0, tlw1 = 0, thw0 = 0, thw1 = 0;  // their lists, for a push
            if (valid) {
                slw = a.st[elw];
                shw = a.st[ehw];
                pel = a.pe[elw];
                peh = a.pe[ehw];
                pz = a.pv[t.z];
                sul = a.sup[elw];
                suh = a.sup[ehw];
                tlw0 = a.tl_off[elw];
                tlw1 = a.tl_off[elw + 1];
                thw0 = a.tl_off[ehw];
                thw1 = a.tl_off[ehw + 1];
            }
            const bool live = valid && slw != ST_N && shw != ST_N;
            const double wgt = live ? t.wgt : 0.0;
            bool q1 = false, q2 = false;
            if (live) {
                const double x1 = pel - wgt;
                const double x2 = peh - wgt;
                a.pe[elw] = x1;
                a.pe[ehw] = x2;
                a.pv[t.z] = pz - wgt;
                a.sup[elw] = sul - 1u;
                a.sup[ehw] = suh - 1u;
                q1 = slw != ST_S && x1 < a.eps * (1 / (double)(dlow * (int64_t)t.dz));
                q2 = shw != ST_S && x2 < a.eps * (1 / (double)(dhigh * (int64_t)t.dz));
            }
            const unsigned lm = __ballot_sync(0xffffffffu, live);
            const unsigned b1 = __ballot_sync(0xffffffffu, q1);
            const unsigned b2 = __ballot_sync(0xffffffffu, q2);
            // live weights packed in list order; the fold reads fixed slots
            if (live) sw[__popc(lm & lt)] = wgt;
            __syncwarp();
            const int nl = __popc(lm);
#pragma unroll 4
            for (int k = 0; k < nl; ++k) {
                const double w = sw[k];
                acc_e -= w;
                acc_u -= w;
                acc_v -= w;
            }
            const int np = __popc(b1) + __popc(b2);
            if (top + np > cap) {
                if (lane == 0) atomicOr(a.err, (unsigned)DEV_ERR_STACK_OVERFLOW);
                overflow = true;
                break;
            }
            const int64_t before = top + __popc(b1 & lt) + __popc(b2 & lt);
            if (q1) {
                stack[before] = DelEntry{elw, lower, t.z, (int32_t)(tlw1 - tlw0), tlw0};
                a.st[elw] = ST_S;
            }
            if (q2) {
                stack[before + (q1 ? 1 : 0)] = DelEntry{ehw, higher, t.z, (int32_t)(thw1 - thw0), thw0};
                a.st[ehw] = ST_S;
            }
            top += np;
            rem += (uint32_t)__popc(lm);
            __syncwarp();
        }
        if (overflow) return;
        // every lane holds the same values: the same stores from all lanes, no branch
        a.pe[e] = acc_e;
        a.pv[u] = acc_u;
        a.pv[v] = acc_v;
        a.sup[e] = s_e - rem;
        a.st[e] = ST_N;
        if (lane == 0 && fabs(acc_e) > a.inv_n) atomicAdd(&a.diag[0], 1ull);
        removed += rem;
    }
    __syncwarp();
    if (lane == 0 && removed) atomicAdd(a.total, (unsigned long long)(-removed));
}

// Ascending sort of distinct vertex ids (the std::set iteration order).
__device__ void sort_ids(int32_t* x, int64_t n)
{
    if (n < 2) return;
    // heapsort: O(n log n), no extra memory
    auto sift = [&](int64_t start, int64_t end) {
        int64_t root = start;
        while (2 * root + 1 <= end) {
            int64_t child = 2 * root + 1;
            if (child + 1 <= end && x[child] < x[child + 1]) ++child;
            if (x[root] < x[child]) {
                const int32_t t = x[root];
                x[root] = x[child];
                x[child] = t;
                root = child;
            } else {
                return;
            }
        }
    };
    for (int64_t s = (n - 2) / 2; s >= 0; --s) sift(s, n - 1);
    for (int64_t end = n - 1; end > 0; --end) {
        const int32_t t = x[0];
        x[0] = x[end];
        x[end] = t;
        sift(0, end - 1);
    }
}

// Per-component state of the seed loop: the scratch regions of the component
// and lane 0's containers (the member set, the output cursor, the cluster count).
struct CompCtx {
    int64_t vb, nv;
    int32_t base;  // graph-local id offset in a batch (the member set hashes local ids)
    int32_t* ukey;
    int32_t* unext;
    int32_t* ubucket;
    int32_t* twohop;
    Cand* cand;
    DelEntry* dstack;
    int64_t scap;
    int64_t out;   // lane 0
    int32_t ncl;   // lane 0
    UsetOrder S;   // lane 0
};

__device__ __forceinline__ CompCtx comp_ctx(const ExtractArgs& a, const CompDesc& cd)
{
    CompCtx cc;
    cc.vb = cd.vbegin;
    cc.nv = cd.vcount;
    cc.base = a.vbase ? a.vbase[a.vlist[cd.vbegin]] : 0;
    cc.ukey = a.ukey + cd.vbegin;
    cc.unext = a.unext + cd.vbegin;
    cc.ubucket = a.ubucket + cd.bbase;
    cc.twohop = a.twohop + cd.vbegin;
    cc.cand = a.cand + cd.vbegin;
    cc.dstack = a.dstack + cd.sbase;
    cc.scap = cd.scap;
    cc.out = cd.vbegin;
    cc.ncl = 0;
    return cc;
}

// Lane 0: the seed's cluster starts as {u} plus its alive neighbours, in row
// order (Decomposition.h:587-620), each marked clustered and in nbdBitMap.
__device__ __forceinline__ void seed_members(const ExtractArgs& a, CompCtx& cc, int32_t u)
{
    cc.S.init(cc.ukey, cc.unext, cc.ubucket);
    cc.S.insert(u - cc.base);
    a.clustered[u] = 1;
    for (int64_t j = a.off[u]; j < a.off[u + 1]; ++j) {
        if (a.st[fwd_slot(u, j, a.nb, a.partner)] == ST_N) continue;
        const int32_t v = a.nb[j];
        cc.S.insert(v - cc.base);
        a.nbd[v] = 1;
        a.clustered[v] = 1;
    }
}

// The two-hop scan of seed u (Decomposition.h:728-805) by one warp: for each
// pair (v, w) of the seed's alive neighbours of degree <= du/eps (w from v on,
// w == v included), the rows of the lower-degree one are taken 32 candidates x
// at a time: within one pair every x is distinct, so each lane updates its own
// triwgt[x] / in2hop[x], and the one shared sum (internal) is folded in lane
// order, i.e. in the reference's order, identically on every lane.
__device__ void two_hop_warp(const ExtractArgs& a, CompCtx& cc, int32_t u, double* sw, double* internal_out,
                             int64_t* n2_out)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t du = a.deg[u];
    const int64_t r0 = a.off[u], r1 = a.off[u + 1];
    double internal = 0;  // the same value on every lane
    int64_t n2 = 0;       // likewise
    const double thr = (double)du / a.eps;
    for (int64_t j = r0; j < r1; ++j) {
        if (a.st[fwd_slot(u, j, a.nb, a.partner)] == ST_N) continue;
        const int32_t v = a.nb[j];
        const int64_t dv = a.deg[v];
        if ((double)dv > thr) continue;
        for (int64_t k = j; k < r1; ++k) {  // k starts at j: w == v included
            if (a.st[fwd_slot(u, k, a.nb, a.partner)] == ST_N) continue;
            const int32_t w = a.nb[k];
            const int64_t dw = a.deg[w];
            if ((double)dw > thr) continue;
            internal += 1.0 / (double)(du * dv * dw);
            const int32_t lower = (dv < dw) ? v : w;
            const int32_t higher = (dv < dw) ? w : v;
            const int64_t l1 = a.off[lower + 1];
            for (int64_t lb = a.off[lower]; lb < l1; lb += 32) {
                const int64_t l = lb + lane;
                bool ok = false, in_nbd = false;
                int32_t x = 0;
                double wgt = 0.0;
                if (l < l1 && a.st[fwd_slot(lower, l, a.nb, a.partner)] != ST_N) {
                    x = a.nb[l];
                    if (x != lower && x != higher && x != u) {
                        const int64_t lh = find_slot(a.off, a.nb, higher, x);
                        if (lh >= 0 && a.st[fwd_slot(higher, lh, a.nb, a.partner)] != ST_N) {
                            ok = true;
                            wgt = 1.0 / (double)((int64_t)a.deg[x] * dv * dw);
                            in_nbd = a.nbd[x] != 0;
                        }
                    }
                }
                // candidates inside the neighbourhood feed internal, in order
                const bool inner = ok && in_nbd && x > v && x > w;
                const unsigned im = __ballot_sync(0xffffffffu, inner);
                if (im) {
                    if (inner) sw[__popc(im & lt)] = wgt;
                    __syncwarp();
                    const int ni = __popc(im);
                    for (int q = 0; q < ni; ++q) internal += sw[q];
                }
                // the others are two-hop candidates: distinct x, one lane each
                bool fresh = false;
                if (ok && !in_nbd) {
                    fresh = !a.in2hop[x];
                    if (fresh) a.in2hop[x] = 1;
                    a.triwgt[x] += wgt;
                }
                const unsigned fm = __ballot_sync(0xffffffffu, fresh);
                if (fresh) cc.twohop[n2 + __popc(fm & lt)] = x;
                n2 += __popc(fm);
                __syncwarp();  // the next chunk or pair may touch the same x from another lane
            }
        }
    }
    *internal_out = internal;
    *n2_out = n2;
}

// Lane 0: rank the two-hop candidates (std::set order, then the reference's
// unstable sort by weight, Decomposition.h:811-829), take the best prefix by
// the ratio (:847-864), clear the neighbour bits, and write the cluster out.
// Returns nonzero when the clusters would not partition the component.
__device__ int seed_select(const ExtractArgs& a, CompCtx& cc, int32_t u, double internal, int64_t n2,
                           int32_t* ncl_members)
{
    sort_ids(cc.twohop, n2);
    double potential = 0;
    for (int64_t k = 0; k < n2; ++k) {
        const int32_t x = cc.twohop[k];
        cc.cand[k].vertex = x;
        cc.cand[k].pad = 0;
        cc.cand[k].wgt = a.triwgt[x];
        potential += a.triwgt[x];
        a.triwgt[x] = 0;
        a.in2hop[x] = 0;
    }
    introsort(cc.cand, cc.cand + n2, [](const Cand& p, const Cand& q) { return p.wgt > q.wgt; });
    double ratio = internal / (internal + potential);
    int64_t maxind = -1;
    double num = 0, den = 0;
    for (int64_t k = 0; k < n2; ++k) {
        num += cc.cand[k].wgt;
        den += a.pv[cc.cand[k].vertex];
        const double nr = (internal + num) / (internal + potential + den);
        if (nr > ratio) {
            ratio = nr;
            maxind = k;
        }
    }
    for (int64_t k = 0; k <= maxind; ++k) {
        cc.S.insert(cc.cand[k].vertex - cc.base);
        a.clustered[cc.cand[k].vertex] = 1;
    }
    // The reference clears the bit of every neighbour of u (Decomposition.h:879-883).
    // Only the alive ones were set, and a dead neighbour may belong to another
    // component that a different thread is processing right now, so clear
    // exactly the bits this seed set.
    for (int64_t j = a.off[u]; j < a.off[u + 1]; ++j)
        if (a.st[fwd_slot(u, j, a.nb, a.partner)] != ST_N) a.nbd[a.nb[j]] = 0;
    if (cc.out + cc.S.size > cc.vb + cc.nv || cc.ncl >= cc.nv) {  // clusters must partition the component
        atomicOr(a.err, (unsigned)DEV_ERR_SCRATCH);
        return 1;
    }
    a.hdr_seed[cc.vb + cc.ncl] = u;
    a.hdr_start[cc.vb + cc.ncl] = cc.out;
    a.hdr_size[cc.vb + cc.ncl] = cc.S.size;
    *ncl_members = cc.S.size;
    for (int32_t p = cc.S.head; p != -1; p = cc.S.next[p]) a.out_vert[cc.out++] = cc.S.key[p] + cc.base;
    ++cc.ncl;
    return 0;
}

// The whole warp: the deletion stack -- every still-'Y' edge of the cluster's
// members, members in set-iteration order (the list lane 0 just wrote to
// out_vert, nm entries ending at out_end) and each member's row in order, 32
// row entries at a time; an edge between two members is pushed from the first
// member's row only ('S' afterwards) -- then the cascade that follows.
__device__ void seed_delete(const ExtractArgs& a, CompCtx& cc, int32_t nm, int64_t out_end, double* sw)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t mbase = out_end - nm;
    int64_t top = 0;
    bool full = false;
    for (int32_t q = 0; q < nm && !full; ++q) {
        const int32_t z = a.out_vert[mbase + q];
        const int64_t j1 = a.off[z + 1];
        for (int64_t jb = a.off[z]; jb < j1; jb += 32) {
            const int64_t j = jb + lane;
            int64_t f = -1;
            bool push = false;
            if (j < j1) {
                f = fwd_slot(z, j, a.nb, a.partner);
                push = a.st[f] == ST_Y;
            }
            const unsigned pm = __ballot_sync(0xffffffffu, push);
            const int np = __popc(pm);
            if (top + np > cc.scap) {
                if (lane == 0) atomicOr(a.err, (unsigned)DEV_ERR_STACK_OVERFLOW);
                full = true;  // stop scanning; the cascade still runs on what was pushed
                break;
            }
            if (push) {
                const int64_t t0 = a.tl_off[f];
                cc.dstack[top + __popc(pm & lt)] = DelEntry{(int32_t)f, z, a.nb[j], (int32_t)(a.tl_off[f + 1] - t0), t0};
                a.st[f] = ST_S;
            }
            top += np;
            __syncwarp();
        }
    }
    __syncwarp();
    delete_and_clean_warp(a, cc.dstack, top, cc.scap, sw);
}

// A component of one vertex: a singleton cluster with no edges to delete.
__device__ __forceinline__ void singleton_component(const ExtractArgs& a, const CompDesc& cd, int64_t c)
{
    const int32_t u = a.vlist[cd.vbegin];
    a.clustered[u] = 1;
    a.hdr_seed[cd.vbegin] = u;
    a.hdr_start[cd.vbegin] = cd.vbegin;
    a.hdr_size[cd.vbegin] = 1;
    a.out_vert[cd.vbegin] = u;
    a.ncl[c] = 1;
}

constexpr int kExtractBlock = 128;

__global__ void __launch_bounds__(kExtractBlock) k_extract_components(ExtractArgs a, const CompDesc* __restrict__ comps,
                                                            const uint64_t* __restrict__ order, int64_t nc,
                                                            unsigned* __restrict__ next_comp)
{
    // One warp per component.  Lane 0 replays the seed loop's sequential parts
    // (the member set, the candidate ranking, the deletion cascade's
    // bookkeeping); the two-hop scan and the deletion stack are taken 32 at a
    // time by the whole warp.  (Giving each thread its own component would put
    // the largest components, which are handed out first, into the same warp
    // and serialise them.)
    const int lane = threadIdx.x & 31;
    __shared__ double s_fold[kExtractBlock / 32][32];
    double* sw = s_fold[threadIdx.x >> 5];
    while (true) {
        unsigned ci = 0;
        if (lane == 0) ci = atomicAdd(next_comp, 1u);
        ci = __shfl_sync(0xffffffffu, ci, 0);
        if ((int64_t)ci >= nc) return;
        const int64_t c = (int64_t)(uint32_t)order[ci];
        const CompDesc cd = comps[c];
        if (cd.vcount == 1) {
            if (lane == 0) singleton_component(a, cd, c);
            continue;
        }
        CompCtx cc = comp_ctx(a, cd);
        for (int64_t idx = 0; idx < cc.nv; ++idx) {
            __syncwarp();  // lane 0's writes of the previous seed are visible
            const int32_t u = a.vlist[cc.vb + idx];
            if (a.clustered[u]) continue;
            if (lane == 0) seed_members(a, cc, u);
            __syncwarp();
            double internal = 0;
            int64_t n2 = 0;
            two_hop_warp(a, cc, u, sw, &internal, &n2);
            int fail = 0;
            int32_t nm = 0;
            if (lane == 0) fail = seed_select(a, cc, u, internal, n2, &nm);
            __syncwarp();
            if (__shfl_sync(0xffffffffu, fail, 0)) break;
            seed_delete(a, cc, __shfl_sync(0xffffffffu, nm, 0), __shfl_sync(0xffffffffu, cc.out, 0), sw);
        }
        if (lane == 0) a.ncl[c] = cc.ncl;
    }
}

// Large components, one thread block each.  The seed loop is the warp kernel's
// (warp 0 runs it), except for the two-hop scan: the block's other warps work
// out, seven pairs (v, w) ahead, each pair's candidates x in row order -- alive,
// in both rows, not u/v/w -- with their weights and whether x is in the
// neighbourhood, into per-warp buffers; warp 0 then applies the pairs in the
// reference's order: internal += 1/(du dv dw), internal += the in-neighbourhood
// candidates' weights (x > v, w) in row order, triwgt[x] += weight for the
// others (distinct x within a pair: one lane each).  Double-buffered: warp 0
// applies round r while the producers fill round r+1, one block barrier per
// round.  Every floating-point operation is the warp kernel's, in its order.
constexpr int kBigWarps = 8;
constexpr int kBigBlock = 32 * kBigWarps;

struct PairHit {
    int32_t x;
    int32_t inner;  // 1: in the neighbourhood and x > v, w (feeds internal); 2: in it, not counted; 0: two-hop
    double w;
};

__global__ void __launch_bounds__(kBigBlock) k_extract_big(ExtractArgs a, const CompDesc* __restrict__ comps,
                                                            const uint64_t* __restrict__ order, int64_t nbig,
                                                            unsigned* __restrict__ next_big, int32_t* __restrict__ fbuf,
                                                            PairHit* __restrict__ hbuf, int64_t hcap)
{
    constexpr int P = kBigWarps - 1;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    __shared__ double s_fold[kBigWarps][32];
    __shared__ int64_t s_cnt[2][P];
    __shared__ int64_t s_pv[2][P], s_pw[2][P];  // the pair's (dv, dw)
    __shared__ unsigned s_ci;
    __shared__ int64_t s_nf;
    __shared__ int s_fail;
    double* sw = s_fold[wib];
    int32_t* flist = fbuf + (int64_t)blockIdx.x * hcap;  // the seed's alive neighbours of degree <= du/eps
    auto hits = [&](int set, int w) { return hbuf + (((int64_t)blockIdx.x * 2 + set) * P + w) * hcap; };
    while (true) {
        if (threadIdx.x == 0) s_ci = atomicAdd(next_big, 1u);
        __syncthreads();
        const unsigned ci = s_ci;
        __syncthreads();
        if ((int64_t)ci >= nbig) return;
        const int64_t c = (int64_t)(uint32_t)order[ci];
        const CompDesc cd = comps[c];
        CompCtx cc = comp_ctx(a, cd);
        for (int64_t idx = 0; idx < cc.nv; ++idx) {
            const int32_t u = a.vlist[cc.vb + idx];
            __syncthreads();  // warp 0's writes of the previous seed are visible
            if (a.clustered[u]) continue;  // uniform: every thread reads it after the barrier
            const int64_t du = a.deg[u];
            const double thr = (double)du / a.eps;
            if (wib == 0) {
                if (lane == 0) seed_members(a, cc, u);
                __syncwarp();
                // the pair list's vertices: alive neighbours within the degree bound, row order
                int64_t nf = 0;
                const int64_t r1 = a.off[u + 1];
                for (int64_t jb = a.off[u]; jb < r1; jb += 32) {
                    const int64_t j = jb + lane;
                    bool keep = false;
                    int32_t v = 0;
                    if (j < r1 && a.st[fwd_slot(u, j, a.nb, a.partner)] != ST_N) {
                        v = a.nb[j];
                        keep = !((double)a.deg[v] > thr);
                    }
                    const unsigned km = __ballot_sync(0xffffffffu, keep);
                    if (keep) flist[nf + __popc(km & lt)] = v;
                    nf += __popc(km);
                }
                if (lane == 0) s_nf = nf;
            }
            __syncthreads();
            const int64_t nf = s_nf;
            const int64_t npairs = nf * (nf + 1) / 2;
            const int64_t rounds = (npairs + P - 1) / P;
            // producer warp w (1..P): pair number p, in (j, k >= j) order, into set
            auto produce = [&](int64_t p, int set) {
                const int w = wib - 1;
                int64_t cnt = 0, dvv = 0, dww = 0;
                if (p < npairs) {
                    // row j holds pairs (j, j..nf-1): find j with p in [S(j), S(j+1)), S(j) = j*nf - j(j-1)/2
                    int64_t lo = 0, hi = nf - 1;
                    while (lo < hi) {
                        const int64_t mid = (lo + hi + 1) >> 1;
                        if (mid * nf - mid * (mid - 1) / 2 <= p) lo = mid;
                        else hi = mid - 1;
                    }
                    const int64_t j = lo, k = j + (p - (j * nf - j * (j - 1) / 2));
                    const int32_t v = flist[j];
                    const int32_t x2 = flist[k];
                    dvv = a.deg[v];
                    dww = a.deg[x2];
                    const int32_t lower = (dvv < dww) ? v : x2;
                    const int32_t higher = (dvv < dww) ? x2 : v;
                    PairHit* out = hits(set, w);
                    const int64_t l1 = a.off[lower + 1];
                    for (int64_t lb = a.off[lower]; lb < l1; lb += 32) {
                        const int64_t l = lb + lane;
                        bool ok = false;
                        PairHit hh{0, 0, 0.0};
                        if (l < l1 && a.st[fwd_slot(lower, l, a.nb, a.partner)] != ST_N) {
                            const int32_t x = a.nb[l];
                            if (x != lower && x != higher && x != u) {
                                const int64_t lh = find_slot(a.off, a.nb, higher, x);
                                if (lh >= 0 && a.st[fwd_slot(higher, lh, a.nb, a.partner)] != ST_N) {
                                    ok = true;
                                    const bool in_nbd = a.nbd[x] != 0;
                                    hh.x = x;
                                    hh.w = 1.0 / (double)((int64_t)a.deg[x] * dvv * dww);
                                    hh.inner = in_nbd ? ((x > v && x > x2) ? 1 : 2) : 0;
                                }
                            }
                        }
                        const unsigned om = __ballot_sync(0xffffffffu, ok);
                        if (ok) out[cnt + __popc(om & lt)] = hh;
                        cnt += __popc(om);
                    }
                }
                if (lane == 0) {
                    s_cnt[set][w] = cnt;
                    s_pv[set][w] = dvv;
                    s_pw[set][w] = dww;
                }
            };
            double internal = 0;  // warp 0, the same on every lane
            int64_t n2 = 0;
            if (wib > 0) produce(wib - 1, 0);
            __syncthreads();
            for (int64_t r = 0; r < rounds; ++r) {
                const int set = (int)(r & 1);
                if (wib == 0) {
                    for (int w = 0; w < P && r * P + w < npairs; ++w) {
                        internal += 1.0 / (double)(du * s_pv[set][w] * s_pw[set][w]);
                        const PairHit* in = hits(set, w);
                        const int64_t cnt = s_cnt[set][w];
                        for (int64_t b = 0; b < cnt; b += 32) {
                            const bool valid = b + lane < cnt;
                            PairHit hh{0, 2, 0.0};
                            if (valid) hh = in[b + lane];
                            const bool inner = valid && hh.inner == 1;
                            const unsigned im = __ballot_sync(0xffffffffu, inner);
                            if (im) {
                                if (inner) sw[__popc(im & lt)] = hh.w;
                                __syncwarp();
                                const int ni = __popc(im);
                                for (int q = 0; q < ni; ++q) internal += sw[q];
                            }
                            bool fresh = false;
                            if (valid && hh.inner == 0) {
                                fresh = !a.in2hop[hh.x];
                                if (fresh) a.in2hop[hh.x] = 1;
                                a.triwgt[hh.x] += hh.w;
                            }
                            const unsigned fm = __ballot_sync(0xffffffffu, fresh);
                            if (fresh) cc.twohop[n2 + __popc(fm & lt)] = hh.x;
                            n2 += __popc(fm);
                            __syncwarp();
                        }
                    }
                } else if (r + 1 < rounds) {
                    produce((r + 1) * P + wib - 1, set ^ 1);
                }
                __syncthreads();
            }
            if (wib == 0) {
                int fail = 0;
                int32_t nm = 0;
                if (lane == 0) fail = seed_select(a, cc, u, internal, n2, &nm);
                __syncwarp();
                fail = __shfl_sync(0xffffffffu, fail, 0);
                if (!fail) seed_delete(a, cc, __shfl_sync(0xffffffffu, nm, 0), __shfl_sync(0xffffffffu, cc.out, 0), sw);
                if (lane == 0) s_fail = fail;
            }
            __syncthreads();
            if (s_fail) break;
        }
        if (threadIdx.x == 0) a.ncl[c] = cc.ncl;
    }
}

__global__ void k_cluster_keys(const CompDesc* __restrict__ comps, int64_t nc, const int32_t* __restrict__ ncl,
                               const int64_t* __restrict__ cpos, const int32_t* __restrict__ hdr_seed,
                               const int32_t* __restrict__ rank, int B, uint64_t* __restrict__ keys)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t vb = comps[c].vbegin;
        for (int32_t k = 0; k < ncl[c]; ++k)
            keys[cpos[c] + k] = ((uint64_t)rank[hdr_seed[vb + k]] << B) | (uint64_t)(vb + k);
    }
}

__global__ void k_cluster_gather(const uint64_t* __restrict__ sorted, int64_t ncl, uint64_t mask,
                                 const int32_t* __restrict__ hdr_seed, const int32_t* __restrict__ hdr_size,
                                 int32_t* __restrict__ cl_seed, int64_t* __restrict__ size64)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ncl; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t h = (int64_t)(sorted[g] & mask);
        cl_seed[g] = hdr_seed[h];
        size64[g] = hdr_size[h];
    }
}

__global__ void k_cluster_members(const uint64_t* __restrict__ sorted, int64_t ncl, uint64_t mask,
                                  const int64_t* __restrict__ hdr_start, const int64_t* __restrict__ cl_off,
                                  const int32_t* __restrict__ out_vert, int32_t* __restrict__ cl_vert,
                                  int32_t* __restrict__ cluster_of)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ncl; g += (int64_t)gridDim.x * blockDim.x) {
        const int64_t h = (int64_t)(sorted[g] & mask);
        const int64_t src = hdr_start[h];
        for (int64_t p = cl_off[g]; p < cl_off[g + 1]; ++p) {
            const int32_t v = out_vert[src + (p - cl_off[g])];
            cl_vert[p] = v;
            cluster_of[v] = (int32_t)g;
        }
    }
}

// populateStats over the original adjacency (integer counts, order-free).
__global__ void k_cluster_stats(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, int64_t n,
                                const int32_t* __restrict__ cluster_of, unsigned long long* __restrict__ ne,
                                unsigned long long* __restrict__ cut)
{
    for (int64_t z = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; z < n; z += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cluster_of[z];
        unsigned long long in = 0, outc = 0;
        for (int64_t j = off[z]; j < off[z + 1]; ++j) {
            if (cluster_of[nb[j]] == c) ++in;
            else ++outc;
        }
        if (in) atomicAdd(&ne[c], in);
        if (outc) atomicAdd(&cut[c], outc);
    }
}

__global__ void k_widen(const int32_t* __restrict__ in, int64_t* __restrict__ out, int64_t k)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

// Components of at least `thr` vertices (the block kernel's) and the largest vertex count among them.
__global__ void k_big_count(const CompDesc* __restrict__ comps, int64_t nc, int64_t thr, unsigned* __restrict__ nbig,
                            unsigned long long* __restrict__ maxv)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < nc; c += (int64_t)gridDim.x * blockDim.x)
        if (comps[c].vcount >= thr) {
            atomicAdd(nbig, 1u);
            atomicMax(maxv, (unsigned long long)comps[c].vcount);
        }
}

__global__ void k_halve(int64_t* __restrict__ ne, int64_t ncl)
{
    for (int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; g < ncl; g += (int64_t)gridDim.x * blockDim.x)
        ne[g] /= 2;
}

// The side stream joined back into the main stream (explicitly, or on an early
// return, before the scratch the side kernel uses is freed).
struct SideJoin {
    cudaStream_t side = nullptr, main = nullptr;
    void join()
    {
        if (!side) return;
        cudaEvent_t done;
        if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) == cudaSuccess) {
            cudaEventRecord(done, side);
            cudaStreamWaitEvent(main, done, 0);
            cudaEventDestroy(done);
        } else {
            cudaStreamSynchronize(side);
        }
        side = nullptr;
    }
    ~SideJoin()
    {
        if (side) cudaStreamSynchronize(side);
    }
};

}  // namespace

int extract_clusters(rtr_graph* g)
{
    if (g->stage < 3) {
        set_error("extract called before the clean");
        return RTR_ERR_STATE;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m = g->m, m2 = g->m2;
    g->expanded = false;
    Scratch sc(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr + 1, 0, 2 * sizeof(unsigned long long), s));

    const int B = bits_for((uint64_t)(n - 1));
    const uint64_t bmask = (1ull << B) - 1;
    const int gn = grid_for(n, kBlock), gm = grid_for(m, kBlock);

    // global seed order: (degree, id)
    uint64_t* k1 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    uint64_t* k2 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    void* rtmp = sc.get(radix_temp_bytes(n));
    int32_t* rank = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    int32_t* by_rank = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    int32_t* root = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    uint32_t* acount = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* head = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* hpos = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* htmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(n + 1));
    uint32_t* d_nc = (uint32_t*)sc.get(sizeof(uint32_t) * 2);
    int32_t* vlist = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    if (!k1 || !k2 || !rtmp || !rank || !by_rank || !root || !acount || !head || !hpos || !htmp || !d_nc || !vlist) {
        set_error("device allocation failed (extract setup)");
        return RTR_ERR_CUDA;
    }
    k_iota_key_deg<<<gn, kBlock, 0, s>>>(g->deg, n, B, k1);
    uint64_t* sorted = radix_sort_u64(k1, k2, n, B + bits_for((uint64_t)m2), rtmp, s);
    k_rank<<<gn, kBlock, 0, s>>>(sorted, n, bmask, rank, by_rank);
    // components of the alive graph
    k_uf_init<<<gn, kBlock, 0, s>>>(root, n);
    k_uf_hook_alive<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->fwd, m, g->st, root);
    k_uf_flatten<<<gn, kBlock, 0, s>>>(root, n);
    RTR_CUDA_TRY(cudaMemsetAsync(acount, 0, sizeof(uint32_t) * (n + 1), s));
    k_alive_count<<<gm, kBlock, 0, s>>>(g->esrc, g->fwd, m, g->st, root, acount);
    k_comp_keys<<<gn, kBlock, 0, s>>>(root, rank, n, B, k1 == sorted ? k2 : k1);
    uint64_t* ck = (k1 == sorted) ? k2 : k1;
    uint64_t* calt = sorted;  // rank/by_rank already captured; reuse as ping-pong
    uint64_t* csorted = radix_sort_u64(ck, calt, n, 2 * B, rtmp, s);
    k_comp_heads<<<gn, kBlock, 0, s>>>(csorted, n, B, by_rank, head, vlist);
    exclusive_scan_u32(head, hpos, n, d_nc, htmp, s);
    g->launches += 12 + 3 * ((B + bits_for((uint64_t)m2) + 7) / 8) + 3 * ((2 * B + 7) / 8);
    RTR_CUDA_TRY(cudaGetLastError());
    uint32_t nc = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nc, d_nc, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));

    CompDesc* comps = (CompDesc*)sc.get(sizeof(CompDesc) * (nc + 1));
    int64_t* bneed = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    int64_t* sneed = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    int64_t* boff = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    int64_t* soff = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    int64_t* ltmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nc + 1));
    int64_t* d_tot = (int64_t*)sc.get(sizeof(int64_t) * 2);
    uint64_t* okeys = (uint64_t*)sc.get(sizeof(uint64_t) * (nc + 1));
    uint64_t* oalt = (uint64_t*)sc.get(sizeof(uint64_t) * (nc + 1));
    void* otmp = sc.get(radix_temp_bytes(nc));
    if (!comps || !bneed || !sneed || !boff || !soff || !ltmp || !d_tot || !okeys || !oalt || !otmp) {
        set_error("device allocation failed (extract components)");
        return RTR_ERR_CUDA;
    }
    k_comp_begin<<<gn, kBlock, 0, s>>>(csorted, n, B, head, hpos, comps);
    const int gc = grid_for(nc, kBlock);
    k_comp_sizes<<<gc, kBlock, 0, s>>>(comps, nc, n, csorted, B, acount, bneed, sneed);
    exclusive_scan_i64(bneed, boff, nc, d_tot, ltmp, s);
    exclusive_scan_i64(sneed, soff, nc, d_tot + 1, ltmp, s);
    k_comp_finish<<<gc, kBlock, 0, s>>>(comps, nc, boff, soff, sneed, okeys, g->extract_big);
    uint64_t* order = radix_sort_u64(okeys, oalt, nc, 64, otmp, s);
    g->launches += 9 + 24;
    int64_t tots[2] = {0, 0};
    RTR_CUDA_TRY(cudaMemcpyAsync(tots, d_tot, sizeof tots, cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));

    ExtractArgs a;
    a.vbase = g->vbase;
    a.off = g->offsets;
    a.nb = g->nbors;
    a.esrc = g->esrc;
    a.partner = g->partner;
    a.deg = g->deg;
    a.tl_off = g->tl_off;
    a.tl = g->tl;
    a.pe = g->pe;
    a.pv = g->pv;
    a.sup = g->sup;
    a.st = g->st;
    a.eps = g->eps;
    a.inv_n = 1 / (double)n;
    a.vlist = vlist;
    a.clustered = (uint8_t*)sc.get(n + 16);
    a.nbd = (uint8_t*)sc.get(n + 16);
    a.in2hop = (uint8_t*)sc.get(n + 16);
    a.triwgt = (double*)sc.get(sizeof(double) * (n + 1));
    a.ukey = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.unext = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.ubucket = (int32_t*)sc.get(sizeof(int32_t) * (tots[0] + 1));
    a.twohop = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.cand = (Cand*)sc.get(sizeof(Cand) * (n + 1));
    a.dstack = (DelEntry*)sc.get(sizeof(DelEntry) * (tots[1] + 1));
    a.hdr_seed = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.hdr_start = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    a.hdr_size = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.out_vert = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    a.ncl = (int32_t*)sc.get(sizeof(int32_t) * (nc + 1));
    a.err = (unsigned*)(g->ctr + 1);
    a.total = g->ctr;
    a.diag = g->ctr + 2;
    unsigned* next_comp = (unsigned*)sc.get(sizeof(unsigned) * 2);
    if (!a.clustered || !a.nbd || !a.in2hop || !a.triwgt || !a.ukey || !a.unext || !a.ubucket || !a.twohop ||
        !a.cand || !a.dstack || !a.hdr_seed || !a.hdr_start || !a.hdr_size || !a.out_vert || !a.ncl || !next_comp) {
        set_error("device allocation failed (extract scratch)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(a.clustered, 0, n + 16, s));
    RTR_CUDA_TRY(cudaMemsetAsync(a.nbd, 0, n + 16, s));
    RTR_CUDA_TRY(cudaMemsetAsync(a.in2hop, 0, n + 16, s));
    RTR_CUDA_TRY(cudaMemsetAsync(a.triwgt, 0, sizeof(double) * (n + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(next_comp, 0, sizeof(unsigned) * 2, s));
    // components of at least extract_big vertices: a thread block each, on the
    // side stream, while the others take a warp each here
    unsigned* d_big = (unsigned*)sc.get(sizeof(unsigned) * 2);
    unsigned long long* d_maxv = (unsigned long long*)sc.get(sizeof(unsigned long long));
    if (!d_big || !d_maxv) {
        set_error("device allocation failed (extract split)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(d_big, 0, sizeof(unsigned) * 2, s));
    RTR_CUDA_TRY(cudaMemsetAsync(d_maxv, 0, sizeof(unsigned long long), s));
    k_big_count<<<gc, kBlock, 0, s>>>(comps, nc, g->extract_big, d_big, d_maxv);
    unsigned nbig = 0;
    unsigned long long maxv = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nbig, d_big, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(&maxv, d_maxv, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->launches += 1;
    SideJoin side_join;  // an early return waits for the side stream before scratch is freed
    if (nbig > 0) {
        const int64_t hcap = (int64_t)maxv + 32;
        int sms = 148;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
        const int64_t per_block = hcap * ((int64_t)sizeof(int32_t) + 2 * (kBigWarps - 1) * (int64_t)sizeof(PairHit));
        int64_t bgrid = std::min<int64_t>((int64_t)nbig, sms);
        bgrid = std::max<int64_t>(1, std::min<int64_t>(bgrid, (4ll << 30) / per_block));
        int32_t* fbuf = (int32_t*)sc.get(sizeof(int32_t) * (size_t)(bgrid * hcap));
        PairHit* hbuf = (PairHit*)sc.get(sizeof(PairHit) * (size_t)(bgrid * 2 * (kBigWarps - 1) * hcap));
        if (!fbuf || !hbuf) {
            set_error("device allocation failed (extract pair buffers)");
            return RTR_ERR_CUDA;
        }
        if (!g->side) RTR_CUDA_TRY(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
        cudaEvent_t ready;
        RTR_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        RTR_CUDA_TRY(cudaEventRecord(ready, s));
        RTR_CUDA_TRY(cudaStreamWaitEvent(g->side, ready, 0));
        cudaEventDestroy(ready);
        side_join.side = g->side;
        side_join.main = s;
        k_extract_big<<<(unsigned)bgrid, kBigBlock, 0, g->side>>>(a, comps, order, (int64_t)nbig, next_comp + 1,
                                                                   fbuf, hbuf, hcap);
        g->launches += 1;
    }
    {
        const int blk = kExtractBlock;
        const int64_t warps = (int64_t)nc - nbig;  // one component per warp
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((warps + 3) / 4, grid_for(1 << 30, blk, 16)));
        ktime_begin(g, KT_EXTRACT);
        if (warps > 0)
            k_extract_components<<<blocks, blk, 0, s>>>(a, comps, order + nbig, warps, next_comp);
        if (nbig > 0) side_join.join();
        ktime_end(g, KT_EXTRACT);
        g->launches += 1;
    }
    RTR_CUDA_TRY(cudaGetLastError());

    // clusters in creation order = ascending rank of their seeds
    int64_t* cpos = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    int64_t* ncl64 = (int64_t*)sc.get(sizeof(int64_t) * (nc + 1));
    if (!cpos || !ncl64) {
        set_error("device allocation failed (cluster order)");
        return RTR_ERR_CUDA;
    }
    k_widen<<<gc, kBlock, 0, s>>>(a.ncl, ncl64, nc);
    exclusive_scan_i64(ncl64, cpos, nc, d_tot, ltmp, s);
    int64_t ncl = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&ncl, d_tot, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    {
        unsigned long long h[3];
        RTR_CUDA_TRY(cudaMemcpy(h, g->ctr, sizeof h, cudaMemcpyDeviceToHost));
        if (h[1] != 0) {
            set_error("device error word 0x%llx during extraction", h[1]);
            return RTR_ERR_DEVICE;
        }
        g->diag_residual += (long long)h[2];
    }
    uint64_t* ckeys = (uint64_t*)sc.get(sizeof(uint64_t) * (ncl + 1));
    uint64_t* calt2 = (uint64_t*)sc.get(sizeof(uint64_t) * (ncl + 1));
    void* ctmp = sc.get(radix_temp_bytes(ncl));
    int64_t* size64 = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 1));
    if (!ckeys || !calt2 || !ctmp || !size64) {
        set_error("device allocation failed (cluster keys)");
        return RTR_ERR_CUDA;
    }
    if (!g->cl_seed || g->ncl < ncl) {
        g->cl_seed = (int32_t*)dev_alloc(g, sizeof(int32_t) * (ncl + 1));
        g->cl_off = (int64_t*)dev_alloc(g, sizeof(int64_t) * (ncl + 2));
        g->cl_ne = (int64_t*)dev_alloc(g, sizeof(int64_t) * (ncl + 1));
        g->cl_cut = (int64_t*)dev_alloc(g, sizeof(int64_t) * (ncl + 1));
    }
    if (!g->cl_vert) {
        g->cl_vert = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        g->cluster_of = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
    }
    if (!g->cl_seed || !g->cl_off || !g->cl_ne || !g->cl_cut || !g->cl_vert || !g->cluster_of) {
        set_error("device allocation failed (cluster outputs)");
        return RTR_ERR_CUDA;
    }
    g->ncl = ncl;
    RTR_CUDA_TRY(cudaMemsetAsync(size64, 0, sizeof(int64_t) * (ncl + 1), s));
    k_cluster_keys<<<gc, kBlock, 0, s>>>(comps, nc, a.ncl, cpos, a.hdr_seed, rank, B, ckeys);
    uint64_t* csort = radix_sort_u64(ckeys, calt2, ncl, 2 * B, ctmp, s);
    const int gk = grid_for(ncl, kBlock);
    k_cluster_gather<<<gk, kBlock, 0, s>>>(csort, ncl, bmask, a.hdr_seed, a.hdr_size, g->cl_seed, size64);
    exclusive_scan_i64(size64, g->cl_off, ncl + 1, nullptr, ltmp, s);
    {
        // the clusters must partition the vertex set
        int64_t members = -1;
        RTR_CUDA_TRY(cudaMemcpyAsync(&members, g->cl_off + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        if (members != n) {
            set_error("extraction produced %lld cluster members for %lld vertices", (long long)members, (long long)n);
            return RTR_ERR_DEVICE;
        }
    }
    k_cluster_members<<<gk, kBlock, 0, s>>>(csort, ncl, bmask, a.hdr_start, g->cl_off, a.out_vert, g->cl_vert,
                                            g->cluster_of);
    RTR_CUDA_TRY(cudaMemsetAsync(g->cl_ne, 0, sizeof(int64_t) * (ncl + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->cl_cut, 0, sizeof(int64_t) * (ncl + 1), s));
    k_cluster_stats<<<gn, kBlock, 0, s>>>(g->offsets, g->nbors, n, g->cluster_of,
                                          (unsigned long long*)g->cl_ne, (unsigned long long*)g->cl_cut);
    k_halve<<<gk, kBlock, 0, s>>>(g->cl_ne, ncl);
    g->launches += 8 + 3 * ((2 * B + 7) / 8);
    RTR_CUDA_TRY(cudaGetLastError());
    cudaEventRecord(e1, s);
    RTR_CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&g->ms_extract, e0, e1);
    ktime_read(g, KT_EXTRACT);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->stage = 4;
    return RTR_OK;
}

}  // namespace rtr
