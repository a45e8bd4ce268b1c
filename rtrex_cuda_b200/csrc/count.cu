// Weighted triangle counting, bit-exact to commonNbr
// (RTRex_Sequential/Escape/Decomposition.h:42-117).
//
// commonNbr finds every triangle once, in lexicographic order of its sorted
// vertex triple, and adds w = 1/double(du*dv*dw) to six directed-edge cells and
// three vertex cells.  Because of that discovery order:
//   perEdge[(x,y)]  = left fold, over common neighbours z of x and y in
//                     ascending z, of w(x,y,z)
//   perVertex[x]    = left fold over y in N(x) ascending, then over
//                     z in N(x) & N(y) with z > y ascending, of w(x,y,z)
// So each cell is produced by one thread as an ordered fold, with no
// floating-point atomics (the CUDA port's nine atomicAdd(double) per triangle,
// gpu_triangle_count.cu:70-88, give run-dependent bits).
//
// Kernels:
//   k_edge_fold    one thread per undirected edge: merge / galloping intersection
//                  of the two rows -> perEdge fold, live support, triangles with z>v
//   k_tri_fill     same intersection, writes the edge's triangle list
//                  {z, fwd(a,z), fwd(b,z), deg z} (used by the clean and for perVertex)
//   k_vertex_fold_light / _heavy  perVertex fold from the triangle lists: a thread
//                  per light vertex, a warp per heavy one
//   k_edge_count_heavy / k_tri_fill_heavy / k_pe_fold_heavy  the same for edges
//                  with deg u + deg v >= g->tune_edge, one warp per edge
// On large graphs (2m >= 2^25, or the rows layout forced) the rows of at least
// 256 entries get hash sets first (rowsets.cuh); an intersection whose longer
// row has one walks the shorter row against it (a warp per heavy edge four
// chunks of 32 per step, the heavy edges in the order of the sets they probe,
// so that the probed sets stay in L2).  The same pass also counts, for both
// slots of every edge, the common neighbours above the slot's neighbour (the
// rows layout's per-slot term counts, count_rows.cu), folds the heavy edges'
// perEdge in z order, and records each heavy edge's per-chunk hit masks for the
// rows layout's list fill.
// Three work-split parameters (g->tune_gallop: the row-length ratio above which
// an intersection gallops instead of merging; g->tune_heavy: the degree from
// which a vertex is folded by a warp; g->tune_edge: the degree sum from which an
// edge is intersected by a warp) change how work is spread, never a result; the
// autotuner (rtr_autotune) times candidates on the graph itself.
#include "intersect.cuh"
#include "primitives.cuh"
#include "rowsets.cuh"
#include "rtr_graph.cuh"

#include <memory>

namespace rtr {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ void block_add_u64(unsigned long long v, unsigned long long* dst)
{
    __shared__ unsigned long long s[kBlock / 32];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) s[w] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int k = 0; k < kBlock / 32; ++k) t += s[k];
        if (t) atomicAdd(dst, t);
    }
}

// cgt (may be null): for each directed slot (x,y), the number of common
// neighbours z > y -- the terms slot (x,y) adds to perVertex[x] -- written for
// both slots of every edge (the rows layout's list offsets).
__global__ void __launch_bounds__(kBlock)
    k_edge_fold(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ esrc,
                const int32_t* __restrict__ deg, const int32_t* __restrict__ fwd,
                const int32_t* __restrict__ partner, int64_t m, RowSets rs, double* __restrict__ pe,
                uint32_t* __restrict__ sup, int64_t* __restrict__ cnt, int64_t* __restrict__ cgt,
                unsigned long long* __restrict__ total, int gallop, int heavy_edge, int32_t* __restrict__ heavy_list,
                unsigned* __restrict__ nheavy)
{
    unsigned long long tri = 0;
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        const int32_t u = esrc[i], v = nb[i];
        if (deg[u] + deg[v] >= heavy_edge) {  // a warp takes it (k_edge_count_heavy)
            heavy_list[atomicAdd(nheavy, 1u)] = (int32_t)k;
            continue;
        }
        const int64_t duv = (int64_t)deg[u] * (int64_t)deg[v];
        double acc = 0.0;
        uint32_t c = 0, above = 0, above_u = 0;
        thread_common(rs, off, nb, u, v, INT32_MIN, gallop, [&](int32_t z) {
            acc += 1.0 / (double)(duv * (int64_t)deg[z]);
            ++c;
            above += (z > v) ? 1u : 0u;
            above_u += (z > u) ? 1u : 0u;
        });
        pe[i] = acc;
        sup[i] = c;
        cnt[i] = c;
        if (cgt) {
            cgt[i] = above;
            cgt[partner[i]] = above_u;
        }
        tri += above;
    }
    block_add_u64(tri, total);
}

__global__ void __launch_bounds__(kBlock)
    k_tri_fill(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ esrc,
               const int32_t* __restrict__ deg, const int32_t* __restrict__ partner, const int32_t* __restrict__ fwd,
               const int32_t* __restrict__ frank, int64_t m, const int64_t* __restrict__ tl_off,
               TriEntry* __restrict__ tl, int gallop, int heavy_edge)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        const int32_t u = esrc[i], v = nb[i];
        if (deg[u] + deg[v] >= heavy_edge) continue;  // k_tri_fill_heavy
        const int64_t duv = (int64_t)deg[u] * (int64_t)deg[v];
        int64_t w = tl_off[i];
        intersect_rows(nb, off[u], off[u + 1], off[v], off[v + 1], gallop, [&](int32_t z, int64_t pu, int64_t pv) {
            TriEntry t;
            t.z = z;
            t.eaz = (u < z) ? (int32_t)pu : partner[pu];
            t.ebz = (v < z) ? (int32_t)pv : partner[pv];
            t.dz = deg[z];
            t.wgt = 1.0 / (double)(duv * (int64_t)t.dz);
            t.raz = frank[t.eaz];
            t.rbz = frank[t.ebz];
            tl[w++] = t;
        });
    }
}

// Heavy edges (deg u + deg v >= heavy_edge), one warp each, dealt from the list
// the light edge fold built.  Counting is integer and order-free, so the lanes
// split the intersection (warp_intersect_part) and sum; the triangle list is
// written by the same split, each lane at its prefix offset, which keeps the
// entries in ascending z; perEdge is then folded from the list in that order
// (the same left fold over z ascending as the thread path).
constexpr int kHeavyEdgeBlock = 128;

// pe (may be null): also fold perEdge of the heavy edges, in ascending z, from
// an ordered walk of the shorter row (the lists layout folds them from the
// lists instead, k_pe_fold_heavy).  cgt as in k_edge_fold.
__global__ void __launch_bounds__(kHeavyEdgeBlock, 6)
    k_edge_count_heavy(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ esrc,
                       const int32_t* __restrict__ deg, const int32_t* __restrict__ fwd,
                       const int32_t* __restrict__ partner, const int32_t* __restrict__ heavy_list,
                       const unsigned* __restrict__ nheavy, int gallop, RowSets rs, uint32_t* __restrict__ sup,
                       int64_t* __restrict__ cnt, int64_t* __restrict__ cgt, double* __restrict__ pe,
                       unsigned long long* __restrict__ total, const int64_t* __restrict__ moff,
                       uint32_t* __restrict__ masks)
{
    __shared__ double s_w[kHeavyEdgeBlock / 32][32];
    __shared__ int32_t s_z[kHeavyEdgeBlock / 32][128];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t nh = *nheavy;
    const int64_t nwarps = (int64_t)gridDim.x * (kHeavyEdgeBlock / 32);
    unsigned long long tri = 0;
    for (int64_t h = (int64_t)blockIdx.x * (kHeavyEdgeBlock / 32) + wib; h < nh; h += nwarps) {
        const int64_t i = fwd[heavy_list[h]];
        const int32_t u = esrc[i], v = nb[i];
        const int64_t u0 = off[u], u1 = off[u + 1], v0 = off[v], v1 = off[v + 1];
        unsigned c = 0, above = 0, above_u = 0;
        // the shorter row walked against the longer one
        const bool u_short = u1 - u0 <= v1 - v0;
        const int32_t t = rs_table(rs, u_short ? v : u);
        const int64_t duv = (int64_t)deg[u] * (int64_t)deg[v];
        double acc = 0.0;
        if (t >= 0) {
            // 4 chunks per step, their lookups and then their degrees in flight together
            constexpr int B = 4;
            // perEdge: the step's hits, in order, are packed one per lane (ballot ranks), so that one
            // pass of divisions serves all four chunks, and enter the chain by shuffle
            const unsigned lt = (1u << lane) - 1u;
            // masks: each chunk's hit ballot, for the rows layout's list fill
            const int64_t mw0 = masks ? moff[h] : 0, mwn = masks ? moff[h + 1] - mw0 : 0;
            int64_t chunk = 0;
            warp_probe_walk<B>(rs, t, nb, u_short ? u0 : v0, u_short ? u1 : v1, nb[(u_short ? v1 : u1) - 1], lane,
                               [&](const bool (&hit)[B], const int32_t (&x)[B]) {
                                   int tot = 0;
#pragma unroll
                                   for (int b = 0; b < B; ++b) {
                                       c += hit[b] ? 1u : 0u;
                                       above += (hit[b] && x[b] > v) ? 1u : 0u;
                                       above_u += (hit[b] && x[b] > u) ? 1u : 0u;
                                       const unsigned mb = __ballot_sync(0xffffffffu, hit[b]);
                                       if (pe && hit[b]) s_z[wib][tot + __popc(mb & lt)] = x[b];
                                       if (lane == 0 && chunk + b < mwn) masks[mw0 + chunk + b] = mb;
                                       tot += __popc(mb);
                                   }
                                   chunk += B;
                                   if (!pe || tot == 0) return;
                                   __syncwarp();
                                   for (int q0 = 0; q0 < tot; q0 += 32) {
                                       const int j = q0 + lane;
                                       const double w =
                                           j < tot ? 1.0 / (double)(duv * (int64_t)deg[s_z[wib][j]]) : 0.0;
                                       const int cc = tot - q0 < 32 ? tot - q0 : 32;
#pragma unroll 4
                                       for (int k = 0; k < cc; ++k) acc += __shfl_sync(0xffffffffu, w, k);
                                   }
                                   __syncwarp();
                               });
            if (pe && lane == 0) pe[i] = acc;
        } else if (pe) {
            warp_walk(rs, off, nb, u_short ? u0 : v0, u_short ? u1 : v1, u_short ? v : u, u_short ? v0 : u0,
                      u_short ? v1 : u1, lane, [&](bool hit, int32_t z) {
                          c += hit ? 1u : 0u;
                          above += (hit && z > v) ? 1u : 0u;
                          above_u += (hit && z > u) ? 1u : 0u;
                          const double w = hit ? 1.0 / (double)(duv * (int64_t)deg[z]) : 0.0;
                          fold_hits(hit, w, s_w[wib], lane, &acc, nullptr, 0);
                      });
            if (lane == 0) pe[i] = acc;
        } else {
            warp_intersect_part(nb, u0, u1, v0, v1, gallop, lane, [&](int32_t z, int64_t, int64_t) {
                ++c;
                above += (z > v) ? 1u : 0u;
                above_u += (z > u) ? 1u : 0u;
            });
        }
        c = __reduce_add_sync(0xffffffffu, c);
        above = __reduce_add_sync(0xffffffffu, above);
        above_u = __reduce_add_sync(0xffffffffu, above_u);
        if (lane == 0) {
            sup[i] = c;
            cnt[i] = c;
            if (cgt) {
                cgt[i] = above;
                cgt[partner[i]] = above_u;
            }
            tri += above;
        }
    }
    if (lane == 0 && tri) atomicAdd(total, tri);
}

// Heavy edges keyed by the vertex whose hash set their intersection probes
// (the longer row; the shorter one is walked): sorted on it, the warps running
// at any one time probe a few sets, which then stay in L2.
__global__ void k_heavy_keys(const int64_t* __restrict__ off, const int32_t* __restrict__ esrc,
                             const int32_t* __restrict__ nb, const int32_t* __restrict__ fwd,
                             const int32_t* __restrict__ heavy_list, int64_t nh, uint64_t* __restrict__ keys)
{
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nh; h += (int64_t)gridDim.x * blockDim.x) {
        const int32_t k = heavy_list[h];
        const int64_t i = fwd[k];
        const int32_t u = esrc[i], v = nb[i];
        const int32_t w = off[u + 1] - off[u] <= off[v + 1] - off[v] ? v : u;
        keys[h] = ((uint64_t)(uint32_t)k << 32) | (uint64_t)(uint32_t)w;
    }
}

// Hit-mask words of each heavy edge: one per 32 elements of its shorter row
// when the longer row has a hash set (the edges the count walks through one),
// else none.
__global__ void k_mask_words(const int64_t* __restrict__ off, const int32_t* __restrict__ esrc,
                             const int32_t* __restrict__ nb, const int32_t* __restrict__ fwd,
                             const int32_t* __restrict__ heavy_list, int64_t nh, RowSets rs,
                             int64_t* __restrict__ words)
{
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h <= nh; h += (int64_t)gridDim.x * blockDim.x) {
        if (h == nh) {
            words[h] = 0;
            continue;
        }
        const int64_t i = fwd[heavy_list[h]];
        const int32_t u = esrc[i], v = nb[i];
        const int64_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
        const bool u_short = du <= dv;
        words[h] = rs_table(rs, u_short ? v : u) >= 0 ? ((u_short ? du : dv) + 31) / 32 : 0;
    }
}

__global__ void k_heavy_order(const uint64_t* __restrict__ keys, int64_t nh, int32_t* __restrict__ heavy_list)
{
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h < nh; h += (int64_t)gridDim.x * blockDim.x)
        heavy_list[h] = (int32_t)(keys[h] >> 32);
}

__global__ void __launch_bounds__(kHeavyEdgeBlock)
    k_tri_fill_heavy(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ esrc,
                     const int32_t* __restrict__ deg, const int32_t* __restrict__ partner,
                     const int32_t* __restrict__ fwd, const int32_t* __restrict__ frank,
                     const int32_t* __restrict__ heavy_list, const unsigned* __restrict__ nheavy, int gallop,
                     const int64_t* __restrict__ tl_off, TriEntry* __restrict__ tl)
{
    const int lane = threadIdx.x & 31;
    const int64_t nh = *nheavy;
    const int64_t nwarps = (int64_t)gridDim.x * (kHeavyEdgeBlock / 32);
    for (int64_t h = (int64_t)blockIdx.x * (kHeavyEdgeBlock / 32) + (threadIdx.x >> 5); h < nh; h += nwarps) {
        const int64_t i = fwd[heavy_list[h]];
        const int32_t u = esrc[i], v = nb[i];
        const int64_t duv = (int64_t)deg[u] * (int64_t)deg[v];
        unsigned c = 0;
        warp_intersect_part(nb, off[u], off[u + 1], off[v], off[v + 1], gallop, lane,
                            [&](int32_t, int64_t, int64_t) { ++c; });
        unsigned incl = c;  // inclusive prefix over lanes
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += y;
        }
        int64_t w = tl_off[i] + (int64_t)(incl - c);
        warp_intersect_part(nb, off[u], off[u + 1], off[v], off[v + 1], gallop, lane,
                            [&](int32_t z, int64_t pu, int64_t pv) {
                                TriEntry t;
                                t.z = z;
                                t.eaz = (u < z) ? (int32_t)pu : partner[pu];
                                t.ebz = (v < z) ? (int32_t)pv : partner[pv];
                                t.dz = deg[z];
                                t.wgt = 1.0 / (double)(duv * (int64_t)t.dz);
                                t.raz = frank[t.eaz];
                                t.rbz = frank[t.ebz];
                                tl[w++] = t;
                            });
    }
}

__global__ void __launch_bounds__(kHeavyEdgeBlock)
    k_pe_fold_heavy(const int32_t* __restrict__ fwd, const int32_t* __restrict__ heavy_list,
                    const unsigned* __restrict__ nheavy, const int64_t* __restrict__ tl_off,
                    const TriEntry* __restrict__ tl, double* __restrict__ pe)
{
    __shared__ double s_w[kHeavyEdgeBlock / 32][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t nh = *nheavy;
    const int64_t nwarps = (int64_t)gridDim.x * (kHeavyEdgeBlock / 32);
    for (int64_t h = (int64_t)blockIdx.x * (kHeavyEdgeBlock / 32) + wib; h < nh; h += nwarps) {
        const int64_t i = fwd[heavy_list[h]];
        const int64_t e0 = tl_off[i], e1 = tl_off[i + 1];
        double acc = 0.0;
        for (int64_t b = e0; b < e1; b += 32) {
            if (b + lane < e1) s_w[wib][lane] = tl[b + lane].wgt;
            __syncwarp();
            const int cnt = e1 - b < 32 ? (int)(e1 - b) : 32;
            for (int j = 0; j < cnt; ++j) acc += s_w[wib][j];
            __syncwarp();
        }
        if (lane == 0) pe[i] = acc;
    }
}

// Entries of edge c = fwd(x,y) with z > y: [first, tl_off[c+1]).
__device__ __forceinline__ int64_t first_above(const TriEntry* __restrict__ tl, int64_t lo, int64_t hi, int32_t y)
{
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (tl[mid].z <= y) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}


// perVertex[x] = left fold over y in N(x) ascending, then z > y ascending, of the
// triangle weights (Decomposition.h:95-101).
//
// k_vertex_fold_light: one thread per vertex of degree < heavy (at most
// heavy^2/2 entries each).
__global__ void __launch_bounds__(kBlock)
    k_vertex_fold_light(const int64_t* __restrict__ off, const int32_t* __restrict__ nb,
                        const int32_t* __restrict__ deg, const int32_t* __restrict__ partner, int64_t n,
                        const int64_t* __restrict__ tl_off, const TriEntry* __restrict__ tl, double* __restrict__ pv,
                        int heavy)
{
    for (int64_t x = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < n; x += (int64_t)gridDim.x * blockDim.x) {
        if (deg[x] >= heavy) continue;
        double acc = 0.0;
        for (int64_t i = off[x]; i < off[x + 1]; ++i) {
            const int32_t y = nb[i];
            const int64_t c = (x < y) ? i : (int64_t)partner[i];
            const int64_t hi = tl_off[c + 1];
            for (int64_t p = first_above(tl, tl_off[c], hi, y); p < hi; ++p) acc += tl[p].wgt;
        }
        pv[x] = acc;
    }
}

// k_vertex_fold_heavy: one warp per vertex of degree >= heavy, dealt by id
// modulo the warp count (power-law generators put hubs at neighbouring ids).
// Per 32 neighbours the lanes find their entry ranges at once; the ranges'
// entries are then loaded 32 at a time in fold order (each lane finds its range
// by a 5-step search over the range ends in shared memory), staged in shared
// memory, and added in order -- only the floating-point chain is sequential.
constexpr int kHeavyBlock = 128;
__global__ void __launch_bounds__(kHeavyBlock)
    k_vertex_fold_heavy(const int64_t* __restrict__ off, const int32_t* __restrict__ nb,
                        const int32_t* __restrict__ deg, const int32_t* __restrict__ partner, int64_t n,
                        const int64_t* __restrict__ tl_off, const TriEntry* __restrict__ tl, double* __restrict__ pv,
                        int heavy)
{
    __shared__ int64_t s_end[kHeavyBlock / 32][32];
    __shared__ int64_t s_beg[kHeavyBlock / 32][32];
    __shared__ double s_w[kHeavyBlock / 32][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * (kHeavyBlock / 32);
    for (int64_t hx = (int64_t)blockIdx.x * (kHeavyBlock / 32) + wib; hx < n; hx += nwarps) {
        if (deg[hx] < heavy) continue;  // uniform across the warp
        const int64_t h0 = off[hx], h1 = off[hx + 1];
        double acc = 0.0;
        for (int64_t cb = h0; cb < h1; cb += 32) {
            const int64_t i = cb + lane;
            int64_t a = 0, len = 0;
            if (i < h1) {
                const int32_t y = nb[i];
                const int64_t c = (hx < y) ? i : (int64_t)partner[i];
                const int64_t hi = tl_off[c + 1];
                a = first_above(tl, tl_off[c], hi, y);
                len = hi - a;
            }
            int64_t end = len;  // inclusive prefix of the range lengths
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t t = __shfl_up_sync(0xffffffffu, end, o);
                if (lane >= o) end += t;
            }
            s_end[wib][lane] = end;
            s_beg[wib][lane] = a - (end - len);  // entry index = s_beg[owner] + k
            __syncwarp();
            const int64_t total = s_end[wib][31];
            for (int64_t k0 = 0; k0 < total; k0 += 32) {
                const int64_t k = k0 + lane;
                if (k < total) {
                    int lo = 0, hi = 31;  // first lane whose range ends after k
                    while (lo < hi) {
                        const int mid = (lo + hi) >> 1;
                        if (s_end[wib][mid] <= k) lo = mid + 1;
                        else hi = mid;
                    }
                    s_w[wib][lane] = tl[s_beg[wib][lo] + k].wgt;
                }
                __syncwarp();
                const int cnt = total - k0 < 32 ? (int)(total - k0) : 32;
                for (int j = 0; j < cnt; ++j) acc += s_w[wib][j];
                __syncwarp();
            }
        }
        if (lane == 0) pv[hx] = acc;
    }
}

}  // namespace

int count_triangles(rtr_graph* g)
{
    if (g->stage < 1) {
        set_error("count called before the graph was built");
        return RTR_ERR_STATE;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m2 = g->m2, m = g->m;
    if (!g->pe) {
        g->pe = (double*)dev_alloc(g, sizeof(double) * (m2 + 1));
        g->pv = (double*)dev_alloc(g, sizeof(double) * (n + 1));
        g->sup = (uint32_t*)dev_alloc(g, sizeof(uint32_t) * (m2 + 1));
        g->st = (uint8_t*)dev_alloc(g, m2 + 16);
        g->tl_off = (int64_t*)dev_alloc(g, sizeof(int64_t) * (m2 + 1));
        if (!g->pe || !g->pv || !g->sup || !g->st || !g->tl_off) {
            set_error("device allocation failed for the triangle state");
            return RTR_ERR_CUDA;
        }
    }
    Scratch sc(g);
    int64_t* cnt = (int64_t*)sc.get(sizeof(int64_t) * (m2 + 1));
    int64_t* tmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(m2 + 1));
    int32_t* heavy_list = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    unsigned* nheavy = (unsigned*)sc.get(sizeof(unsigned) * 2);
    if (!cnt || !tmp || !heavy_list || !nheavy) {
        set_error("device allocation failed (count scratch)");
        return RTR_ERR_CUDA;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, 2 * sizeof(unsigned long long), s));
    RTR_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(int64_t) * (m2 + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->pe, 0, sizeof(double) * (m2 + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->sup, 0, sizeof(uint32_t) * (m2 + 1), s));
    const int ge = grid_for(m, kBlock);
    const int gh = grid_for(1ll << 40, kHeavyEdgeBlock, 16);
    RTR_CUDA_TRY(cudaMemsetAsync(nheavy, 0, sizeof(unsigned), s));
    ktime_begin(g, KT_EDGE_FOLD);
    // Hash sets of the long rows, for the heavy-edge count and the rows layout:
    // built when the rows layout is asked for, or may be chosen (2m >= 2^25).
    RowSets rs{nullptr, nullptr, nullptr, nullptr};
    if (g->count_mode == 2 || (g->count_mode == 0 && m2 >= (1ll << 25))) {
        const int rc = build_row_sets(g, sc, kSetDegree, &rs);
        if (rc) return rc;
    }
    // per-slot counts of perVertex terms, for the rows layout's lists
    int64_t* cgt = nullptr;
    if (g->count_mode != 1) {
        cgt = (int64_t*)sc.get(sizeof(int64_t) * (m2 + 1));
        if (!cgt) {
            set_error("device allocation failed (count scratch)");
            return RTR_ERR_CUDA;
        }
        RTR_CUDA_TRY(cudaMemsetAsync(cgt, 0, sizeof(int64_t) * (m2 + 1), s));
    }
    // heavy-edge perEdge folded by the count when the rows layout is likely
    const bool heavy_pe = g->count_mode == 2 || rs.tab != nullptr;
    ktime_begin(g, KT_EDGE_LIGHT);
    k_edge_fold<<<ge, kBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, g->deg, g->fwd, g->partner, m, rs, g->pe,
                                      g->sup, cnt, cgt, g->ctr, g->tune_gallop, g->tune_edge, heavy_list, nheavy);
    ktime_end(g, KT_EDGE_LIGHT);
    if (rs.tab) {  // heavy edges in the order of the sets they probe
        unsigned nh = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nh, nheavy, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        if (nh > 1) {
            uint64_t* hkeys = (uint64_t*)sc.get(sizeof(uint64_t) * (nh + 1));
            uint64_t* halt = (uint64_t*)sc.get(sizeof(uint64_t) * (nh + 1));
            void* htmp = sc.get(radix_temp_bytes(nh));
            if (!hkeys || !halt || !htmp) {
                set_error("device allocation failed (heavy-edge order)");
                return RTR_ERR_CUDA;
            }
            k_heavy_keys<<<grid_for(nh, 256), 256, 0, s>>>(g->offsets, g->esrc, g->nbors, g->fwd, heavy_list, nh,
                                                            hkeys);
            const uint64_t* sorted = radix_sort_u64(hkeys, halt, nh, bits_for((uint64_t)(n > 0 ? n - 1 : 0)),
                                                    htmp, s);
            k_heavy_order<<<grid_for(nh, 256), 256, 0, s>>>(sorted, nh, heavy_list);
            g->launches += 2 + 3 * ((bits_for((uint64_t)(n > 0 ? n - 1 : 0)) + 7) / 8);
        }
    }
    // Hit masks of the heavy edges (rows layout possible): the list fill then reads the masks
    // instead of repeating the lookups.  A graph-owned buffer (reused by later counts);
    // skipped when it would take more than a third of the free memory.
    std::unique_ptr<Scratch> msc;
    int64_t* moff = nullptr;
    uint32_t* masks = nullptr;
    if (rs.tab && cgt) {
        unsigned nh = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nh, nheavy, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        if (nh > 0) {
            msc.reset(new Scratch(g));
            int64_t* wcount = (int64_t*)msc->get(sizeof(int64_t) * (nh + 1));
            moff = (int64_t*)msc->get(sizeof(int64_t) * (nh + 1));
            int64_t* wtmp = (int64_t*)msc->get(sizeof(int64_t) * scan_temp_elems(nh + 1));
            if (!wcount || !moff || !wtmp) {
                set_error("device allocation failed (hit masks)");
                return RTR_ERR_CUDA;
            }
            k_mask_words<<<grid_for(nh + 1, 256), 256, 0, s>>>(g->offsets, g->esrc, g->nbors, g->fwd, heavy_list,
                                                                nh, rs, wcount);
            exclusive_scan_i64(wcount, moff, nh + 1, nullptr, wtmp, s);
            int64_t words = 0;
            RTR_CUDA_TRY(cudaMemcpyAsync(&words, moff + nh, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
            RTR_CUDA_TRY(cudaStreamSynchronize(s));
            const int64_t bytes = (int64_t)sizeof(uint32_t) * (words + 1);
            if (g->rows_masks_cap >= bytes)
                masks = (uint32_t*)g->rows_masks;
            else if (bytes < (int64_t)((device_avail_bytes(g) + g->rows_masks_cap) / 3))
                masks = (uint32_t*)grow_owned(g, &g->rows_masks, &g->rows_masks_cap, bytes);
            if (masks) {
                RTR_CUDA_TRY(cudaMemsetAsync(masks, 0, (size_t)bytes, s));
            } else {
                moff = nullptr;
            }
            g->launches += 2;
        }
    }
    ktime_begin(g, KT_EDGE_HEAVY);
    k_edge_count_heavy<<<gh, kHeavyEdgeBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, g->deg, g->fwd, g->partner,
                                                      heavy_list, nheavy, g->tune_gallop, rs, g->sup, cnt, cgt,
                                                      heavy_pe ? g->pe : nullptr, g->ctr, moff, masks);
    ktime_end(g, KT_EDGE_HEAVY);
    ktime_end(g, KT_EDGE_FOLD);
    exclusive_scan_i64(cnt, g->tl_off, m2 + 1, nullptr, tmp, s);
    g->launches += 6;
    RTR_CUDA_TRY(cudaGetLastError());
    int64_t tl_len = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&tl_len, g->tl_off + m2, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    bool keep_lists = g->count_mode != 2;
    if (g->count_mode == 0 && (tl_len > g->tl_len || !g->tl)) {
        // keep the lists only when they fit beside what the clean will need (records, stacks);
        // a large graph first has the pool return its cached blocks
        // free memory counts the pool's cached blocks (an earlier graph's freed buffers, which a
        // later allocation reuses) and this graph's own rows-layout buffers
        const size_t free_b = device_avail_bytes(g) + (size_t)g->rows_masks_cap + (size_t)g->rows_lists_cap;
        const double need = (double)sizeof(TriEntry) * (double)(tl_len + 1) + 64.0 * (double)(m + 1) +
                            (double)(1ll << 30);
        keep_lists = need <= (double)free_b;
    }
    if (!keep_lists) {
        // rows layout: perVertex and heavy-edge perEdge straight from the CSR rows
        g->lists = false;
        g->tl_len = 0;
        if (!heavy_pe) {  // fold the heavy edges' perEdge now (the counts are recomputed, unchanged)
            unsigned long long* junk = (unsigned long long*)sc.get(sizeof(unsigned long long) * 2);
            if (!junk) {
                set_error("device allocation failed (count scratch)");
                return RTR_ERR_CUDA;
            }
            k_edge_count_heavy<<<gh, kHeavyEdgeBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, g->deg, g->fwd,
                                                              g->partner, heavy_list, nheavy, g->tune_gallop, rs,
                                                              g->sup, cnt, nullptr, g->pe, junk, nullptr, nullptr);
            g->launches += 1;
        }
        // cnt (scanned into tl_off above) is free: it takes the lists' offsets
        const int rc = count_rows(g, sc, rs, cgt, cnt, heavy_list, nheavy, moff, masks);
        if (rc) return rc;
        RTR_CUDA_TRY(cudaGetLastError());
        cudaEventRecord(e1, s);
        RTR_CUDA_TRY(cudaEventSynchronize(e1));
        cudaEventElapsedTime(&g->ms_count, e0, e1);
        ktime_read(g, KT_EDGE_FOLD);
        ktime_read(g, KT_EDGE_LIGHT);
        ktime_read(g, KT_EDGE_HEAVY);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        g->stage = 2;
        return RTR_OK;
    }
    msc.reset();
    // the rows layout's buffers are not needed with lists
    release_owned(g, &g->rows_masks, &g->rows_masks_cap);
    release_owned(g, &g->rows_lists, &g->rows_lists_cap);
    if (tl_len > g->tl_len || !g->tl) {
        // grow-only buffer owned by the graph
        g->tl = (TriEntry*)dev_alloc(g, sizeof(TriEntry) * (tl_len + 1));
        if (!g->tl) {
            set_error("device allocation failed for %lld triangle-list entries", (long long)tl_len);
            return RTR_ERR_CUDA;
        }
    }
    g->tl_len = tl_len;
    g->lists = true;
    ktime_begin(g, KT_TRI_FILL);
    k_tri_fill<<<ge, kBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, g->deg, g->partner, g->fwd, g->frank, m,
                                     g->tl_off, g->tl, g->tune_gallop, g->tune_edge);
    k_tri_fill_heavy<<<gh, kHeavyEdgeBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, g->deg, g->partner, g->fwd,
                                                    g->frank, heavy_list, nheavy, g->tune_gallop, g->tl_off, g->tl);
    k_pe_fold_heavy<<<gh, kHeavyEdgeBlock, 0, s>>>(g->fwd, heavy_list, nheavy, g->tl_off, g->tl, g->pe);
    ktime_end(g, KT_TRI_FILL);
    ktime_begin(g, KT_VERTEX_FOLD);
    k_vertex_fold_light<<<grid_for(n, kBlock), kBlock, 0, s>>>(g->offsets, g->nbors, g->deg, g->partner, n,
                                                                g->tl_off, g->tl, g->pv, g->tune_heavy);
    k_vertex_fold_heavy<<<grid_for(1ll << 40, kHeavyBlock, 16), kHeavyBlock, 0, s>>>(
        g->offsets, g->nbors, g->deg, g->partner, n, g->tl_off, g->tl, g->pv, g->tune_heavy);
    ktime_end(g, KT_VERTEX_FOLD);
    g->launches += 5;
    RTR_CUDA_TRY(cudaGetLastError());
    cudaEventRecord(e1, s);
    RTR_CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&g->ms_count, e0, e1);
    ktime_read(g, KT_EDGE_FOLD);
    ktime_read(g, KT_EDGE_LIGHT);
    ktime_read(g, KT_EDGE_HEAVY);
    ktime_read(g, KT_TRI_FILL);
    ktime_read(g, KT_VERTEX_FOLD);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    g->stage = 2;
    return RTR_OK;
}

}  // namespace rtr
