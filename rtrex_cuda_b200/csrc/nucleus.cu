// The nucleus (truss-hierarchy) path on the device, bit-exact to the
// reference's nucleus driver (RTRex_Sequential/clustering/nucleus.cpp:12-81):
//
//   1. relabel by (degree, id)      CGraph::renameByDegreeOrderMapping (Graph.cpp:261-310):
//                                   a radix sort of (degree, id) keys, then the CSR of the
//                                   relabelled pairs built like any graph (rows ascending)
//   2. per-edge triangle lists      storeAllTriangles (Escape/Nucleus.h:125-163): the list
//                                   layout of count_triangles on the relabelled graph -- for
//                                   each forward edge (i, j), i < j, its common neighbours
//                                   ascending, with the forward ranks of (i, k) and (j, k)
//   3. integer peel                 nuclei's deletion loop (Nucleus.h:349-458): one warp
//                                   replays it in the reference's order -- per threshold c,
//                                   the edges with fewer than c live triangles pushed in slot
//                                   order, popped last-first, each pop's triangles taken 32 at
//                                   a time (within one pop they touch distinct edges, so the
//                                   lanes decrement their own counters; neighbour entries and
//                                   pushes are appended in triangle order)
//   4. edge hierarchy and clusters  findConnectedComponent / completeCluster (Nucleus.h:169-301,
//                                   :460-563): one device thread walks the levels from the top,
//                                   as the reference does; members are gathered with a stamp per
//                                   vertex and sorted by a radix sort of (cluster, vertex) keys
//                                   (the std::set order of relabelled ids), then mapped back to
//                                   the original labels.
//
// Edges are identified by forward rank of the relabelled CSR (the reference uses
// the forward slot; both are ordered the same way and only compared for equality
// past the seeding).  No floating point is involved.
#include "../../include/rtr.h"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>
#include <cstdio>
#include <string>
#include <vector>

namespace rtr {
int make_graph_handle(int64_t n, int device, rtr_graph** out);
}

using namespace rtr;

namespace {

constexpr int kBlock = 256;

__global__ void k_nuc_keys(const int32_t* __restrict__ deg, int64_t n, int B, uint64_t* __restrict__ keys)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)deg[v] << B) | (uint64_t)v;
}

__global__ void k_nuc_rank(const uint64_t* __restrict__ sorted, int64_t n, uint64_t mask, int32_t* __restrict__ inv,
                           int32_t* __restrict__ newid)
{
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        const int32_t v = (int32_t)(sorted[r] & mask);
        inv[r] = v;
        newid[v] = (int32_t)r;
    }
}

__global__ void k_nuc_pairs(const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                            const int32_t* __restrict__ nb, const int32_t* __restrict__ newid, int64_t m,
                            int64_t* __restrict__ u, int64_t* __restrict__ v)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int32_t f = fwd[k];
        u[k] = newid[esrc[f]];
        v[k] = newid[nb[f]];
    }
}

__device__ __forceinline__ int warp_excl(int x, int lane, int* total)
{
    int incl = x;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    *total = __shfl_sync(0xffffffffu, incl, 31);
    return incl - x;
}

enum NucErr : int64_t { NUC_ERR_LEVELS = 1, NUC_ERR_NBR = 2, NUC_ERR_STACK = 4, NUC_ERR_VERT = 8 };

struct PeelArgs {
    int64_t m;               // forward edges of the relabelled graph
    const int32_t* fwd;      // rank -> forward slot
    const int64_t* tl_off;   // slot -> first triangle entry
    const TriEntry* tl;
    const uint32_t* sup;     // slot -> triangle count
    int32_t* tc;             // rank -> live triangles
    uint8_t* del;            // rank -> deleted
    int32_t* kappa;          // rank -> level - 1 at deletion
    int32_t* dtime;          // rank -> deletion index
    int32_t* del_edges;      // deletion index -> rank
    int64_t* del_off;        // level -> first deletion index of the edges of that kappa
    int64_t lv_cap;
    int32_t* nbr;            // neighbour entries, in deletion order
    int64_t* nbr_off;        // deletion index -> first entry
    int64_t nbr_cap;
    int32_t* stack;
    int64_t stack_cap;
    int64_t* out;            // [0] highest kappa, [1] deletions, [2] neighbour entries, [3] error bits
};

__global__ void k_nuc_peel(PeelArgs a)
{
    const int lane = threadIdx.x & 31;
    for (int64_t k = lane; k < a.m; k += 32) {
        a.tc[k] = (int32_t)a.sup[a.fwd[k]];
        a.del[k] = 0;
    }
    if (lane == 0) {
        a.nbr_off[0] = 0;
        a.del_off[0] = 0;
    }
    __syncwarp();
    int64_t c = 1, total = 0, ndel = 0, nn = 0, top = 0, err = 0;
    while (total < a.m && !err) {
        if (c + 1 >= a.lv_cap) {
            err |= NUC_ERR_LEVELS;
            break;
        }
        // the level's seeds, in slot order
        for (int64_t kb = 0; kb < a.m; kb += 32) {
            const int64_t k = kb + lane;
            const bool push = k < a.m && !a.del[k] && a.tc[k] < c;
            const unsigned pm = __ballot_sync(0xffffffffu, push);
            const int np = __popc(pm);
            if (top + np > a.stack_cap) {
                err |= NUC_ERR_STACK;
                break;
            }
            if (push) a.stack[top + __popc(pm & ((1u << lane) - 1u))] = (int32_t)k;
            top += np;
        }
        __syncwarp();
        while (top > 0 && !err) {
            const int32_t e = a.stack[--top];
            const bool gone = a.del[e] != 0;
            __syncwarp();
            if (gone) continue;
            if (lane == 0) {
                a.del[e] = 1;
                a.kappa[e] = (int32_t)(c - 1);
                a.dtime[e] = (int32_t)ndel;
                a.del_edges[ndel] = e;
            }
            ++ndel;
            ++total;
            const int32_t f = a.fwd[e];
            const int64_t t1 = a.tl_off[f + 1];
            for (int64_t tb = a.tl_off[f]; tb < t1; tb += 32) {
                const int64_t t = tb + lane;
                const bool valid = t < t1;
                int32_t ra = 0, rb = 0;
                bool da = true, db = true;
                if (valid) {
                    const TriEntry te = a.tl[t];
                    ra = te.raz;  // (i, k)
                    rb = te.rbz;  // (j, k)
                    da = a.del[ra] != 0;
                    db = a.del[rb] != 0;
                }
                int tn = 0;
                const int on = warp_excl(valid ? (!da) + (!db) : 0, lane, &tn);
                if (nn + tn > a.nbr_cap) {
                    err |= NUC_ERR_NBR;
                    break;
                }
                if (valid && !da) a.nbr[nn + on] = ra;
                if (valid && !db) a.nbr[nn + on + (da ? 0 : 1)] = rb;
                nn += tn;
                bool p1 = false, p2 = false;
                if (valid && !da && !db) {  // the triangle dies: both other edges lose one
                    p1 = --a.tc[ra] < c;
                    p2 = --a.tc[rb] < c;
                }
                int tp = 0;
                const int op = warp_excl((p1 ? 1 : 0) + (p2 ? 1 : 0), lane, &tp);
                if (top + tp > a.stack_cap) {
                    err |= NUC_ERR_STACK;
                    break;
                }
                if (p1) a.stack[top + op] = ra;
                if (p2) a.stack[top + op + (p1 ? 1 : 0)] = rb;
                top += tp;
                __syncwarp();
            }
            if (lane == 0) a.nbr_off[ndel] = nn;
            __syncwarp();
        }
        if (lane == 0) a.del_off[c] = ndel;
        ++c;
    }
    if (lane == 0) {
        a.out[0] = c - 2;
        a.out[1] = ndel;
        a.out[2] = nn;
        a.out[3] = err;
    }
}

struct TreeArgs {
    int64_t m, n, max_c;
    const int32_t* kappa;
    const int32_t* dtime;
    const int32_t* del_edges;
    const int64_t* del_off;
    const int32_t* nbr;
    const int64_t* nbr_off;
    const int32_t* fwd;   // rank -> slot of the relabelled CSR
    const int32_t* esrc;  // slot -> source
    const int32_t* nb;    // slot -> neighbour
    int32_t* parent;
    int32_t* cparent;
    int32_t* ptime;
    int32_t* children;
    int64_t* child_off;
    uint8_t* in_cluster;
    int32_t* roots;
    int64_t* root_off;
    int32_t* stack;
    int64_t stack_cap;
    int32_t* root_to_cluster;
    int32_t* stamp;  // vertex -> last cluster that took it
    int64_t* cl_c;
    int64_t* cl_nv;
    int64_t* cl_ne;
    int64_t* cl_parent;
    int64_t* cl_voff;
    int32_t* cl_vert;
    int64_t vert_cap;
    int64_t* out;  // [0] clusters, [1] member entries, [2] error bits
};

// One thread: the hierarchy walk of nuclei, then completeCluster for every root.
__global__ void k_nuc_tree(TreeArgs a)
{
    int64_t err = 0;
    for (int64_t p = 0; p < a.m; ++p) {
        a.parent[p] = a.cparent[p] = (int32_t)p;
        a.in_cluster[p] = 0;
    }
    for (int64_t v = 0; v < a.n; ++v) a.stamp[v] = -1;
    int64_t pt = 0, nchild = 0, nroots = 0;
    auto push_nbrs = [&](int32_t e, int64_t& sp) {
        const int64_t d = a.dtime[e];
        for (int64_t q = a.nbr_off[d]; q < a.nbr_off[d + 1]; ++q) {
            if (sp >= a.stack_cap) {
                err |= NUC_ERR_STACK;
                return;
            }
            a.stack[sp++] = a.nbr[q];
        }
    };
    for (int64_t lv = a.max_c; lv > 0 && !err; --lv) {
        for (int64_t q = a.del_off[lv]; q < a.del_off[lv + 1]; ++q) {
            const int32_t e = a.del_edges[q];
            a.ptime[e] = (int32_t)pt;
            a.child_off[pt] = nchild;
            ++pt;
            if (a.in_cluster[e]) continue;
            // findConnectedComponent (Nucleus.h:169-242)
            int64_t sp = 0;
            push_nbrs(e, sp);
            a.in_cluster[e] = 1;
            while (sp > 0 && !err) {
                const int32_t x = a.stack[--sp];
                if (a.cparent[x] == e) continue;
                if (a.in_cluster[x]) {
                    int32_t t = x;
                    while (a.cparent[t] != t) {
                        const int32_t up = a.cparent[t];
                        a.cparent[t] = e;
                        t = up;
                    }
                    if (t != e) {
                        a.parent[t] = e;
                        a.cparent[t] = e;
                        a.children[nchild++] = t;
                    }
                    continue;
                }
                a.parent[x] = e;
                a.cparent[x] = e;
                a.children[nchild++] = x;
                a.in_cluster[x] = 1;
                push_nbrs(x, sp);
            }
        }
        a.root_off[a.max_c - lv] = nroots;
        for (int64_t q = a.del_off[lv]; q < a.del_off[lv + 1]; ++q) {
            const int32_t e = a.del_edges[q];
            if (a.parent[e] == e || a.kappa[a.parent[e]] < lv) a.roots[nroots++] = e;
        }
    }
    if (a.max_c >= 0) {
        a.root_off[a.max_c] = nroots;
        for (int64_t q = a.del_off[0]; q < a.del_off[1]; ++q) {
            a.ptime[a.del_edges[q]] = (int32_t)pt;
            a.child_off[pt] = nchild;
            ++pt;
        }
    }
    a.child_off[pt] = nchild;
    // completeCluster (Nucleus.h:246-301), clusters highest level first
    int64_t ncl = 0, vn = 0;
    auto take = [&](int32_t v, int64_t k, int64_t& nv) {
        if (err || a.stamp[v] == (int32_t)k) return;
        if (vn >= a.vert_cap) {  // out of room: stop; the host runs the walk again with more
            err |= NUC_ERR_VERT;
            return;
        }
        a.stamp[v] = (int32_t)k;
        a.cl_vert[vn++] = v;
        ++nv;
    };
    for (int64_t lv = a.max_c; lv > 0 && !err; --lv) {
        for (int64_t q = a.root_off[a.max_c - lv]; q < a.root_off[a.max_c - lv + 1] && !err; ++q) {
            const int32_t root = a.roots[q];
            const int64_t k = ncl++;
            a.root_to_cluster[root] = (int32_t)k;
            a.cl_c[k] = lv;
            a.cl_parent[k] = -1;
            a.cl_voff[k] = vn;
            int64_t ne = 0, nv = 0, sp = 0;
            a.stack[sp++] = root;
            while (sp > 0 && !err) {
                const int32_t e = a.stack[--sp];
                if (a.kappa[e] > lv) {
                    const int64_t ch = a.root_to_cluster[e];
                    ne += a.cl_ne[ch];
                    a.cl_parent[ch] = k;
                    for (int64_t p = a.cl_voff[ch]; p < a.cl_voff[ch] + a.cl_nv[ch] && !err; ++p)
                        take(a.cl_vert[p], k, nv);
                } else {
                    ++ne;
                    const int32_t f = a.fwd[e];
                    take(a.esrc[f], k, nv);
                    take(a.nb[f], k, nv);
                    for (int64_t t = a.child_off[a.ptime[e]]; t < a.child_off[a.ptime[e] + 1]; ++t) {
                        if (sp >= a.stack_cap) {
                            err |= NUC_ERR_STACK;
                            break;
                        }
                        a.stack[sp++] = a.children[t];
                    }
                }
            }
            a.cl_ne[k] = ne;
            a.cl_nv[k] = nv;
        }
    }
    a.cl_voff[ncl] = vn;
    a.out[0] = ncl;
    a.out[1] = vn;
    a.out[2] = err;
}

__global__ void k_nuc_member_keys(const int64_t* __restrict__ voff, int64_t ncl, const int32_t* __restrict__ vert,
                                  int B, uint64_t* __restrict__ keys)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < ncl; k += (int64_t)gridDim.x * blockDim.x)
        for (int64_t p = voff[k]; p < voff[k + 1]; ++p) keys[p] = ((uint64_t)k << B) | (uint64_t)vert[p];
}

__global__ void k_nuc_members(const uint64_t* __restrict__ sorted, int64_t cnt, uint64_t mask,
                              const int32_t* __restrict__ inv, int64_t* __restrict__ out)
{
    for (int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; p < cnt; p += (int64_t)gridDim.x * blockDim.x)
        out[p] = inv[sorted[p] & mask];
}

struct GraphGuard {
    rtr_graph* g = nullptr;
    ~GraphGuard()
    {
        if (g) rtr_graph_destroy(g);
    }
};

int nucleus_run(rtr_graph* g)
{
    const int64_t n = g->n, m = g->m;
    cudaStream_t s = g->stream;
    g->nuc_done = false;
    g->nuc_c.clear();
    g->nuc_nv.clear();
    g->nuc_ne.clear();
    g->nuc_parent.clear();
    g->nuc_off.assign(1, 0);
    g->nuc_vert.clear();
    if (m == 0) {  // no edges, no levels, no clusters
        g->nuc_done = true;
        return RTR_OK;
    }
    const int B = bits_for((uint64_t)(n - 1));
    const uint64_t mask = (1ull << B) - 1;
    GraphGuard rel;
    int32_t* inv = nullptr;
    {
        Scratch sc(g);
        uint64_t* k1 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
        uint64_t* k2 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
        void* rtmp = sc.get(radix_temp_bytes(n));
        int32_t* newid = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
        int64_t* du = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
        int64_t* dv = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
        inv = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        if (!k1 || !k2 || !rtmp || !newid || !du || !dv || !inv) {
            set_error("device allocation failed (nucleus relabel)");
            return RTR_ERR_CUDA;
        }
        const int gn = grid_for(n, kBlock);
        k_nuc_keys<<<gn, kBlock, 0, s>>>(g->deg, n, B, k1);
        uint64_t* sorted = radix_sort_u64(k1, k2, n, B + bits_for((uint64_t)g->m2), rtmp, s);
        k_nuc_rank<<<gn, kBlock, 0, s>>>(sorted, n, mask, inv, newid);
        k_nuc_pairs<<<grid_for(m, kBlock), kBlock, 0, s>>>(g->fwd, g->esrc, g->nbors, newid, m, du, dv);
        g->launches += 3 + 3 * ((B + bits_for((uint64_t)g->m2) + 7) / 8);
        RTR_CUDA_TRY(cudaGetLastError());
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        int rc = make_graph_handle(n, g->device, &rel.g);
        if (rc) return rc;
        rc = build_csr(rel.g, du, dv, m, false);
        if (!rc) RTR_CUDA_TRY(cudaStreamSynchronize(rel.g->stream));
        if (rc) return rc;
    }
    rtr_graph* r = rel.g;
    r->count_mode = 1;  // the lists are the reference's triangle lists
    int rc = count_triangles(r);
    if (rc) return rc;
    cudaStream_t rs = r->stream;
    Scratch sc(r);
    const int64_t T3 = r->tl_len;  // 3 x triangles
    const int64_t lv_cap = std::min<int64_t>(n, m) + 4;
    PeelArgs pa;
    pa.m = m;
    pa.fwd = r->fwd;
    pa.tl_off = r->tl_off;
    pa.tl = r->tl;
    pa.sup = r->sup;
    pa.tc = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    pa.del = (uint8_t*)sc.get(m + 16);
    pa.kappa = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    pa.dtime = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    pa.del_edges = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    pa.del_off = (int64_t*)sc.get(sizeof(int64_t) * (lv_cap + 1));
    pa.lv_cap = lv_cap;
    pa.nbr_cap = T3 + 32;  // every triangle yields at most three entries
    pa.nbr = (int32_t*)sc.get(sizeof(int32_t) * (pa.nbr_cap + 1));
    pa.nbr_off = (int64_t*)sc.get(sizeof(int64_t) * (m + 2));
    pa.stack_cap = m + 2 * (T3 / 3) + 64;  // the seeds of a level plus one push per triangle decrement
    pa.stack = (int32_t*)sc.get(sizeof(int32_t) * (pa.stack_cap + 1));
    pa.out = (int64_t*)sc.get(sizeof(int64_t) * 8);
    if (!pa.tc || !pa.del || !pa.kappa || !pa.dtime || !pa.del_edges || !pa.del_off || !pa.nbr || !pa.nbr_off ||
        !pa.stack || !pa.out) {
        set_error("device allocation failed (nucleus peel)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(pa.out, 0, sizeof(int64_t) * 8, rs));
    k_nuc_peel<<<1, 32, 0, rs>>>(pa);
    g->launches += 1;
    int64_t po[4] = {0, 0, 0, 0};
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaMemcpyAsync(po, pa.out, sizeof po, cudaMemcpyDeviceToHost, rs));
    RTR_CUDA_TRY(cudaStreamSynchronize(rs));
    if (po[3] || po[1] != m) {
        set_error("nucleus peel reported 0x%llx (%lld of %lld edges deleted)", (long long)po[3], (long long)po[1],
                  (long long)m);
        return RTR_ERR_DEVICE;
    }
    TreeArgs ta;
    ta.m = m;
    ta.n = n;
    ta.max_c = po[0];
    ta.kappa = pa.kappa;
    ta.dtime = pa.dtime;
    ta.del_edges = pa.del_edges;
    ta.del_off = pa.del_off;
    ta.nbr = pa.nbr;
    ta.nbr_off = pa.nbr_off;
    ta.fwd = r->fwd;
    ta.esrc = r->esrc;
    ta.nb = r->nbors;
    ta.parent = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.cparent = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.ptime = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.children = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.child_off = (int64_t*)sc.get(sizeof(int64_t) * (m + 2));
    ta.in_cluster = (uint8_t*)sc.get(m + 16);
    ta.roots = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.root_off = (int64_t*)sc.get(sizeof(int64_t) * (lv_cap + 2));
    ta.stack_cap = std::max<int64_t>(po[2], m) + 64;
    ta.stack = (int32_t*)sc.get(sizeof(int32_t) * (ta.stack_cap + 1));
    ta.root_to_cluster = (int32_t*)sc.get(sizeof(int32_t) * (m + 1));
    ta.stamp = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    ta.cl_c = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    ta.cl_nv = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    ta.cl_ne = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    ta.cl_parent = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    ta.cl_voff = (int64_t*)sc.get(sizeof(int64_t) * (m + 2));
    ta.out = (int64_t*)sc.get(sizeof(int64_t) * 4);
    if (!ta.parent || !ta.cparent || !ta.ptime || !ta.children || !ta.child_off || !ta.in_cluster || !ta.roots ||
        !ta.root_off || !ta.stack || !ta.root_to_cluster || !ta.stamp || !ta.cl_c || !ta.cl_nv || !ta.cl_ne ||
        !ta.cl_parent || !ta.cl_voff || !ta.out) {
        set_error("device allocation failed (nucleus hierarchy)");
        return RTR_ERR_CUDA;
    }
    // member entries: clusters nest, so a vertex can sit in one cluster per level;
    // start from a few times n and grow if that is short
    int64_t vcap = 4 * n + 2 * m + 64;
    int64_t to[3] = {0, 0, 0};
    for (int attempt = 0; attempt < 4; ++attempt) {
        ta.vert_cap = vcap;
        ta.cl_vert = (int32_t*)sc.get(sizeof(int32_t) * (vcap + 1));
        if (!ta.cl_vert) {
            set_error("device allocation failed (%lld nucleus member entries)", (long long)vcap);
            return RTR_ERR_CUDA;
        }
        k_nuc_tree<<<1, 1, 0, rs>>>(ta);
        g->launches += 1;
        RTR_CUDA_TRY(cudaGetLastError());
        RTR_CUDA_TRY(cudaMemcpyAsync(to, ta.out, sizeof to, cudaMemcpyDeviceToHost, rs));
        RTR_CUDA_TRY(cudaStreamSynchronize(rs));
        if (to[2] != NUC_ERR_VERT) break;
        vcap *= 4;  // the walk stopped at the first entry it could not store; run it again with room
    }
    if (to[2]) {
        set_error("nucleus hierarchy reported 0x%llx", (long long)to[2]);
        return RTR_ERR_DEVICE;
    }
    const int64_t ncl = to[0], cnt = to[1];
    g->nuc_c.resize(ncl);
    g->nuc_nv.resize(ncl);
    g->nuc_ne.resize(ncl);
    g->nuc_parent.resize(ncl);
    g->nuc_off.resize(ncl + 1);
    g->nuc_vert.resize(cnt);
    if (ncl > 0) {
        RTR_CUDA_TRY(cudaMemcpyAsync(g->nuc_c.data(), ta.cl_c, sizeof(int64_t) * ncl, cudaMemcpyDeviceToHost, rs));
        RTR_CUDA_TRY(cudaMemcpyAsync(g->nuc_nv.data(), ta.cl_nv, sizeof(int64_t) * ncl, cudaMemcpyDeviceToHost, rs));
        RTR_CUDA_TRY(cudaMemcpyAsync(g->nuc_ne.data(), ta.cl_ne, sizeof(int64_t) * ncl, cudaMemcpyDeviceToHost, rs));
        RTR_CUDA_TRY(
            cudaMemcpyAsync(g->nuc_parent.data(), ta.cl_parent, sizeof(int64_t) * ncl, cudaMemcpyDeviceToHost, rs));
    }
    RTR_CUDA_TRY(cudaMemcpyAsync(g->nuc_off.data(), ta.cl_voff, sizeof(int64_t) * (ncl + 1), cudaMemcpyDeviceToHost,
                                 rs));
    if (cnt > 0) {
        // members of each cluster ascending in relabelled id (std::set order), then original labels
        const int KB = bits_for((uint64_t)ncl);
        uint64_t* mk = (uint64_t*)sc.get(sizeof(uint64_t) * (cnt + 1));
        uint64_t* ma = (uint64_t*)sc.get(sizeof(uint64_t) * (cnt + 1));
        void* mt = sc.get(radix_temp_bytes(cnt));
        int64_t* mv = (int64_t*)sc.get(sizeof(int64_t) * (cnt + 1));
        if (!mk || !ma || !mt || !mv) {
            set_error("device allocation failed (nucleus members)");
            return RTR_ERR_CUDA;
        }
        k_nuc_member_keys<<<grid_for(ncl, kBlock), kBlock, 0, rs>>>(ta.cl_voff, ncl, ta.cl_vert, B, mk);
        uint64_t* ms = radix_sort_u64(mk, ma, cnt, B + KB, mt, rs);
        k_nuc_members<<<grid_for(cnt, kBlock), kBlock, 0, rs>>>(ms, cnt, mask, inv, mv);
        g->launches += 2 + 3 * ((B + KB + 7) / 8);
        RTR_CUDA_TRY(cudaGetLastError());
        RTR_CUDA_TRY(cudaMemcpyAsync(g->nuc_vert.data(), mv, sizeof(int64_t) * cnt, cudaMemcpyDeviceToHost, rs));
    }
    RTR_CUDA_TRY(cudaStreamSynchronize(rs));
    g->nuc_done = true;
    return RTR_OK;
}

}  // namespace

extern "C" {

int rtr_nucleus(rtr_graph* g, int64_t* n_clusters)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (g->stage < 1) {
        set_error("nucleus called before the graph was built");
        return RTR_ERR_STATE;
    }
    if (g->nbatch > 0) {
        set_error("the nucleus path is not defined for a batch handle");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, g->stream);
    const int rc = nucleus_run(g);
    cudaEventRecord(e1, g->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&g->ms_nucleus, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    if (n_clusters) *n_clusters = (int64_t)g->nuc_c.size();
    return RTR_OK;
}

int rtr_get_nuclei(const rtr_graph* g, int64_t* n_clusters, int64_t* n_members, int64_t* c, int64_t* nv,
                   int64_t* ne, int64_t* parent, int64_t* off, int64_t* vert)
{
    if (!g || !g->nuc_done) {
        set_error("the nucleus path has not run on this graph");
        return RTR_ERR_STATE;
    }
    const size_t k = g->nuc_c.size();
    if (n_clusters) *n_clusters = (int64_t)k;
    if (n_members) *n_members = (int64_t)g->nuc_vert.size();
    if (c) std::copy(g->nuc_c.begin(), g->nuc_c.end(), c);
    if (nv) std::copy(g->nuc_nv.begin(), g->nuc_nv.end(), nv);
    if (ne) std::copy(g->nuc_ne.begin(), g->nuc_ne.end(), ne);
    if (parent) std::copy(g->nuc_parent.begin(), g->nuc_parent.end(), parent);
    if (off) std::copy(g->nuc_off.begin(), g->nuc_off.end(), off);
    if (vert) std::copy(g->nuc_vert.begin(), g->nuc_vert.end(), vert);
    return RTR_OK;
}

int rtr_write_nuclei(const rtr_graph* g, const char* path)
{
    if (!g || !path || !g->nuc_done) {
        set_error("null argument, or the nucleus path has not run on this graph");
        return !g || !path ? RTR_ERR_ARG : RTR_ERR_STATE;
    }
    FILE* f = fopen(path, "w");
    if (!f) {
        set_error("could not open %s for writing", path);
        return RTR_ERR_IO;
    }
    std::string line;
    for (size_t k = 0; k < g->nuc_c.size(); ++k) {
        char head[160];
        snprintf(head, sizeof head, "Cluster id: %lld, C: %lld, n_vertices: %lld, n_edges: %lld, parent: %lld\n",
                 (long long)k, (long long)g->nuc_c[k], (long long)g->nuc_nv[k], (long long)g->nuc_ne[k],
                 (long long)g->nuc_parent[k]);
        line.assign(head);
        for (int64_t p = g->nuc_off[k]; p < g->nuc_off[k + 1]; ++p) {
            line += std::to_string(g->nuc_vert[p]);
            line += ' ';
        }
        line += '\n';
        if (fwrite(line.data(), 1, line.size(), f) != line.size()) {
            fclose(f);
            set_error("short write to %s", path);
            return RTR_ERR_IO;
        }
    }
    if (fclose(f) != 0) {
        set_error("could not close %s", path);
        return RTR_ERR_IO;
    }
    return RTR_OK;
}

}  // extern "C"
