// Cluster expansion: expandClusters (RTRex_Sequential/Escape/Decomposition.h:958-1008),
// the RTRex driver's mode e (RTRex_Sequential/clustering/RTRex.cpp:196-201).
//
// The reference walks the clusters in creation order; for every cluster that had
// one vertex when extraction ended it takes the set's first vertex v, counts v's
// neighbours per cluster of the extraction's (never updated) cluster map, and
// moves v into the cluster whose count first reached the maximum, when that
// maximum exceeds the threshold; the score of v is max / deg(v).  Statistics are
// then recomputed for every cluster.
//
// On the device:
//   * votes (k_expand_vote): one warp per singleton; a chunk of 32 neighbours is
//     ranked per cluster id with __match_any_sync, running counts live in a
//     per-warp open-addressing table (shared memory up to kTabDeg neighbours, a
//     global slice beyond), and the first position whose prefix count reaches the
//     running maximum gives the winner, exactly as the reference's strict '>'
//     update does.  The vote of a vertex depends only on the extraction's map.
//   * moves, threshold >= 1: a singleton cluster can never win (one member gives a
//     count of at most 1), so no singleton set changes before it is processed and
//     every singleton's vote is its own vertex's.  Moves are grouped by target
//     (stable radix sort keeps creation order) and each target cluster replays its
//     inserts on a rebuilt std::unordered_set state (UsetOrder) in parallel.
//   * moves, threshold <= 0: singleton clusters can win, so a later singleton set
//     may hold several vertices and its "first" vertex depends on the inserts
//     before it.  One device thread replays the loop over rebuilt set states
//     (insert into the winner, erase from the singleton), using the precomputed
//     votes.  A vertex moved into a singleton cluster and then voting for that
//     same cluster is erased from every set, as in the reference.
//   * statistics from the new membership (k_expand_stats: populateStats,
//     Decomposition.h:473-491), scores in ascending vertex order (std::map).
#include "primitives.cuh"
#include "rtr_graph.cuh"
#include "stl_order.cuh"

#include <algorithm>

namespace rtr {
namespace {

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kTab = 1024;        // per-warp shared table slots (power of two)
constexpr int kTabDeg = kTab / 2; // singletons up to this degree use the shared table

__global__ void k_singleton_flags(const int64_t* __restrict__ cl_off, int64_t ncl, uint32_t* __restrict__ flag)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x)
        flag[c] = (cl_off[c + 1] - cl_off[c] == 1) ? 1u : 0u;
}

__host__ __device__ inline int64_t pow2_at_least(int64_t x)
{
    int64_t p = 1;
    while (p < x) p <<= 1;
    return p;
}

// Singleton list in creation order; vertex -> singleton index; global table size
// for high-degree singletons.
__global__ void k_singleton_list(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, int64_t ncl,
                                 const int64_t* __restrict__ cl_off, const int32_t* __restrict__ cl_vert,
                                 const int64_t* __restrict__ off, int32_t* __restrict__ s_cluster,
                                 int32_t* __restrict__ s_vertex, int32_t* __restrict__ vs,
                                 int64_t* __restrict__ s_tab)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        if (!flag[c]) continue;
        const uint32_t s = pos[c];
        const int32_t v = cl_vert[cl_off[c]];
        s_cluster[s] = (int32_t)c;
        s_vertex[s] = v;
        vs[v] = (int32_t)s;
        const int64_t d = off[v + 1] - off[v];
        s_tab[s] = d > kTabDeg ? pow2_at_least(2 * d) : 0;
    }
}

// Adds `add` to cid's running count; returns the count before.  Only one lane
// of the warp touches a given cid per call round, other lanes may race for
// empty slots (claimed with CAS).  Keys are stored as cid + 1 (0 = empty).  The
// table has at least twice as many slots as the row has entries, so a probe
// sequence always ends; a full sweep without a slot is reported, not looped.
__device__ inline int table_add(int* tk, int* tc, int64_t cap, int cid, int add, unsigned* err)
{
    int64_t h = ((uint32_t)cid * 2654435761u) & (cap - 1);
    for (int64_t probe = 0; probe < cap; ++probe) {
        const int k = tk[h];
        if (k == cid + 1) return atomicAdd(&tc[h], add);
        if (k == 0) {
            const int prev = atomicCAS(&tk[h], 0, cid + 1);
            if (prev == 0 || prev == cid + 1) return atomicAdd(&tc[h], add);
        }
        h = (h + 1) & (cap - 1);
    }
    atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
    return 0;
}

__global__ void __launch_bounds__(kBlock) k_expand_vote(
    const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ cluster_of,
    const int32_t* __restrict__ s_vertex, int64_t S, const int64_t* __restrict__ s_toff, int* __restrict__ gtab,
    int64_t threshold, int32_t* __restrict__ s_best, double* __restrict__ s_score, unsigned* __restrict__ err)
{
    extern __shared__ int smem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    int* stk = smem + wib * 2 * kTab;
    int* stc = stk + kTab;
    const unsigned lane_le = (lane == 31) ? 0xffffffffu : ((1u << (lane + 1)) - 1);
    const int64_t nwarps = (int64_t)gridDim.x * kWarps;
    for (int64_t s = blockIdx.x * (int64_t)kWarps + wib; s < S; s += nwarps) {
        const int32_t v = s_vertex[s];
        const int64_t r0 = off[v], r1 = off[v + 1], d = r1 - r0;
        int* tk = stk;
        int* tc = stc;
        int64_t cap = kTab;
        if (d > kTabDeg) {
            tk = gtab + 2 * s_toff[s];
            cap = s_toff[s + 1] - s_toff[s];
            tc = tk + cap;
        } else if (d > 32) {
            for (int i = lane; i < kTab; i += 32) {
                stk[i] = 0;
                stc[i] = 0;
            }
            __syncwarp();
        }
        int curmax = 0, best = -1;
        for (int64_t base = r0; base < r1; base += 32) {
            const int64_t j = base + lane;
            const int cid = j < r1 ? cluster_of[nb[j]] : -1;
            const bool act = cid >= 0;  // cluster_map[u] == -1 is skipped (Decomposition.h:976-978)
            const unsigned amask = __ballot_sync(0xffffffffu, act);
            int p = 0;
            if (act) {
                const unsigned peers = __match_any_sync(amask, cid);
                const int leader = __ffs(peers) - 1;
                int before = 0;
                if (d > 32 && lane == leader) before = table_add(tk, tc, cap, cid, __popc(peers), err);
                before = __shfl_sync(peers, before, leader);
                p = before + __popc(peers & lane_le);
            }
            const int pmax = __reduce_max_sync(0xffffffffu, (unsigned)p);
            if (pmax > curmax) {
                const unsigned at = __ballot_sync(0xffffffffu, p == pmax);
                best = __shfl_sync(0xffffffffu, cid, __ffs(at) - 1);
                curmax = pmax;
            }
            __syncwarp();
        }
        if (lane == 0) {
            const bool won = best >= 0 && (int64_t)curmax > threshold;
            s_best[s] = won ? best : -1;
            s_score[s] = won ? (double)curmax / (double)d : 0.0;
        }
        __syncwarp();
    }
}

__global__ void k_inbound(const int32_t* __restrict__ s_best, int64_t S, uint32_t* __restrict__ inbound)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S; s += (int64_t)gridDim.x * blockDim.x)
        if (s_best[s] >= 0) atomicAdd(&inbound[s_best[s]], 1u);
}

// Capacity of the rebuilt set of each cluster that changes: members plus
// possible arrivals.  all_singletons: the sequential replay also needs a state
// for every singleton cluster.
__global__ void k_caps(const int64_t* __restrict__ cl_off, int64_t ncl, const uint32_t* __restrict__ inbound,
                       int all_singletons, int64_t* __restrict__ ncap, int64_t* __restrict__ bcap)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nv = cl_off[c + 1] - cl_off[c];
        const bool touched = inbound[c] > 0 || (all_singletons && nv == 1);
        const int64_t cap = touched ? nv + inbound[c] : 0;
        ncap[c] = cap;
        bcap[c] = cap ? uset_buckets_after(cap) : 0;
    }
}

struct SetStates {
    int32_t* key;
    int32_t* next;
    int32_t* bucket;
    const int64_t* noff;
    const int64_t* boff;
    int32_t* head;
    int32_t* size;
    int32_t* used;
    int64_t* nbuckets;

    __device__ UsetOrder load(int64_t c) const
    {
        UsetOrder u;
        u.key = key + noff[c];
        u.next = next + noff[c];
        u.bucket = bucket + boff[c];
        u.head = head[c];
        u.size = size[c];
        u.used = used[c];
        u.nbuckets = nbuckets[c];
        return u;
    }
    __device__ void store(int64_t c, const UsetOrder& u) const
    {
        head[c] = u.head;
        size[c] = u.size;
        used[c] = u.used;
        nbuckets[c] = u.nbuckets;
    }
};

// Rebuild the member sets of the clusters that change from their iteration
// order (a set built by inserts only; copies keep order and bucket count).
__global__ void k_states_init(SetStates st, const int64_t* __restrict__ cl_off, const int32_t* __restrict__ cl_vert,
                              int64_t ncl)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        if (st.noff[c + 1] == st.noff[c]) continue;
        const int64_t b = cl_off[c], nv = cl_off[c + 1] - b;
        int32_t* key = st.key + st.noff[c];
        for (int64_t i = 0; i < nv; ++i) key[i] = cl_vert[b + i];
        UsetOrder u;
        u.init_from_list(key, st.next + st.noff[c], st.bucket + st.boff[c], (int32_t)nv);
        st.store(c, u);
    }
}

__global__ void k_move_keys(const int32_t* __restrict__ s_best, int64_t S, int sbits, uint64_t* __restrict__ keys,
                            uint32_t* __restrict__ nmoves)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S; s += (int64_t)gridDim.x * blockDim.x) {
        if (s_best[s] < 0) continue;
        const uint32_t i = atomicAdd(nmoves, 1u);
        keys[i] = ((uint64_t)s_best[s] << sbits) | (uint64_t)s;
    }
}

// threshold >= 1: each target cluster inserts its arrivals in creation order.
__global__ void k_apply_parallel(SetStates st, const uint64_t* __restrict__ mk, int64_t nm, int sbits,
                                 const int32_t* __restrict__ s_vertex, unsigned* __restrict__ err)
{
    const uint64_t smask = (1ull << sbits) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nm; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t c = (int64_t)(mk[i] >> sbits);
        if (i > 0 && (int64_t)(mk[i - 1] >> sbits) == c) continue;
        UsetOrder u = st.load(c);
        const int64_t cap = st.noff[c + 1] - st.noff[c];
        for (int64_t j = i; j < nm && (int64_t)(mk[j] >> sbits) == c; ++j) {
            if (u.used >= cap) {
                atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
                break;
            }
            u.insert(s_vertex[mk[j] & smask]);
        }
        st.store(c, u);
    }
}

// threshold <= 0: the reference's loop, one thread, over rebuilt states.
__global__ void k_apply_sequential(SetStates st, const int32_t* __restrict__ s_cluster, int64_t S,
                                   const int32_t* __restrict__ vs, const int32_t* __restrict__ s_best,
                                   uint8_t* __restrict__ moved, unsigned* __restrict__ err)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int64_t s = 0; s < S; ++s) {
        const int64_t c = s_cluster[s];
        UsetOrder u = st.load(c);
        if (u.head < 0) continue;
        const int32_t v = u.key[u.head];  // *decomposition[i].vertices.cbegin()
        const int32_t sv = vs[v];
        if (sv < 0) {  // only singleton vertices ever move
            atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
            return;
        }
        const int32_t b = s_best[sv];
        if (b < 0) continue;
        if (b != c) {
            UsetOrder t = st.load(b);
            if (t.used >= st.noff[b + 1] - st.noff[b] && !t.contains(v)) {
                atomicOr(err, (unsigned)DEV_ERR_SCRATCH);
                return;
            }
            t.insert(v);
            st.store(b, t);
        }
        u.erase(v);  // with b == c the insert was a no-op and v leaves every set
        st.store(c, u);
        moved[v] = 1;
    }
}

__global__ void k_mark_moved(const int32_t* __restrict__ s_best, const int32_t* __restrict__ s_vertex, int64_t S,
                             uint8_t* __restrict__ moved)
{
    for (int64_t s = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; s < S; s += (int64_t)gridDim.x * blockDim.x)
        if (s_best[s] >= 0) moved[s_vertex[s]] = 1;
}

__global__ void k_new_sizes(SetStates st, const int64_t* __restrict__ cl_off, const int32_t* __restrict__ cl_vert,
                            int64_t ncl, const uint8_t* __restrict__ moved, int64_t* __restrict__ nsz)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        const int64_t nv = cl_off[c + 1] - cl_off[c];
        if (st.noff[c + 1] > st.noff[c]) nsz[c] = st.size[c];
        else if (nv == 1 && moved[cl_vert[cl_off[c]]]) nsz[c] = 0;  // emptied singleton
        else nsz[c] = nv;
    }
}

__global__ void k_emit(SetStates st, const int64_t* __restrict__ cl_off, const int32_t* __restrict__ cl_vert,
                       int64_t ncl, const int64_t* __restrict__ xoff, int32_t* __restrict__ xvert,
                       int32_t* __restrict__ xcof)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x) {
        int64_t w = xoff[c];
        const int64_t end = xoff[c + 1];
        if (st.noff[c + 1] > st.noff[c]) {
            const UsetOrder u = st.load(c);
            for (int32_t p = u.head; p != -1 && w < end; p = u.next[p]) {
                xvert[w++] = u.key[p];
                xcof[u.key[p]] = (int32_t)c;
            }
        } else {
            for (int64_t p = cl_off[c]; w < end; ++p) {
                xvert[w++] = cl_vert[p];
                xcof[cl_vert[p]] = (int32_t)c;
            }
        }
    }
}

// populateStats (Decomposition.h:473-491) over the new membership; vertices in
// no cluster (see the header) are skipped.
__global__ void k_expand_stats(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, int64_t n,
                               const int32_t* __restrict__ cof, unsigned long long* __restrict__ ne,
                               unsigned long long* __restrict__ cut)
{
    for (int64_t z = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; z < n; z += (int64_t)gridDim.x * blockDim.x) {
        const int32_t c = cof[z];
        if (c < 0) continue;
        unsigned long long in = 0, outc = 0;
        for (int64_t j = off[z]; j < off[z + 1]; ++j) {
            if (cof[nb[j]] == c) ++in;
            else ++outc;
        }
        if (in) atomicAdd(&ne[c], in);
        if (outc) atomicAdd(&cut[c], outc);
    }
}

__global__ void k_halve_ne(int64_t* __restrict__ ne, int64_t ncl)
{
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < ncl; c += (int64_t)gridDim.x * blockDim.x)
        ne[c] /= 2;
}

__global__ void k_u8_to_u32(const uint8_t* __restrict__ a, int64_t n, uint32_t* __restrict__ b)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        b[i] = a[i];
}

__global__ void k_scores(const uint8_t* __restrict__ moved, const uint32_t* __restrict__ pos, int64_t n,
                         const int32_t* __restrict__ vs, const double* __restrict__ s_score,
                         int32_t* __restrict__ scv, double* __restrict__ scx)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (!moved[v]) continue;
        scv[pos[v]] = (int32_t)v;
        scx[pos[v]] = s_score[vs[v]];
    }
}

}  // namespace

int expand_clusters(rtr_graph* g, int64_t threshold)
{
    if (g->stage < 4) {
        set_error("expand called before extraction");
        return RTR_ERR_STATE;
    }
    if (g->vbase) {
        set_error("expand is defined for a single graph, not a batch");
        return RTR_ERR_ARG;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, ncl = g->ncl;
    Scratch sc(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr + 1, 0, sizeof(unsigned long long), s));
    unsigned* err = (unsigned*)(g->ctr + 1);

    if (!g->x_off) {
        g->x_off = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 2));
        g->x_vert = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        g->x_ne = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 1));
        g->x_cut = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 1));
        g->x_cof = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        g->x_scv = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        g->x_scx = (double*)dev_alloc(g, sizeof(double) * (n + 1));
        if (!g->x_off || !g->x_vert || !g->x_ne || !g->x_cut || !g->x_cof || !g->x_scv || !g->x_scx) {
            set_error("device allocation failed (expand outputs)");
            return RTR_ERR_CUDA;
        }
    }
    if (ncl == 0) {
        RTR_CUDA_TRY(cudaMemsetAsync(g->x_off, 0, sizeof(int64_t), s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        g->x_nscores = 0;
        g->x_threshold = threshold;
        g->expanded = true;
        return RTR_OK;
    }
    const int gk = grid_for(ncl, kBlock), gn = grid_for(n, kBlock);

    // singletons in creation order
    uint32_t* flag = (uint32_t*)sc.get(sizeof(uint32_t) * (ncl + 1));
    uint32_t* fpos = (uint32_t*)sc.get(sizeof(uint32_t) * (ncl + 1));
    uint32_t* utmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(std::max(ncl, n) + 1));
    uint32_t* d_cnt = (uint32_t*)sc.get(sizeof(uint32_t) * 4);
    int32_t* vs = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    uint8_t* moved = (uint8_t*)sc.get(n + 16);
    if (!flag || !fpos || !utmp || !d_cnt || !vs || !moved) {
        set_error("device allocation failed (expand setup)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(vs, 0xff, sizeof(int32_t) * (n + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(moved, 0, n + 16, s));
    RTR_CUDA_TRY(cudaMemsetAsync(d_cnt, 0, sizeof(uint32_t) * 4, s));
    k_singleton_flags<<<gk, kBlock, 0, s>>>(g->cl_off, ncl, flag);
    exclusive_scan_u32(flag, fpos, ncl, d_cnt, utmp, s);
    g->launches += 4;
    uint32_t S32 = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&S32, d_cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    const int64_t S = S32;

    int32_t* s_cluster = (int32_t*)sc.get(sizeof(int32_t) * (S + 1));
    int32_t* s_vertex = (int32_t*)sc.get(sizeof(int32_t) * (S + 1));
    int32_t* s_best = (int32_t*)sc.get(sizeof(int32_t) * (S + 1));
    double* s_score = (double*)sc.get(sizeof(double) * (S + 1));
    int64_t* s_tab = (int64_t*)sc.get(sizeof(int64_t) * (S + 1));
    int64_t* s_toff = (int64_t*)sc.get(sizeof(int64_t) * (S + 2));
    int64_t* ltmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(std::max(S, ncl) + 2));
    int64_t* d_tot = (int64_t*)sc.get(sizeof(int64_t) * 4);
    if (!s_cluster || !s_vertex || !s_best || !s_score || !s_tab || !s_toff || !ltmp || !d_tot) {
        set_error("device allocation failed (expand singletons)");
        return RTR_ERR_CUDA;
    }
    const int gs = grid_for(S, kBlock);
    if (S > 0) {
        k_singleton_list<<<gk, kBlock, 0, s>>>(flag, fpos, ncl, g->cl_off, g->cl_vert, g->offsets, s_cluster,
                                               s_vertex, vs, s_tab);
        exclusive_scan_i64(s_tab, s_toff, S, s_toff + S, ltmp, s);
        g->launches += 4;
    }
    int64_t tab_total = 0;
    if (S > 0) {
        RTR_CUDA_TRY(cudaMemcpyAsync(&tab_total, s_toff + S, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
    }
    int* gtab = (int*)sc.get(sizeof(int) * (2 * tab_total + 2));
    if (!gtab) {
        set_error("device allocation failed (expand vote tables)");
        return RTR_ERR_CUDA;
    }
    if (tab_total) RTR_CUDA_TRY(cudaMemsetAsync(gtab, 0, sizeof(int) * 2 * tab_total, s));

    const size_t smem = sizeof(int) * 2 * kTab * kWarps;
    RTR_CUDA_TRY(cudaFuncSetAttribute(k_expand_vote, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    if (S > 0) {
        const int blocks = (int)std::max<int64_t>(1, std::min<int64_t>((S + kWarps - 1) / kWarps,
                                                                        grid_for(1 << 30, kBlock, 4)));
        k_expand_vote<<<blocks, kBlock, smem, s>>>(g->offsets, g->nbors, g->cluster_of, s_vertex, S, s_toff, gtab,
                                                   threshold, s_best, s_score, err);
        g->launches += 1;
    }

    // rebuilt set states of the clusters that change
    uint32_t* inbound = (uint32_t*)sc.get(sizeof(uint32_t) * (ncl + 1));
    int64_t* ncap = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 1));
    int64_t* bcap = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 1));
    int64_t* noff = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 2));
    int64_t* boff = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 2));
    if (!inbound || !ncap || !bcap || !noff || !boff) {
        set_error("device allocation failed (expand states)");
        return RTR_ERR_CUDA;
    }
    const bool sequential = threshold <= 0;
    RTR_CUDA_TRY(cudaMemsetAsync(inbound, 0, sizeof(uint32_t) * (ncl + 1), s));
    if (S > 0) k_inbound<<<gs, kBlock, 0, s>>>(s_best, S, inbound);
    k_caps<<<gk, kBlock, 0, s>>>(g->cl_off, ncl, inbound, sequential ? 1 : 0, ncap, bcap);
    exclusive_scan_i64(ncap, noff, ncl, noff + ncl, ltmp, s);
    exclusive_scan_i64(bcap, boff, ncl, boff + ncl, ltmp, s);
    g->launches += 9;
    int64_t caps[2] = {0, 0};
    RTR_CUDA_TRY(cudaMemcpyAsync(&caps[0], noff + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(&caps[1], boff + ncl, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));

    SetStates st;
    st.key = (int32_t*)sc.get(sizeof(int32_t) * (caps[0] + 1));
    st.next = (int32_t*)sc.get(sizeof(int32_t) * (caps[0] + 1));
    st.bucket = (int32_t*)sc.get(sizeof(int32_t) * (caps[1] + 1));
    st.noff = noff;
    st.boff = boff;
    st.head = (int32_t*)sc.get(sizeof(int32_t) * (ncl + 1));
    st.size = (int32_t*)sc.get(sizeof(int32_t) * (ncl + 1));
    st.used = (int32_t*)sc.get(sizeof(int32_t) * (ncl + 1));
    st.nbuckets = (int64_t*)sc.get(sizeof(int64_t) * (ncl + 1));
    if (!st.key || !st.next || !st.bucket || !st.head || !st.size || !st.used || !st.nbuckets) {
        set_error("device allocation failed (expand set states)");
        return RTR_ERR_CUDA;
    }
    k_states_init<<<gk, kBlock, 0, s>>>(st, g->cl_off, g->cl_vert, ncl);
    g->launches += 1;

    if (sequential) {
        if (S > 0) k_apply_sequential<<<1, 1, 0, s>>>(st, s_cluster, S, vs, s_best, moved, err);
        g->launches += 1;
    } else if (S > 0) {
        uint64_t* mk = (uint64_t*)sc.get(sizeof(uint64_t) * (S + 1));
        uint64_t* malt = (uint64_t*)sc.get(sizeof(uint64_t) * (S + 1));
        void* rtmp = sc.get(radix_temp_bytes(S));
        if (!mk || !malt || !rtmp) {
            set_error("device allocation failed (expand moves)");
            return RTR_ERR_CUDA;
        }
        const int sbits = bits_for((uint64_t)S);
        k_move_keys<<<gs, kBlock, 0, s>>>(s_best, S, sbits, mk, d_cnt + 1);
        uint32_t nm = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nm, d_cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        if (nm > 0) {
            const int nbits = sbits + bits_for((uint64_t)ncl);
            uint64_t* sorted = radix_sort_u64(mk, malt, nm, nbits, rtmp, s);
            k_apply_parallel<<<grid_for(nm, kBlock), kBlock, 0, s>>>(st, sorted, nm, sbits, s_vertex, err);
            g->launches += 1 + 3 * ((nbits + 7) / 8);
        }
        k_mark_moved<<<gs, kBlock, 0, s>>>(s_best, s_vertex, S, moved);
        g->launches += 2;
    }

    // new membership, statistics, scores
    int64_t* nsz = ncap;  // capacities are no longer needed
    k_new_sizes<<<gk, kBlock, 0, s>>>(st, g->cl_off, g->cl_vert, ncl, moved, nsz);
    exclusive_scan_i64(nsz, g->x_off, ncl, g->x_off + ncl, ltmp, s);
    RTR_CUDA_TRY(cudaMemsetAsync(g->x_cof, 0xff, sizeof(int32_t) * (n + 1), s));
    k_emit<<<gk, kBlock, 0, s>>>(st, g->cl_off, g->cl_vert, ncl, g->x_off, g->x_vert, g->x_cof);
    RTR_CUDA_TRY(cudaMemsetAsync(g->x_ne, 0, sizeof(int64_t) * (ncl + 1), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->x_cut, 0, sizeof(int64_t) * (ncl + 1), s));
    k_expand_stats<<<gn, kBlock, 0, s>>>(g->offsets, g->nbors, n, g->x_cof, (unsigned long long*)g->x_ne,
                                         (unsigned long long*)g->x_cut);
    k_halve_ne<<<gk, kBlock, 0, s>>>(g->x_ne, ncl);
    uint32_t* m32 = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* mpos = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    if (!mpos || !m32) {
        set_error("device allocation failed (expand scores)");
        return RTR_ERR_CUDA;
    }
    k_u8_to_u32<<<gn, kBlock, 0, s>>>(moved, n, m32);
    exclusive_scan_u32(m32, mpos, n, d_cnt + 2, utmp, s);
    k_scores<<<gn, kBlock, 0, s>>>(moved, mpos, n, vs, s_score, g->x_scv, g->x_scx);
    g->launches += 12;
    RTR_CUDA_TRY(cudaGetLastError());
    uint32_t nsc = 0;
    unsigned long long errw = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nsc, d_cnt + 2, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(&errw, g->ctr + 1, sizeof(errw), cudaMemcpyDeviceToHost, s));
    cudaEventRecord(e1, s);
    RTR_CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&g->ms_expand, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (errw) {
        set_error("expand kernel reported an internal inconsistency (0x%llx)", errw);
        return RTR_ERR_DEVICE;
    }
    g->x_nscores = nsc;
    g->x_threshold = threshold;
    g->expanded = true;
    return RTR_OK;
}

}  // namespace rtr
