// List-free weighted triangle counting ("rows" layout): perVertex and the
// perEdge of heavy edges folded straight from the CSR rows, with no
// per-triangle storage, for graphs whose triangle lists do not fit in HBM
// (R-MAT scale 22 already has 2.1 G triangles, i.e. ~200 GB of lists; scale 24
// 10.3 G).  commonNbr itself keeps no lists either
// (RTRex_Sequential/Escape/Decomposition.h:70-115): it re-intersects rows.
//
// What runs before this (count.cu): k_edge_fold folds perEdge for every light
// edge (deg u + deg v below the heavy-edge threshold) and k_edge_count_heavy
// counts the heavy ones, so support, the triangle total and light perEdge are
// known.  This file adds, bit-exact to commonNbr's discovery order:
//   perVertex[x] = left fold over y in N(x) ascending, then over
//                  z in N(x) & N(y), z > y ascending, of 1/double(dx*dy*dz)
//   perEdge[(x,y)] for heavy edges, x < y = left fold over z in N(x) & N(y)
//                  ascending, computed by x's pass from the same intersection.
// For y > x owning a heavy edge the pass intersects the full rows (perEdge
// needs every z; the z > y suffix continues perVertex[x]); otherwise it
// intersects N(x) beyond y with N(y).  Every intersection walks the shorter
// range in ascending order and looks its elements up in the longer row: in that
// row's hash set when it has one (rowsets.cuh; build_row_sets below makes one
// for every row of at least kSetDegree entries), else by binary search.
//
// Three kernels by the degree of x:
//   k_rows_light   a thread per vertex of degree < light
//   k_rows_medium  a warp per vertex of degree in [light, hub): for each y in
//                  turn the warp walks the shorter range 32 elements at a time
//                  and folds the hits in lane order (ascending z)
//   k_rows_hub     a thread block per vertex of degree >= hub, hubs in
//                  descending degree, two blocks per SM: 7 producer warps take
//                  7 consecutive y at once, each writing its y's z > y weights,
//                  in order, to its own buffer, which warp 0 folds in y order
//                  while the producers work on the next 7 (double-buffered) --
//                  only the perVertex chain itself is sequential.
// The hub kernel runs on the graph's second stream, concurrently with the
// other two (it holds the longest dependent chain: ~10^8 adds for the largest
// R-MAT scale-24 hub).
#include "intersect.cuh"
#include "primitives.cuh"
#include "rowsets.cuh"
#include "rtr_graph.cuh"

namespace rtr {

namespace {

constexpr int kLightBlock = 256;
constexpr int kMediumBlock = 128;
constexpr int kHubWarps = 8;
constexpr int kHubBlock = 32 * kHubWarps;

struct RowsArgs {
    const int64_t* off;
    const int32_t* nb;
    const int32_t* deg;
    int64_t n;
    double* pe;
    double* pv;
    int gallop;
    int heavy_edge;  // deg x + deg y from which perEdge is folded here (k_edge_fold left it)
    int light;       // vertices below this degree: a thread
    int hub;         // vertices from this degree: a thread block
    RowSets rs;
};

__device__ __forceinline__ bool owns_heavy(const RowsArgs& a, int32_t x, int32_t y, int dx, int dy)
{
    return x < y && dx + dy >= a.heavy_edge;
}

// The warp's hits of the ascending range S = [s0, s1) in the range [l0, l1) of
// row w: chunk(hit, z) per 32 elements of S, hits ascending.  Through w's hash
// set when it has one -- exact because every caller passes either w's whole
// row, or x's row cut just after y together with an S whose elements all
// exceed y -- else by binary search.
template <typename F>
__device__ __forceinline__ void warp_hits(const RowsArgs& a, int64_t s0, int64_t s1, int32_t w, int64_t l0,
                                          int64_t l1, int lane, F&& chunk)
{
    const int32_t t = rs_table(a.rs, w);
    if (t >= 0) {
        const int32_t zmax = a.nb[a.off[w + 1] - 1];
        warp_scan(a.nb, s0, s1, zmax, lane, [&](int32_t z) { return rs_member(a.rs, t, z); }, chunk);
    } else {
        warp_chunks(a.nb, s0, s1, l0, l1, lane,
                    [&](int64_t lo, int64_t hi, int32_t v) { return lower_bound_row(a.nb, lo, hi, v); }, chunk);
    }
}

__global__ void __launch_bounds__(kLightBlock) k_rows_light(RowsArgs a)
{
    for (int64_t xi = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; xi < a.n;
         xi += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = (int32_t)xi;
        const int dx = a.deg[x];
        if (dx >= a.light) continue;
        const int64_t a0 = a.off[x], a1 = a.off[x + 1];
        double pvacc = 0.0;
        for (int64_t i = a0; i < a1; ++i) {
            const int32_t y = a.nb[i];
            const int dy = a.deg[y];
            const int64_t dxy = (int64_t)dx * (int64_t)dy;
            const int64_t b0 = a.off[y], b1 = a.off[y + 1];
            const int32_t ty = rs_table(a.rs, y);  // x is light: its row is the one walked
            // common neighbours of x's range [s0, a1) and y's row, ascending: f(z)
            auto each = [&](int64_t s0, auto&& f) {
                if (ty >= 0) {
                    for (int64_t p = s0; p < a1; ++p) {
                        const int32_t z = a.nb[p];
                        if (rs_member(a.rs, ty, z)) f(z);
                    }
                } else {
                    intersect_rows(a.nb, s0, a1, b0, b1, a.gallop, [&](int32_t z, int64_t, int64_t) { f(z); });
                }
            };
            if (owns_heavy(a, x, y, dx, dy)) {
                double peacc = 0.0;
                each(a0, [&](int32_t z) {
                    const double w = 1.0 / (double)(dxy * (int64_t)a.deg[z]);
                    peacc += w;
                    if (z > y) pvacc += w;
                });
                a.pe[i] = peacc;
            } else {
                each(i + 1, [&](int32_t z) { pvacc += 1.0 / (double)(dxy * (int64_t)a.deg[z]); });
            }
        }
        a.pv[x] = pvacc;
    }
}

__global__ void __launch_bounds__(kMediumBlock) k_rows_medium(RowsArgs a)
{
    __shared__ double s_w[kMediumBlock / 32][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * (kMediumBlock / 32);
    for (int64_t xi = (int64_t)blockIdx.x * (kMediumBlock / 32) + wib; xi < a.n; xi += nwarps) {
        const int32_t x = (int32_t)xi;
        const int dx = a.deg[x];
        if (dx < a.light || dx >= a.hub) continue;  // uniform across the warp
        const int64_t a0 = a.off[x], a1 = a.off[x + 1];
        double pvacc = 0.0;
        for (int64_t i = a0; i < a1; ++i) {
            const int32_t y = a.nb[i];
            const int dy = a.deg[y];
            const int64_t dxy = (int64_t)dx * (int64_t)dy;
            const bool owner = owns_heavy(a, x, y, dx, dy);
            const int64_t A0 = owner ? a0 : i + 1, A1 = a1;
            int64_t B0 = a.off[y];
            const int64_t B1 = a.off[y + 1];
            if (!owner && B1 - B0 <= A1 - A0) B0 = lower_bound_row(a.nb, B0, B1, y + 1);  // A holds only z > y
            double peacc = 0.0;
            auto chunk = [&](bool hit, int32_t z) {
                const double w = hit ? 1.0 / (double)(dxy * (int64_t)a.deg[z]) : 0.0;
                const int below = owner ? __popc(__ballot_sync(0xffffffffu, hit && z < y)) : 0;
                fold_hits(hit, w, s_w[wib], lane, owner ? &peacc : nullptr, &pvacc, below);
            };
            if (A1 - A0 <= B1 - B0) warp_hits(a, A0, A1, y, B0, B1, lane, chunk);
            else warp_hits(a, B0, B1, x, A0, A1, lane, chunk);
            if (owner && lane == 0) a.pe[i] = peacc;
        }
        if (lane == 0) a.pv[x] = pvacc;
    }
}

// Hubs: hubs[] in descending degree.  Warp 0 of the block folds perVertex;
// warps 1..kHubWarps-1 produce: round r gives them the next kHubWarps-1
// consecutive y, each writing its y's z > y weights in order to its own region
// of buffer set r&1 (buf holds 2 x (kHubWarps-1) regions of cap doubles per
// block; cap >= the largest hub degree bounds the hits of one y), while warp 0
// folds round r-1 from the other set.  One block barrier per round.
__global__ void __launch_bounds__(kHubBlock, 2) k_rows_hub(RowsArgs a, const int32_t* __restrict__ hubs,
                                                            int64_t nhub, double* __restrict__ buf, int64_t cap)
{
    constexpr int P = kHubWarps - 1;  // producer warps
    __shared__ double s_w[kHubWarps][32];
    __shared__ int64_t s_len[2][P];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    auto region = [&](int set, int w) { return buf + (((int64_t)blockIdx.x * 2 + set) * P + w) * cap; };
    for (int64_t h = blockIdx.x; h < nhub; h += gridDim.x) {
        const int32_t x = hubs[h];
        const int dx = a.deg[x];
        const int64_t a0 = a.off[x], a1 = a.off[x + 1], d = a1 - a0;
        // producer warp w (1..P) on slot i: y's z > y weights into region(set, w-1)
        auto produce = [&](int64_t i, int set) {
            int64_t len = 0;
            double* reg = region(set, wib - 1);
            if (i < a1) {  // uniform across the warp
                const int32_t y = a.nb[i];
                const int dy = a.deg[y];
                const int64_t dxy = (int64_t)dx * (int64_t)dy;
                const bool owner = owns_heavy(a, x, y, dx, dy);
                const int64_t A0 = owner ? a0 : i + 1, A1 = a1;
                int64_t B0 = a.off[y];
                const int64_t B1 = a.off[y + 1];
                double peacc = 0.0;
                auto chunk = [&](bool hit, int32_t z) {
                    const unsigned mask = __ballot_sync(0xffffffffu, hit);
                    const int cnt = __popc(mask);
                    if (cnt == 0) return;
                    const double w = hit ? 1.0 / (double)(dxy * (int64_t)a.deg[z]) : 0.0;
                    const int below = owner ? __popc(__ballot_sync(0xffffffffu, hit && z < y)) : 0;
                    const int rank = __popc(mask & ((1u << lane) - 1u));
                    if (owner) fold_hits(hit, w, s_w[wib], lane, &peacc, nullptr, 0);
                    if (hit && rank >= below) reg[len + rank - below] = w;
                    len += cnt - below;
                };
                if (B1 - B0 <= A1 - A0) {
                    if (!owner) B0 = lower_bound_row(a.nb, B0, B1, y + 1);  // A holds only z > y
                    warp_hits(a, B0, B1, x, A0, A1, lane, chunk);
                } else {
                    warp_hits(a, A0, A1, y, B0, B1, lane, chunk);
                }
                if (owner && lane == 0) a.pe[i] = peacc;
            }
            if (lane == 0) s_len[set][wib - 1] = len;
        };
        double pvacc = 0.0;  // meaningful in warp 0
        const int64_t rounds = (d + P - 1) / P;
        if (wib > 0) produce(a0 + wib - 1, 0);
        __syncthreads();
        for (int64_t r = 0; r < rounds; ++r) {
            const int set = (int)(r & 1);
            if (wib == 0) {
                for (int w = 0; w < P; ++w) {
                    const int64_t L = s_len[set][w];
                    const double* rg = region(set, w);
                    double v = lane < L ? rg[lane] : 0.0;
                    for (int64_t k0 = 0; k0 < L; k0 += 32) {
                        const double vn = k0 + 32 + lane < L ? rg[k0 + 32 + lane] : 0.0;  // next 32, ahead of the chain
                        const int c = L - k0 < 32 ? (int)(L - k0) : 32;
#pragma unroll
                        for (int j = 0; j < 32; ++j) {
                            const double t = __shfl_sync(0xffffffffu, v, j);
                            if (j < c) pvacc += t;
                        }
                        v = vn;
                    }
                }
            } else if (r + 1 < rounds) {
                produce(a0 + (r + 1) * P + wib - 1, set ^ 1);
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) a.pv[x] = pvacc;
        __syncthreads();
    }
}

__global__ void k_hub_keys(const int32_t* __restrict__ deg, int64_t n, int hub, uint64_t* __restrict__ keys,
                           unsigned* __restrict__ nh)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        if (deg[v] >= hub)
            keys[atomicAdd(nh, 1u)] = ((uint64_t)(0x7fffffff - deg[v]) << 32) | (uint64_t)v;
}

__global__ void k_hub_ids(const uint64_t* __restrict__ keys, int64_t nh, int32_t* __restrict__ ids)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nh; i += (int64_t)gridDim.x * blockDim.x)
        ids[i] = (int32_t)(keys[i] & 0xffffffffu);
}

// Row sets: the vertices of at least min_deg neighbours, numbered in id order
// (flag + scan), each with a power-of-two table of >= 2 deg slots.
__global__ void k_rs_flags(const int32_t* __restrict__ deg, int64_t n, int min_deg, int64_t* __restrict__ flag)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= n; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = (v < n && deg[v] >= min_deg) ? 1 : 0;
}

__global__ void k_rs_sizes(const int32_t* __restrict__ deg, int64_t n, const int64_t* __restrict__ num,
                           int32_t* __restrict__ tab, int32_t* __restrict__ owner, int32_t* __restrict__ tbits,
                           int64_t* __restrict__ tsize)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (num[v + 1] == num[v]) {
            tab[v] = -1;
            continue;
        }
        const int32_t t = (int32_t)num[v];
        int bits = 1;
        while ((1ll << bits) < 2ll * deg[v]) ++bits;
        tab[v] = t;
        owner[t] = (int32_t)v;
        tbits[t] = bits;
        tsize[t] = 1ll << bits;
    }
}

// A warp per table (dealt modulo the warp count) inserts its row; the table
// is at least half empty, so every probe sequence meets an empty slot.
__global__ void k_rs_insert(const int32_t* __restrict__ owner, int64_t nt, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ nb, const int64_t* __restrict__ toff,
                            const int32_t* __restrict__ tbits, int32_t* __restrict__ slot)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; t < nt; t += nwarps) {
        const int32_t v = owner[t];
        const int bits = tbits[t];
        const uint32_t mask = (1u << bits) - 1u;
        int32_t* tb = slot + toff[t];
        for (int64_t p = off[v] + lane; p < off[v + 1]; p += 32) {
            const int32_t z = nb[p];
            uint32_t h = rs_hash(z, bits);
            while (atomicCAS(&tb[h], -1, z) != -1) h = (h + 1u) & mask;
        }
    }
}

}  // namespace

// Hash sets of every row of at least min_deg entries, in scratch (live until
// sc is released); *out stays empty when no row qualifies.
int build_row_sets(rtr_graph* g, Scratch& sc, int min_deg, RowSets* out)
{
    *out = RowSets{nullptr, nullptr, nullptr, nullptr};
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    int64_t* flag = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    int64_t* num = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    int64_t* tmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(n + 1));
    int32_t* tab = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    if (!flag || !num || !tmp || !tab) {
        set_error("device allocation failed (row sets)");
        return RTR_ERR_CUDA;
    }
    k_rs_flags<<<grid_for(n + 1, 256), 256, 0, s>>>(g->deg, n, min_deg, flag);
    exclusive_scan_i64(flag, num, n + 1, nullptr, tmp, s);
    int64_t nt = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nt, num + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->launches += 2;
    if (nt == 0) return RTR_OK;
    int32_t* owner = (int32_t*)sc.get(sizeof(int32_t) * (nt + 1));
    int32_t* tbits = (int32_t*)sc.get(sizeof(int32_t) * (nt + 1));
    int64_t* tsize = (int64_t*)sc.get(sizeof(int64_t) * (nt + 1));
    int64_t* toff = (int64_t*)sc.get(sizeof(int64_t) * (nt + 1));
    int64_t* ltmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nt + 1));
    if (!owner || !tbits || !tsize || !toff || !ltmp) {
        set_error("device allocation failed (row sets)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(tsize + nt, 0, sizeof(int64_t), s));
    k_rs_sizes<<<grid_for(n, 256), 256, 0, s>>>(g->deg, n, num, tab, owner, tbits, tsize);
    exclusive_scan_i64(tsize, toff, nt + 1, nullptr, ltmp, s);
    int64_t total = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&total, toff + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    int32_t* slot = (int32_t*)sc.get(sizeof(int32_t) * (total + 1));
    if (!slot) {
        set_error("device allocation failed (row sets: %lld slots)", (long long)total);
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(slot, 0xff, sizeof(int32_t) * (total + 1), s));
    k_rs_insert<<<grid_for(1ll << 40, 256, 8), 256, 0, s>>>(owner, nt, g->offsets, g->nbors, toff, tbits, slot);
    g->launches += 3;
    RTR_CUDA_TRY(cudaGetLastError());
    *out = RowSets{tab, toff, tbits, slot};
    return RTR_OK;
}

// perVertex (all vertices) and heavy-edge perEdge from the rows; the caller has
// run the edge fold and heavy-edge count.  Synchronises the graph's stream.
int count_rows(rtr_graph* g, Scratch& sc, const RowSets& rs)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    RowsArgs a{g->offsets, g->nbors, g->deg, n, g->pe, g->pv, g->tune_gallop, g->tune_edge, g->tune_heavy,
               g->count_hub, rs};
    if (a.hub < a.light) a.hub = a.light;
    uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    unsigned* d_nh = (unsigned*)sc.get(sizeof(unsigned) * 2);
    if (!keys || !alt || !d_nh) {
        set_error("device allocation failed (hub list)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(d_nh, 0, sizeof(unsigned), s));
    k_hub_keys<<<grid_for(n, 256), 256, 0, s>>>(g->deg, n, a.hub, keys, d_nh);
    unsigned nh = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nh, d_nh, sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->launches += 1;
    int32_t* hubs = nullptr;
    double* hbuf = nullptr;
    int64_t cap = 0;
    int hub_grid = 0;
    if (nh > 0) {
        void* rtmp = sc.get(radix_temp_bytes(nh));
        hubs = (int32_t*)sc.get(sizeof(int32_t) * (nh + 1));
        if (!rtmp || !hubs) {
            set_error("device allocation failed (hub list)");
            return RTR_ERR_CUDA;
        }
        uint64_t* sorted = radix_sort_u64(keys, alt, nh, 64, rtmp, s);
        uint64_t first = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&first, sorted, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        k_hub_ids<<<grid_for(nh, 256), 256, 0, s>>>(sorted, nh, hubs);
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        g->launches += 1 + 3 * 8;
        cap = (int64_t)(0x7fffffff - (int64_t)(first >> 32));  // the largest hub degree
        int dev_sms = 148;
        cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, g->device);
        const int64_t want = 2ll * dev_sms;  // two hub blocks per SM
        hub_grid = (int)((int64_t)nh < want ? (int64_t)nh : want);
        hbuf = (double*)sc.get(sizeof(double) * (size_t)hub_grid * 2 * (kHubWarps - 1) * (size_t)(cap + 32));
        if (!hbuf) {
            set_error("device allocation failed (hub fold buffers, %lld hubs of degree up to %lld)", (long long)nh,
                      (long long)cap);
            return RTR_ERR_CUDA;
        }
        cap += 32;
    }
    cudaEvent_t ready = nullptr, joined = nullptr;
    if (hub_grid > 0) {
        if (!g->side) RTR_CUDA_TRY(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
        RTR_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        RTR_CUDA_TRY(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
        RTR_CUDA_TRY(cudaEventRecord(ready, s));
        RTR_CUDA_TRY(cudaStreamWaitEvent(g->side, ready, 0));
        ktime_begin(g, KT_ROWS_HUB, g->side);
        k_rows_hub<<<hub_grid, kHubBlock, 0, g->side>>>(a, hubs, nh, hbuf, cap);
        ktime_end(g, KT_ROWS_HUB, g->side);
        RTR_CUDA_TRY(cudaEventRecord(joined, g->side));
        g->launches += 1;
    }
    ktime_begin(g, KT_ROWS_LIGHT);
    k_rows_light<<<grid_for(n, kLightBlock), kLightBlock, 0, s>>>(a);
    ktime_end(g, KT_ROWS_LIGHT);
    ktime_begin(g, KT_ROWS_MEDIUM);
    k_rows_medium<<<grid_for(1ll << 40, kMediumBlock, 16), kMediumBlock, 0, s>>>(a);
    ktime_end(g, KT_ROWS_MEDIUM);
    g->launches += 2;
    cudaError_t e = cudaGetLastError();
    if (joined) {
        cudaStreamWaitEvent(s, joined, 0);
        cudaStreamSynchronize(s);  // scratch (hub list, buffers) is freed on return
        cudaEventDestroy(ready);
        cudaEventDestroy(joined);
        ktime_read(g, KT_ROWS_HUB);
    } else {
        g->kms[KT_ROWS_HUB] = 0;
    }
    cudaStreamSynchronize(s);
    ktime_read(g, KT_ROWS_LIGHT);
    ktime_read(g, KT_ROWS_MEDIUM);
    if (e != cudaSuccess) return cuda_fail(e, "rows-layout counting launch", __FILE__, __LINE__);
    return RTR_OK;
}

}  // namespace rtr
