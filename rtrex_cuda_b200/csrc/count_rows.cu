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
// intersects N(x) beyond y with N(y).
//
// Three kernels by the degree of x:
//   k_rows_light   a thread per vertex of degree < light (merge / gallop)
//   k_rows_medium  a warp per vertex of degree in [light, hub): for each y in
//                  turn the warp walks the shorter row 32 elements at a time,
//                  every lane binary-searching its element in the longer one,
//                  and folds the hits in lane order (ascending z)
//   k_rows_hub     a thread block per vertex of degree >= hub, hubs in
//                  descending degree: 7 producer warps take 7 consecutive y at
//                  once, searching x's row through a shared-memory sample of it
//                  (every stride-th element) and a one-window global search;
//                  each writes its y's z > y weights, in order, to its own
//                  buffer, which warp 0 folds in y order while the producers
//                  work on the next 7 (double-buffered) -- only the perVertex
//                  chain itself is sequential.
// The hub kernel runs on the graph's second stream, concurrently with the
// other two (it holds the longest dependent chain: ~10^8 adds for the largest
// R-MAT scale-24 hub).
#include "intersect.cuh"
#include "primitives.cuh"
#include "rtr_graph.cuh"

namespace rtr {

namespace {

constexpr int kLightBlock = 256;
constexpr int kMediumBlock = 128;
constexpr int kHubWarps = 8;
constexpr int kHubBlock = 32 * kHubWarps;
constexpr int kHubIndexMax = 11264;  // sample entries of a hub row in shared memory (44 KB, static limit 48 KB)

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
    // every kIdxStride-th neighbour of each hub (hub_pos[v]: v's place in the hub
    // list, -1 for the others), so that a lookup in a hub's long row searches
    // this compact array and then a single window of the row
    const int32_t* hub_pos;
    const int64_t* idx_off;
    const int32_t* idx;
};

constexpr int kIdxStride = 32;

// Lower bound of v in the row of y (the range [lo, hi) of the caller is y's
// whole row): through y's sample index when y is a hub.  A search that the
// index places before lo returns that position; the callers only count hits at
// or after lo.
__device__ __forceinline__ int64_t row_lower_bound(const RowsArgs& a, int32_t y, int64_t lo, int64_t hi, int32_t v)
{
    const int32_t h = a.hub_pos ? a.hub_pos[y] : -1;
    if (h < 0) return lower_bound_row(a.nb, lo, hi, v);
    const int64_t s0 = a.idx_off[h], s1 = a.idx_off[h + 1];
    int64_t l = s0, r = s1;  // first sample above v
    while (l < r) {
        const int64_t mid = (l + r) >> 1;
        if (a.idx[mid] <= v) l = mid + 1;
        else r = mid;
    }
    const int64_t base = a.off[y], end = a.off[y + 1];
    if (l == s0) return base;
    const int64_t w0 = base + (l - 1 - s0) * kIdxStride;
    const int64_t w1 = w0 + kIdxStride < end ? w0 + kIdxStride : end;
    return lower_bound_row(a.nb, w0, w1, v);
}

// Common neighbours of the short ascending range [s0, s1) and hub y's row, in
// ascending order: f(z).  One thread.
template <typename F>
__device__ __forceinline__ void intersect_with_hub(const RowsArgs& a, int64_t s0, int64_t s1, int32_t y, F&& f)
{
    const int64_t b0 = a.off[y], b1 = a.off[y + 1];
    for (int64_t p = s0; p < s1; ++p) {
        const int32_t x = a.nb[p];
        const int64_t pos = row_lower_bound(a, y, b0, b1, x);
        if (pos < b1 && a.nb[pos] == x) f(x);
    }
}

__device__ __forceinline__ bool owns_heavy(const RowsArgs& a, int32_t x, int32_t y, int dx, int dy)
{
    return x < y && dx + dy >= a.heavy_edge;
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
            const bool y_hub = a.hub_pos && a.hub_pos[y] >= 0;  // x is light: its row is the short one
            if (owns_heavy(a, x, y, dx, dy)) {
                double peacc = 0.0;
                auto f = [&](int32_t z) {
                    const double w = 1.0 / (double)(dxy * (int64_t)a.deg[z]);
                    peacc += w;
                    if (z > y) pvacc += w;
                };
                if (y_hub) intersect_with_hub(a, a0, a1, y, f);
                else intersect_rows(a.nb, a0, a1, b0, b1, a.gallop, [&](int32_t z, int64_t, int64_t) { f(z); });
                a.pe[i] = peacc;
            } else {
                auto f = [&](int32_t z) { pvacc += 1.0 / (double)(dxy * (int64_t)a.deg[z]); };
                if (y_hub) intersect_with_hub(a, i + 1, a1, y, f);
                else intersect_rows(a.nb, i + 1, a1, b0, b1, a.gallop, [&](int32_t z, int64_t, int64_t) { f(z); });
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
    auto search = [&](int64_t lo, int64_t hi, int32_t v) { return lower_bound_row(a.nb, lo, hi, v); };
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
            // A shorter: y's whole row is searched (through its index when y is a hub)
            auto search_y = [&](int64_t lo, int64_t hi, int32_t v) { return row_lower_bound(a, y, lo, hi, v); };
            if (A1 - A0 <= B1 - B0) warp_chunks(a.nb, A0, A1, B0, B1, lane, search_y, chunk);
            else warp_chunks(a.nb, B0, B1, A0, A1, lane, search, chunk);
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
__global__ void __launch_bounds__(kHubBlock) k_rows_hub(RowsArgs a, const int32_t* __restrict__ hubs, int64_t nhub,
                                                         double* __restrict__ buf, int64_t cap)
{
    constexpr int P = kHubWarps - 1;  // producer warps
    __shared__ int32_t s_idx[kHubIndexMax];
    __shared__ double s_w[kHubWarps][32];
    __shared__ int64_t s_len[2][P];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    auto region = [&](int set, int w) { return buf + (((int64_t)blockIdx.x * 2 + set) * P + w) * cap; };
    for (int64_t h = blockIdx.x; h < nhub; h += gridDim.x) {
        const int32_t x = hubs[h];
        const int dx = a.deg[x];
        const int64_t a0 = a.off[x], a1 = a.off[x + 1], d = a1 - a0;
        int64_t stride = (d + kHubIndexMax - 1) / kHubIndexMax;
        if (stride < 32) stride = 32;
        const int K = (int)((d + stride - 1) / stride);
        for (int k = threadIdx.x; k < K; k += kHubBlock) s_idx[k] = a.nb[a0 + (int64_t)k * stride];
        __syncthreads();
        // lower bound of v in x's whole row: the sample narrows it to one window
        auto search_x = [&](int64_t, int64_t, int32_t v) -> int64_t {
            int lo = 0, hi = K;  // first sample above v
            while (lo < hi) {
                const int mid = (lo + hi) >> 1;
                if (s_idx[mid] <= v) lo = mid + 1;
                else hi = mid;
            }
            if (lo == 0) return a0;
            const int64_t w0 = a0 + (int64_t)(lo - 1) * stride;
            const int64_t w1 = w0 + stride < a1 ? w0 + stride : a1;
            return lower_bound_row(a.nb, w0, w1, v);
        };
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
                    warp_chunks(a.nb, B0, B1, A0, A1, lane, search_x, chunk);
                } else {
                    auto search_y = [&](int64_t lo, int64_t hi, int32_t v) { return row_lower_bound(a, y, lo, hi, v); };
                    warp_chunks(a.nb, A0, A1, B0, B1, lane, search_y, chunk);
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
                        double t[32];
#pragma unroll
                        for (int j = 0; j < 32; ++j) t[j] = __shfl_sync(0xffffffffu, v, j);
#pragma unroll
                        for (int j = 0; j < 32; ++j)
                            if (j < c) pvacc += t[j];
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

__global__ void k_hub_index_sizes(const int32_t* __restrict__ hubs, int64_t nh, const int32_t* __restrict__ deg,
                                  int32_t* __restrict__ hub_pos, int64_t* __restrict__ cnt)
{
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h <= nh; h += (int64_t)gridDim.x * blockDim.x) {
        if (h == nh) {
            cnt[h] = 0;
            continue;
        }
        hub_pos[hubs[h]] = (int32_t)h;
        cnt[h] = (deg[hubs[h]] + kIdxStride - 1) / kIdxStride;
    }
}

// A warp per hub (dealt modulo the warp count): sample k of hub h is its row's entry kIdxStride*k.
__global__ void k_hub_index_fill(const int32_t* __restrict__ hubs, int64_t nh, const int64_t* __restrict__ off,
                                 const int32_t* __restrict__ nb, const int64_t* __restrict__ ioff,
                                 int32_t* __restrict__ idx)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t h = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; h < nh; h += nwarps) {
        const int64_t x = hubs[h], base = off[x];
        const int64_t cnt = ioff[h + 1] - ioff[h];
        for (int64_t k = lane; k < cnt; k += 32) idx[ioff[h] + k] = nb[base + k * kIdxStride];
    }
}

__global__ void k_hub_ids(const uint64_t* __restrict__ keys, int64_t nh, int32_t* __restrict__ ids)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nh; i += (int64_t)gridDim.x * blockDim.x)
        ids[i] = (int32_t)(keys[i] & 0xffffffffu);
}

}  // namespace

// perVertex (all vertices) and heavy-edge perEdge from the rows; the caller has
// run the edge fold and heavy-edge count.  Synchronises the graph's stream.
int count_rows(rtr_graph* g, Scratch& sc)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    RowsArgs a{g->offsets, g->nbors, g->deg, n, g->pe, g->pv, g->tune_gallop, g->tune_edge, g->tune_heavy,
               g->count_hub, nullptr, nullptr, nullptr};
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
        hub_grid = (int)((int64_t)nh < dev_sms ? (int64_t)nh : dev_sms);
        hbuf = (double*)sc.get(sizeof(double) * (size_t)hub_grid * 2 * (kHubWarps - 1) * (size_t)(cap + 32));
        if (!hbuf) {
            set_error("device allocation failed (hub fold buffers, %lld hubs of degree up to %lld)", (long long)nh,
                      (long long)cap);
            return RTR_ERR_CUDA;
        }
        cap += 32;
        // the hubs' sample index
        int32_t* hub_pos = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
        int64_t* icnt = (int64_t*)sc.get(sizeof(int64_t) * (nh + 1));
        int64_t* ioff = (int64_t*)sc.get(sizeof(int64_t) * (nh + 1));
        int64_t* itmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nh + 1));
        int64_t* itot = (int64_t*)sc.get(sizeof(int64_t) * 2);
        if (!hub_pos || !icnt || !ioff || !itmp || !itot) {
            set_error("device allocation failed (hub index)");
            return RTR_ERR_CUDA;
        }
        RTR_CUDA_TRY(cudaMemsetAsync(hub_pos, 0xff, sizeof(int32_t) * (n + 1), s));
        k_hub_index_sizes<<<grid_for(nh, 256), 256, 0, s>>>(hubs, nh, g->deg, hub_pos, icnt);
        exclusive_scan_i64(icnt, ioff, nh + 1, itot, itmp, s);
        int64_t ntot = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&ntot, itot, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        int32_t* idx = (int32_t*)sc.get(sizeof(int32_t) * (ntot + 1));
        if (!idx) {
            set_error("device allocation failed (hub index)");
            return RTR_ERR_CUDA;
        }
        k_hub_index_fill<<<grid_for(1ll << 40, 256, 8), 256, 0, s>>>(hubs, nh, g->offsets, g->nbors, ioff, idx);
        g->launches += 5;
        a.hub_pos = hub_pos;
        a.idx_off = ioff;
        a.idx = idx;
    }
    cudaEvent_t ready = nullptr, joined = nullptr;
    if (hub_grid > 0) {
        if (!g->side) RTR_CUDA_TRY(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
        RTR_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
        RTR_CUDA_TRY(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
        RTR_CUDA_TRY(cudaEventRecord(ready, s));
        RTR_CUDA_TRY(cudaStreamWaitEvent(g->side, ready, 0));
        k_rows_hub<<<hub_grid, kHubBlock, 0, g->side>>>(a, hubs, nh, hbuf, cap);
        RTR_CUDA_TRY(cudaEventRecord(joined, g->side));
        g->launches += 1;
    }
    k_rows_light<<<grid_for(n, kLightBlock), kLightBlock, 0, s>>>(a);
    k_rows_medium<<<grid_for(1ll << 40, kMediumBlock, 16), kMediumBlock, 0, s>>>(a);
    g->launches += 2;
    cudaError_t e = cudaGetLastError();
    if (joined) {
        cudaStreamWaitEvent(s, joined, 0);
        cudaStreamSynchronize(s);  // scratch (hub list, buffers) is freed on return
        cudaEventDestroy(ready);
        cudaEventDestroy(joined);
    }
    if (e != cudaSuccess) return cuda_fail(e, "rows-layout counting launch", __FILE__, __LINE__);
    return RTR_OK;
}

}  // namespace rtr
