// C ABI of librtr.so (declared in include/rtr.h).
#include "../../include/rtr.h"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <cstdio>
#include <cstdlib>
#include <new>
#include <vector>

namespace rtr {
const char* last_error();
}

using namespace rtr;

namespace {

__global__ void k_expand_pe(const double* __restrict__ pe, const uint32_t* __restrict__ sup,
                            const uint8_t* __restrict__ st, const int32_t* __restrict__ esrc,
                            const int32_t* __restrict__ nb, const int32_t* __restrict__ partner, int64_t m2,
                            double* __restrict__ ope, uint32_t* __restrict__ osup, uint8_t* __restrict__ ost)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t f = (esrc[i] < nb[i]) ? i : (int64_t)partner[i];
        if (ope) ope[i] = pe[f];
        if (osup) osup[i] = sup[f];
        if (ost) ost[i] = st[f];
    }
}

// vbase[v] = first vertex id of v's graph (binary search over the batch bases).
__global__ void k_fill_vbase(const int64_t* __restrict__ bases, int64_t K, int64_t n, int32_t* __restrict__ vbase)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t lo = 0, hi = K;  // largest k with bases[k] <= v
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (bases[mid] <= v) lo = mid;
            else hi = mid;
        }
        vbase[v] = (int32_t)bases[lo];
    }
}

__global__ void k_widen32(const int32_t* __restrict__ in, int64_t* __restrict__ out, int64_t k)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < k; i += (int64_t)gridDim.x * blockDim.x)
        out[i] = in[i];
}

int make_graph(int64_t n, int device, rtr_graph** out)
{
    if (!out) {
        set_error("null output pointer");
        return RTR_ERR_ARG;
    }
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        set_error("no CUDA device is visible (librtr has no CPU path)");
        return RTR_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) {
        set_error("device %d out of range (%d devices)", device, ndev);
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(device));
    rtr_graph* g = new (std::nothrow) rtr_graph();
    if (!g) {
        set_error("host allocation failed");
        return RTR_ERR_ARG;
    }
    g->device = device;
    g->n = n;
    if (cudaStreamCreateWithFlags(&g->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete g;
        set_error("cudaStreamCreate failed");
        return RTR_ERR_CUDA;
    }
    g->own_stream = true;
    for (int k = 0; k < 2 * rtr_graph::kTimers; ++k) cudaEventCreate(&g->kev[k]);
    {
        // keep freed blocks cached in the device pool between graphs
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            uint64_t thr = ~0ull;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    g->ctr = (unsigned long long*)dev_alloc(g, 8 * sizeof(unsigned long long));
    if (!g->ctr) {
        rtr_graph_destroy(g);
        set_error("device allocation failed");
        return RTR_ERR_CUDA;
    }
    *out = g;
    return RTR_OK;
}

// Typed D2H copy of the first k device int32 values widened to int64.
int copy_i32_as_i64(rtr_graph* g, const int32_t* d, int64_t k, int64_t* h)
{
    if (k <= 0) return RTR_OK;
    Scratch sc(g);
    int64_t* w = (int64_t*)sc.get(sizeof(int64_t) * k);
    if (!w) {
        set_error("device allocation failed");
        return RTR_ERR_CUDA;
    }
    k_widen32<<<grid_for(k, 256), 256, 0, g->stream>>>(d, w, k);
    RTR_CUDA_TRY(cudaMemcpyAsync(h, w, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, g->stream));
    RTR_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return RTR_OK;
}

}  // namespace

namespace rtr {
int make_graph_handle(int64_t n, int device, rtr_graph** out) { return make_graph(n, device, out); }
}  // namespace rtr

extern "C" {

const char* rtr_version(void) { return "rtrex-b200 0.1 (sm_100a)"; }

const char* rtr_last_error(void) { return last_error(); }

int rtr_graph_create_from_edges(const int64_t* src, const int64_t* dst, int64_t m, int64_t n, int device, int flags,
                                rtr_graph** out)
{
    if ((!src || !dst) && m > 0) {
        set_error("null edge arrays");
        return RTR_ERR_ARG;
    }
    int rc = make_graph(n, device, out);
    if (rc) return rc;
    rtr_graph* g = *out;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, g->stream);
    {
        Scratch sc(g);
        int64_t* du = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
        int64_t* dv = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
        if (!du || !dv) {
            set_error("device allocation failed for %lld edges", (long long)m);
            rc = RTR_ERR_CUDA;
        } else {
            if (m > 0) {
                cudaMemcpyAsync(du, src, sizeof(int64_t) * m, cudaMemcpyHostToDevice, g->stream);
                cudaMemcpyAsync(dv, dst, sizeof(int64_t) * m, cudaMemcpyHostToDevice, g->stream);
            }
            rc = build_csr(g, du, dv, m, (flags & RTR_FLAG_SIMPLIFY) != 0);
        }
    }
    cudaEventRecord(e1, g->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&g->ms_build, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        rtr_graph_destroy(g);
        *out = nullptr;
    }
    return rc;
}

// Escape text -> device parse -> device CSR, without host edge arrays.
static int create_from_escape(const char* h_text, FILE* f, int64_t len, const char* what, int device, int flags,
                              rtr_graph** out)
{
    int rc = make_graph(0, device, out);
    if (rc) return rc;
    rtr_graph* g = *out;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, g->stream);
    {
        Scratch sc(g);
        int64_t n = 0, m = 0;
        int64_t *du = nullptr, *dv = nullptr;
        rc = parse_escape_device(g, sc, h_text, f, len, what, &n, &m, &du, &dv);
        if (!rc) {
            g->n = n;
            rc = build_csr(g, du, dv, m, (flags & RTR_FLAG_SIMPLIFY) != 0);
        }
    }
    cudaEventRecord(e1, g->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&g->ms_build, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        rtr_graph_destroy(g);
        *out = nullptr;
    }
    return rc;
}

int rtr_graph_create_from_escape_text(const char* text, int64_t len, int device, int flags, rtr_graph** out)
{
    if (!out || (!text && len > 0) || len < 0) {
        set_error("null or negative arguments");
        return RTR_ERR_ARG;
    }
    return create_from_escape(text ? text : "", nullptr, len, "escape text", device, flags, out);
}

int rtr_graph_create_from_escape_file(const char* path, int device, int flags, rtr_graph** out)
{
    if (!path || !out) {
        set_error("null argument");
        return RTR_ERR_ARG;
    }
    *out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) {
        set_error("could not open file %s", path);
        return RTR_ERR_IO;
    }
    fseek(f, 0, SEEK_END);
    const long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    const int rc = create_from_escape(nullptr, f, sz > 0 ? (int64_t)sz : 0, path, device, flags, out);
    fclose(f);
    return rc;
}

int rtr_batch_create(const int64_t* src, const int64_t* dst, const int64_t* eoff, const int64_t* nverts, int64_t K,
                     int device, int flags, rtr_graph** out)
{
    if (!eoff || !nverts || K <= 0 || ((!src || !dst) && eoff[K] > 0)) {
        set_error("rtr_batch_create: null arrays or empty batch");
        return RTR_ERR_ARG;
    }
    std::vector<int64_t> bases(K + 1, 0);
    for (int64_t k = 0; k < K; ++k) {
        if (nverts[k] <= 0 || eoff[k + 1] < eoff[k]) {
            set_error("rtr_batch_create: graph %lld has no vertices or a negative edge range", (long long)k);
            return RTR_ERR_INPUT;
        }
        bases[k + 1] = bases[k] + nverts[k];
    }
    const int64_t n = bases[K], m = eoff[K];
    if (n >= (int64_t)INT32_MAX) {
        set_error("rtr_batch_create: %lld vertices in total exceeds the int32 id width", (long long)n);
        return RTR_ERR_LIMIT;
    }
    // union edge list with graph-local ids shifted by each graph's base
    std::vector<int64_t> gs((size_t)m), gd((size_t)m);
    for (int64_t k = 0; k < K; ++k)
        for (int64_t i = eoff[k]; i < eoff[k + 1]; ++i) {
            if (src[i] < 0 || src[i] >= nverts[k] || dst[i] < 0 || dst[i] >= nverts[k]) {
                set_error("rtr_batch_create: graph %lld edge %lld has an endpoint outside [0, %lld)", (long long)k,
                          (long long)(i - eoff[k]), (long long)nverts[k]);
                return RTR_ERR_INPUT;
            }
            gs[i] = src[i] + bases[k];
            gd[i] = dst[i] + bases[k];
        }
    int rc = rtr_graph_create_from_edges(gs.data(), gd.data(), m, n, device, flags, out);
    if (rc) return rc;
    rtr_graph* g = *out;
    g->nbatch = K;
    g->batch_vbase = new (std::nothrow) int64_t[K + 1];
    Scratch sc(g);
    int64_t* dbases = (int64_t*)sc.get(sizeof(int64_t) * (K + 1));
    g->vbase = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
    if (!g->batch_vbase || !dbases || !g->vbase) {
        rtr_graph_destroy(g);
        *out = nullptr;
        set_error("allocation failed for the batch bases");
        return RTR_ERR_CUDA;
    }
    for (int64_t k = 0; k <= K; ++k) g->batch_vbase[k] = bases[k];
    RTR_CUDA_TRY(cudaMemcpyAsync(dbases, bases.data(), sizeof(int64_t) * (K + 1), cudaMemcpyHostToDevice, g->stream));
    k_fill_vbase<<<grid_for(n, 256), 256, 0, g->stream>>>(dbases, K, n, g->vbase);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaStreamSynchronize(g->stream));
    return RTR_OK;
}

int rtr_batch_cluster_counts(const rtr_graph* gc, int64_t* counts)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || !counts || g->nbatch <= 0) {
        set_error("not a batch graph");
        return RTR_ERR_ARG;
    }
    if (g->stage < 4) {
        set_error("clusters are not extracted yet");
        return RTR_ERR_STATE;
    }
    std::vector<int64_t> seed(g->ncl);
    int rc = copy_i32_as_i64(g, g->cl_seed, g->ncl, seed.data());
    if (rc) return rc;
    for (int64_t k = 0; k < g->nbatch; ++k) counts[k] = 0;
    for (int64_t c = 0; c < g->ncl; ++c) {
        const int64_t* b = g->batch_vbase;
        int64_t lo = 0, hi = g->nbatch;
        while (hi - lo > 1) {
            const int64_t mid = (lo + hi) >> 1;
            if (b[mid] <= seed[c]) lo = mid;
            else hi = mid;
        }
        counts[lo]++;
    }
    return RTR_OK;
}

int rtr_graph_create_from_csr(const int64_t* offsets, const int64_t* nbors, int64_t n, int device, rtr_graph** out)
{
    if (!offsets || (!nbors && offsets[n] > 0)) {
        set_error("null CSR arrays");
        return RTR_ERR_ARG;
    }
    if (offsets[0] != 0) {
        set_error("offsets[0] must be 0");
        return RTR_ERR_INPUT;
    }
    for (int64_t v = 0; v < n; ++v)
        if (offsets[v + 1] < offsets[v]) {
            set_error("offsets must be non-decreasing (vertex %lld)", (long long)v);
            return RTR_ERR_INPUT;
        }
    int rc = make_graph(n, device, out);
    if (rc) return rc;
    rtr_graph* g = *out;
    rc = build_csr_from_host_csr(g, offsets, nbors);
    if (rc) {
        rtr_graph_destroy(g);
        *out = nullptr;
    }
    return rc;
}

int rtr_graph_destroy(rtr_graph* g)
{
    if (!g) return RTR_OK;
    cudaSetDevice(g->device);
    dev_free_all(g);
    if (g->stream) cudaStreamSynchronize(g->stream);
    for (int k = 0; k < 2 * rtr_graph::kTimers; ++k)
        if (g->kev[k]) cudaEventDestroy(g->kev[k]);
    if (g->own_stream && g->stream) cudaStreamDestroy(g->stream);
    if (g->side) cudaStreamDestroy(g->side);
    delete[] g->batch_vbase;
    delete g;
    return RTR_OK;
}

int rtr_set_tuning(rtr_graph* g, int gallop_ratio, int heavy_degree, int heavy_edge)
{
    if (!g || gallop_ratio < 1 || heavy_degree < 1 || heavy_edge < 1) {
        set_error("rtr_set_tuning: null graph or parameter below 1");
        return RTR_ERR_ARG;
    }
    g->tune_gallop = gallop_ratio;
    g->tune_heavy = heavy_degree;
    g->tune_edge = heavy_edge;
    return RTR_OK;
}

int rtr_set_count_mode(rtr_graph* g, int mode, int hub_degree)
{
    if (!g || mode < 0 || mode > 2 || hub_degree < 1) {
        set_error("rtr_set_count_mode: null graph, mode outside 0..2 or hub_degree below 1");
        return RTR_ERR_ARG;
    }
    g->count_mode = mode;
    g->count_hub = hub_degree;
    return RTR_OK;
}

int rtr_get_count_mode(const rtr_graph* g, int* mode, int* hub_degree, int* lists_kept)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (mode) *mode = g->count_mode;
    if (hub_degree) *hub_degree = g->count_hub;
    if (lists_kept) *lists_kept = g->lists ? 1 : 0;
    return RTR_OK;
}

int rtr_set_count_window(rtr_graph* g, int64_t max_entries)
{
    if (!g || max_entries < 0) {
        set_error("rtr_set_count_window: null graph or negative entry count");
        return RTR_ERR_ARG;
    }
    g->rows_window_cap = max_entries;
    return RTR_OK;
}

int rtr_get_count_windows(const rtr_graph* g, int64_t* windows, int64_t* list_entries)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (windows) *windows = g->lists ? 0 : g->rows_windows;
    if (list_entries) *list_entries = g->lists ? 0 : g->rows_entries;
    return RTR_OK;
}

int rtr_set_clean_split(rtr_graph* g, int64_t min_seeds, double max_mean_list)
{
    if (!g || min_seeds < 1 || !(max_mean_list >= 0)) {
        set_error("rtr_set_clean_split: null graph, min_seeds below 1 or max_mean_list negative");
        return RTR_ERR_ARG;
    }
    g->clean_round_min = min_seeds;
    g->clean_round_list = max_mean_list;
    return RTR_OK;
}

int rtr_set_clean_checks(rtr_graph* g, int64_t first_wait_rounds, int64_t stack_entries)
{
    if (!g || first_wait_rounds < 0 || stack_entries < -1) {
        set_error("rtr_set_clean_checks: null graph, negative wait rounds or stack entries below -1");
        return RTR_ERR_ARG;
    }
    g->clean_wait_first = first_wait_rounds;
    g->clean_stack_limit = stack_entries;
    return RTR_OK;
}

int rtr_set_extract_split(rtr_graph* g, int64_t min_vertices)
{
    if (!g || min_vertices < 2) {
        set_error("rtr_set_extract_split: null graph or min_vertices below 2");
        return RTR_ERR_ARG;
    }
    g->extract_big = min_vertices;
    return RTR_OK;
}

int rtr_get_clean_split(const rtr_graph* g, int64_t* min_seeds, double* max_mean_list)
{
    if (!g || !min_seeds || !max_mean_list) {
        set_error("rtr_get_clean_split: null argument");
        return RTR_ERR_ARG;
    }
    *min_seeds = g->clean_round_min;
    *max_mean_list = g->clean_round_list;
    return RTR_OK;
}

int rtr_get_tuning(const rtr_graph* g, int* gallop_ratio, int* heavy_degree, int* heavy_edge)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (gallop_ratio) *gallop_ratio = g->tune_gallop;
    if (heavy_degree) *heavy_degree = g->tune_heavy;
    if (heavy_edge) *heavy_edge = g->tune_edge;
    return RTR_OK;
}

int rtr_autotune(rtr_graph* g, int* gallop_ratio, int* heavy_degree, int* heavy_edge)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    // one counting pass per candidate, timed by the kernels' own events;
    // coordinate descent over the three parameters in turn
    auto timed = [&](int gal, int heavy, int edge, double* ms) -> int {
        g->tune_gallop = gal;
        g->tune_heavy = heavy;
        g->tune_edge = edge;
        const int rc = count_triangles(g);
        if (rc) return rc;
        *ms = (double)g->kms[KT_EDGE_FOLD] + g->kms[KT_TRI_FILL] + g->kms[KT_VERTEX_FOLD];
        return RTR_OK;
    };
    static const int kGallop[] = {4, 8, 16, 32, 64};
    static const int kHeavy[] = {8, 16, 32, 64, 128};
    static const int kEdge[] = {128, 256, 512, 1024, 4096, 1 << 30};
    int bg = g->tune_gallop, bh = g->tune_heavy, be = g->tune_edge;
    double best = 1e300, ms = 0;
    int rc = timed(bg, bh, be, &ms);  // warm-up (first allocation of the lists)
    if (rc) return rc;
    for (int gal : kGallop) {
        if ((rc = timed(gal, bh, be, &ms))) return rc;
        if (ms < best) {
            best = ms;
            bg = gal;
        }
    }
    for (int heavy : kHeavy) {
        if (heavy == bh) continue;
        if ((rc = timed(bg, heavy, be, &ms))) return rc;
        if (ms < best) {
            best = ms;
            bh = heavy;
        }
    }
    for (int edge : kEdge) {
        if (edge == be) continue;
        if ((rc = timed(bg, bh, edge, &ms))) return rc;
        if (ms < best) {
            best = ms;
            be = edge;
        }
    }
    if ((rc = timed(bg, bh, be, &ms))) return rc;  // leave the graph counted with the choice
    if (gallop_ratio) *gallop_ratio = bg;
    if (heavy_degree) *heavy_degree = bh;
    if (heavy_edge) *heavy_edge = be;
    return RTR_OK;
}

int rtr_get_memory(const rtr_graph* g, int64_t* resident_bytes, int64_t* peak_scratch_bytes)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (resident_bytes) *resident_bytes = g->owned_bytes;
    if (peak_scratch_bytes) *peak_scratch_bytes = g->scratch_peak;
    return RTR_OK;
}

int rtr_graph_info(const rtr_graph* g, int64_t* n, int64_t* m)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (n) *n = g->n;
    if (m) *m = g->m;
    return RTR_OK;
}

int rtr_count(rtr_graph* g, int64_t* total)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    int rc = count_triangles(g);
    if (rc) return rc;
    if (total) {
        unsigned long long t = 0;
        RTR_CUDA_TRY(cudaMemcpy(&t, g->ctr, sizeof t, cudaMemcpyDeviceToHost));
        *total = (int64_t)t;
    }
    return RTR_OK;
}

int rtr_clean(rtr_graph* g, double eps, int64_t* left)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    int rc = initial_clean(g, eps);
    if (rc) return rc;
    if (left) {
        unsigned long long t = 0;
        RTR_CUDA_TRY(cudaMemcpy(&t, g->ctr, sizeof t, cudaMemcpyDeviceToHost));
        *left = (int64_t)t;
    }
    return RTR_OK;
}

int rtr_extract(rtr_graph* g, int64_t* ncl)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    int rc = extract_clusters(g);
    if (rc) return rc;
    if (ncl) *ncl = g->ncl;
    return RTR_OK;
}

int rtr_decompose(rtr_graph* g, double eps, int64_t* ncl)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    ktime_begin(g, KT_DECOMPOSE);
    int rc = rtr_count(g, nullptr);
    if (!rc) rc = rtr_clean(g, eps, nullptr);
    if (!rc) rc = rtr_extract(g, ncl);
    ktime_end(g, KT_DECOMPOSE);
    if (!rc) {
        RTR_CUDA_TRY(cudaEventSynchronize(g->kev[2 * KT_DECOMPOSE + 1]));
        ktime_read(g, KT_DECOMPOSE);
        g->ms_decompose = g->kms[KT_DECOMPOSE];
    }
    return rc;
}

int rtr_get_csr(const rtr_graph* gc, int64_t* offsets, int64_t* nbors)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 1) {
        set_error("graph not built");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    if (offsets) {
        RTR_CUDA_TRY(cudaMemcpyAsync(offsets, g->offsets, sizeof(int64_t) * (g->n + 1), cudaMemcpyDeviceToHost,
                                     g->stream));
        RTR_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    if (nbors) return copy_i32_as_i64(g, g->nbors, g->m2, nbors);
    return RTR_OK;
}

int rtr_get_weights(const rtr_graph* gc, double* perEdge, double* perVertex, uint32_t* support, int64_t* total)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 2) {
        set_error("weights are not computed yet");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int64_t m2 = g->m2;
    Scratch sc(g);
    double* ope = perEdge ? (double*)sc.get(sizeof(double) * (m2 + 1)) : nullptr;
    uint32_t* osup = support ? (uint32_t*)sc.get(sizeof(uint32_t) * (m2 + 1)) : nullptr;
    if ((perEdge && !ope) || (support && !osup)) {
        set_error("device allocation failed");
        return RTR_ERR_CUDA;
    }
    if (perEdge || support) {
        k_expand_pe<<<grid_for(m2, 256), 256, 0, s>>>(g->pe, g->sup, g->st, g->esrc, g->nbors, g->partner, m2, ope,
                                                       osup, nullptr);
        RTR_CUDA_TRY(cudaGetLastError());
    }
    if (perEdge) RTR_CUDA_TRY(cudaMemcpyAsync(perEdge, ope, sizeof(double) * m2, cudaMemcpyDeviceToHost, s));
    if (support) RTR_CUDA_TRY(cudaMemcpyAsync(support, osup, sizeof(uint32_t) * m2, cudaMemcpyDeviceToHost, s));
    if (perVertex) RTR_CUDA_TRY(cudaMemcpyAsync(perVertex, g->pv, sizeof(double) * g->n, cudaMemcpyDeviceToHost, s));
    if (total) {
        unsigned long long t = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&t, g->ctr, sizeof t, cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        *total = (int64_t)t;
    }
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    return RTR_OK;
}

int rtr_get_status(const rtr_graph* gc, uint8_t* status)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 3) {
        set_error("status is not available before the clean");
        return RTR_ERR_STATE;
    }
    if (g->m2 == 0) return RTR_OK;
    if (!status) {
        set_error("null status buffer");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    Scratch sc(g);
    uint8_t* ost = (uint8_t*)sc.get(g->m2 + 16);
    if (!ost) {
        set_error("device allocation failed");
        return RTR_ERR_CUDA;
    }
    k_expand_pe<<<grid_for(g->m2, 256), 256, 0, s>>>(g->pe, g->sup, g->st, g->esrc, g->nbors, g->partner, g->m2,
                                                      nullptr, nullptr, ost);
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaMemcpyAsync(status, ost, g->m2, cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    return RTR_OK;
}

int rtr_get_clusters(const rtr_graph* gc, int64_t* seed, int64_t* nv, int64_t* ne, int64_t* cut, int64_t* off,
                     int64_t* vert)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 4) {
        set_error("clusters are not extracted yet");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int64_t k = g->ncl;
    int rc = RTR_OK;
    if (seed && (rc = copy_i32_as_i64(g, g->cl_seed, k, seed))) return rc;
    if (vert && (rc = copy_i32_as_i64(g, g->cl_vert, g->n, vert))) return rc;
    std::vector<int64_t> o(k + 1);
    RTR_CUDA_TRY(cudaMemcpyAsync(o.data(), g->cl_off, sizeof(int64_t) * (k + 1), cudaMemcpyDeviceToHost, s));
    if (ne) RTR_CUDA_TRY(cudaMemcpyAsync(ne, g->cl_ne, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
    if (cut) RTR_CUDA_TRY(cudaMemcpyAsync(cut, g->cl_cut, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    if (off)
        for (int64_t i = 0; i <= k; ++i) off[i] = o[i];
    if (nv)
        for (int64_t i = 0; i < k; ++i) nv[i] = o[i + 1] - o[i];
    return RTR_OK;
}

int rtr_num_clusters(const rtr_graph* g, int64_t* ncl)
{
    if (!g || !ncl) {
        set_error("null argument");
        return RTR_ERR_ARG;
    }
    *ncl = g->stage >= 4 ? g->ncl : 0;
    return RTR_OK;
}

int rtr_get_cluster_of(const rtr_graph* gc, int64_t* cluster_of)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 4 || !cluster_of) {
        set_error("clusters are not extracted yet");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    return copy_i32_as_i64(g, g->cluster_of, g->n, cluster_of);
}

int rtr_expand(rtr_graph* g, int64_t threshold, int64_t* num_scores)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    const int rc = expand_clusters(g, threshold);
    if (rc) return rc;
    if (num_scores) *num_scores = g->x_nscores;
    return RTR_OK;
}

int rtr_get_expanded(const rtr_graph* gc, int64_t* nv, int64_t* ne, int64_t* cut, int64_t* off, int64_t* vert,
                     int64_t* cluster_of)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 4 || !g->expanded) {
        set_error("clusters are not expanded yet");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    cudaStream_t s = g->stream;
    const int64_t k = g->ncl;
    std::vector<int64_t> o(k + 1);
    RTR_CUDA_TRY(cudaMemcpyAsync(o.data(), g->x_off, sizeof(int64_t) * (k + 1), cudaMemcpyDeviceToHost, s));
    if (ne) RTR_CUDA_TRY(cudaMemcpyAsync(ne, g->x_ne, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
    if (cut) RTR_CUDA_TRY(cudaMemcpyAsync(cut, g->x_cut, sizeof(int64_t) * k, cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    int rc = RTR_OK;
    if (vert && (rc = copy_i32_as_i64(g, g->x_vert, o[k], vert))) return rc;
    if (cluster_of && (rc = copy_i32_as_i64(g, g->x_cof, g->n, cluster_of))) return rc;
    if (off)
        for (int64_t i = 0; i <= k; ++i) off[i] = o[i];
    if (nv)
        for (int64_t i = 0; i < k; ++i) nv[i] = o[i + 1] - o[i];
    return RTR_OK;
}

int rtr_get_scores(const rtr_graph* gc, int64_t* num_scores, int64_t* vertices, double* scores)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || g->stage < 4 || !g->expanded) {
        set_error("clusters are not expanded yet");
        return RTR_ERR_STATE;
    }
    if (num_scores) *num_scores = g->x_nscores;
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    int rc = RTR_OK;
    if (vertices && (rc = copy_i32_as_i64(g, g->x_scv, g->x_nscores, vertices))) return rc;
    if (scores && g->x_nscores) {
        RTR_CUDA_TRY(cudaMemcpyAsync(scores, g->x_scx, sizeof(double) * g->x_nscores, cudaMemcpyDeviceToHost,
                                     g->stream));
        RTR_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    return RTR_OK;
}

int rtr_connected_components(rtr_graph* g, int64_t* ncomp)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    const int rc = connected_components(g);
    if (rc) return rc;
    if (ncomp) *ncomp = g->ncc;
    return RTR_OK;
}

int rtr_get_components(const rtr_graph* gc, int64_t* off, int64_t* vert)
{
    rtr_graph* g = const_cast<rtr_graph*>(gc);
    if (!g || !g->cc_vert) {
        set_error("components are not computed yet");
        return RTR_ERR_STATE;
    }
    RTR_CUDA_TRY(cudaSetDevice(g->device));
    if (off) {
        RTR_CUDA_TRY(cudaMemcpyAsync(off, g->cc_off, sizeof(int64_t) * (g->ncc + 1), cudaMemcpyDeviceToHost,
                                     g->stream));
        RTR_CUDA_TRY(cudaStreamSynchronize(g->stream));
    }
    if (vert) return copy_i32_as_i64(g, g->cc_vert, g->n, vert);
    return RTR_OK;
}

int rtr_get_stats(const rtr_graph* g, double* ms4, int64_t* launches, int64_t* residual)
{
    if (!g) {
        set_error("null graph");
        return RTR_ERR_ARG;
    }
    if (ms4) {
        ms4[0] = g->ms_build;
        ms4[1] = g->ms_count;
        ms4[2] = g->ms_clean;
        ms4[3] = g->ms_extract;
    }
    if (launches) *launches = g->launches;
    if (residual) *residual = g->diag_residual;
    return RTR_OK;
}

int rtr_get_kernel_ms(const rtr_graph* g, double* ms, int n)
{
    if (!g || !ms) {
        set_error("null argument");
        return RTR_ERR_ARG;
    }
    for (int k = 0; k < n && k < rtr_graph::kTimers; ++k) ms[k] = g->kms[k];
    return RTR_OK;
}

void rtr_free(void* p) { free(p); }

}  // extern "C"
