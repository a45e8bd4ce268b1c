// Host-side handle for one graph resident in HBM, and the stage entry points
// the C ABI (capi.cu) drives.  All device work of a graph runs on its own
// stream; calls on different graphs may run concurrently.
#pragma once

#include "rtr_common.cuh"

#include <cstddef>
#include <cstdio>
#include <cstdint>
#include <vector>

struct rtr_graph {
    int device = 0;
    cudaStream_t stream = nullptr;
    bool own_stream = false;

    int64_t n = 0;   // vertices
    int64_t m2 = 0;  // directed slots (2 x undirected edges)
    int64_t m = 0;   // undirected edges

    // CSR (see rtr_common.cuh for the layout)
    int64_t* offsets = nullptr;
    int32_t* nbors = nullptr;
    int32_t* esrc = nullptr;
    int32_t* partner = nullptr;
    int32_t* deg = nullptr;
    int32_t* fwd = nullptr;    // the m forward slots, ascending
    int32_t* frank = nullptr;  // [2m] position of a forward slot in fwd

    // weighted-triangle state
    double* pe = nullptr;
    double* pv = nullptr;
    uint32_t* sup = nullptr;
    uint8_t* st = nullptr;
    int64_t* tl_off = nullptr;  // [m2+1]
    rtr::TriEntry* tl = nullptr;
    int64_t tl_len = 0;

    // small device counters: [0] triangle total, [1] error word, [2..] stage stats
    unsigned long long* ctr = nullptr;

    // extraction results: clusters in creation order
    int64_t ncl = 0;
    int32_t* cl_seed = nullptr;    // [ncl]
    int64_t* cl_off = nullptr;     // [ncl+1] into cl_vert
    int32_t* cl_vert = nullptr;    // [n] members, in set-iteration order
    int64_t* cl_ne = nullptr;      // [ncl] internal edges
    int64_t* cl_cut = nullptr;     // [ncl] cut edges
    int32_t* cluster_of = nullptr; // [n]

    // expandClusters results (same clusters, creation order; emptied ones have no members)
    bool expanded = false;
    int64_t x_threshold = 0;
    int64_t* x_off = nullptr;     // [ncl+1] into x_vert
    int32_t* x_vert = nullptr;    // members in set-iteration order
    int64_t* x_ne = nullptr;      // [ncl]
    int64_t* x_cut = nullptr;     // [ncl]
    int32_t* x_cof = nullptr;     // [n] cluster of each vertex, -1 when in none
    int64_t x_nscores = 0;
    int32_t* x_scv = nullptr;     // moved vertices, ascending
    double* x_scx = nullptr;      // their scores

    // nucleus (truss-hierarchy) clusters in output order, members in original labels
    bool nuc_done = false;
    std::vector<int64_t> nuc_c, nuc_nv, nuc_ne, nuc_parent, nuc_off, nuc_vert;
    float ms_nucleus = 0;

    // connected components of the original graph, creation order, BFS discovery order inside
    int64_t ncc = 0;
    int64_t* cc_off = nullptr;   // [ncc+1]
    int32_t* cc_vert = nullptr;  // [n]

    // batch of independent graphs held as one disjoint union
    int64_t nbatch = 0;
    int32_t* vbase = nullptr;   // [n] first vertex id of the vertex's graph (null: single graph)
    int64_t* batch_vbase = nullptr;  // host copy, [nbatch+1]

    double eps = 0.3;
    int stage = 0;  // 1 built, 2 counted, 3 cleaned, 4 extracted
    // counting work split (results do not depend on it): gallop ratio and heavy-vertex degree
    int tune_gallop = 16;
    int tune_heavy = 32;
    int tune_edge = 1024;  // deg u + deg v from which an edge is intersected by a warp
    // counting layout: 0 keep triangle lists when they fit in free device memory,
    // 1 always keep them, 2 never (rows layout: folds straight from the CSR);
    // count_hub: perVertex terms from which the rows layout folds a vertex with a warp
    int count_mode = 0;
    int64_t rows_window_cap = 0;  // rows layout: list entries per window at most (0: as many as fit)
    int64_t rows_windows = 0;  // rows layout: windows the last count took, and its list entries
    int64_t rows_entries = 0;
    // rows layout buffers, owned by the graph and reused by later counts (grow-only)
    void* rows_masks = nullptr;
    int64_t rows_masks_cap = 0;
    void* rows_lists = nullptr;
    int64_t rows_lists_cap = 0;
    int count_hub = 1024;
    bool lists = false;  // the last count kept the triangle lists (the clean needs them)
    // clean units with at least this many seeds and triangle lists of at most
    // this mean length replay in parallel rounds (one thread block each); the
    // others one warp per unit
    int64_t clean_round_min = 2048;
    double clean_round_list = 8.0;
    // bounds of the clean's device-side checks, lowered only to test their reports:
    // try_wait rounds of a window's first wait (0: the full limit), unit stack entries (-1: as sized)
    int64_t clean_wait_first = 0;
    int64_t clean_stack_limit = -1;
    // extraction: components of at least this many vertices are replayed by a
    // whole thread block (the two-hop scan's pairs worked out ahead), the others by a warp
    int64_t extract_big = 512;
    cudaStream_t side = nullptr;  // second stream of the graph (created on first use)

    // stage timings from CUDA events (ms)
    float ms_build = 0, ms_count = 0, ms_clean = 0, ms_extract = 0, ms_decompose = 0, ms_expand = 0;
    // per-kernel device times of the last run (ms), CUDA events on the graph's stream:
    // [0] k_edge_fold [1] k_tri_fill [2] k_vertex_fold [3] k_clean_units [4] k_extract_components
    // [5] decompose [6] k_edge_fold alone [7] k_edge_count_heavy alone [8] the rows
    // layout's warp perVertex fold (second stream, concurrent with the thread fold)
    // [9] k_fill_light [10] k_fill_heavy [11] the block perVertex fold (rows layout; second
    // stream, while [8] is then the warp fold alone on the graph's stream)
    static constexpr int kTimers = 12;
    cudaEvent_t kev[2 * kTimers] = {};
    float kms[kTimers] = {};
    // launch accounting for this graph (kernels issued by the library)
    long long launches = 0;

    // diagnostics mirroring the reference's print-and-continue self-checks
    long long diag_residual = 0;
    long long diag_bad_status = 0;

    std::vector<void*> owned;  // device allocations released by rtr_graph_destroy
    // device bytes: held by the graph (owned), and temporary scratch now / at most
    int64_t owned_bytes = 0;
    int64_t scratch_bytes = 0;
    int64_t scratch_peak = 0;
};

namespace rtr {

void* dev_alloc(rtr_graph* g, size_t bytes);  // stream-ordered, owned by g

// Kernel timers: record around a launch on the graph's stream, read after a sync.
enum KernelTimer {
    KT_EDGE_FOLD = 0,
    KT_TRI_FILL,
    KT_VERTEX_FOLD,
    KT_CLEAN_UNITS,
    KT_EXTRACT,
    KT_DECOMPOSE,
    KT_EDGE_LIGHT,
    KT_EDGE_HEAVY,
    KT_FOLD_WARP,
    KT_FILL_LIGHT,
    KT_FILL_HEAVY,
    KT_FOLD_BLOCK
};
inline void ktime_begin(rtr_graph* g, int k, cudaStream_t s = nullptr)
{
    cudaEventRecord(g->kev[2 * k], s ? s : g->stream);
}
inline void ktime_end(rtr_graph* g, int k, cudaStream_t s = nullptr)
{
    cudaEventRecord(g->kev[2 * k + 1], s ? s : g->stream);
}
inline void ktime_read(rtr_graph* g, int k)
{
    float ms = 0;
    if (cudaEventElapsedTime(&ms, g->kev[2 * k], g->kev[2 * k + 1]) == cudaSuccess) g->kms[k] = ms;
}
void dev_free_all(rtr_graph* g);

// Temporary device memory released before the call returns.
struct Scratch {
    rtr_graph* g;
    std::vector<void*> ptrs;
    int64_t bytes = 0;
    explicit Scratch(rtr_graph* gr) : g(gr) {}
    void* get(size_t bytes);
    ~Scratch();
};

// free device memory; trim: first return the pool's cached blocks (graph.cu)
size_t free_device_bytes(rtr_graph* g, bool trim);
// free device memory plus the pool's cached blocks, without trimming
size_t device_avail_bytes(rtr_graph* g);
// a graph-owned grow-only buffer of at least `bytes` (trims the pool before growing; null on failure)
void* grow_owned(rtr_graph* g, void** buf, int64_t* cap, int64_t bytes);
void release_owned(rtr_graph* g, void** buf, int64_t* cap);
int build_csr(rtr_graph* g, const int64_t* d_u, const int64_t* d_v, int64_t m, bool simplify);
int build_csr_from_host_csr(rtr_graph* g, const int64_t* h_offsets, const int64_t* h_nbors);
int count_triangles(rtr_graph* g);
struct RowSets;
// hash sets of the rows of at least min_deg entries, in sc (count_rows.cu)
int build_row_sets(rtr_graph* g, Scratch& sc, int min_deg, RowSets* out);
// rows layout: perVertex from per-slot lists of z (count_rows.cu); cgt the
// per-slot term counts, lpos room for their scan, heavy_list the heavy edges,
// masks (may be null) the count's hit masks of them at word offsets moff
int count_rows(rtr_graph* g, Scratch& sc, const RowSets& rs, const int64_t* cgt, int64_t* lpos,
               const int32_t* heavy_list, const unsigned* nheavy, const int64_t* moff, const uint32_t* masks);
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);
int initial_clean(rtr_graph* g, double eps);
int extract_clusters(rtr_graph* g);
int connected_components(rtr_graph* g);
int expand_clusters(rtr_graph* g, int64_t threshold);
// Escape text (host buffer h_text, or the open file f when h_text is null) of
// len bytes -> device edge arrays in sc.
int parse_escape_device(rtr_graph* g, Scratch& sc, const char* h_text, FILE* f, int64_t len, const char* what,
                        int64_t* n_out, int64_t* m_out, int64_t** du_out, int64_t** dv_out);

}  // namespace rtr
