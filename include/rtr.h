/* rtr.h -- C ABI of librtr.so, the B200 (sm_100a) implementation of the
 * RTRExtractor decomposition path: weighted per-edge triangle counting,
 * cascading edge cleaning and dense-cluster extraction.
 *
 * Plain pointers and sizes only.  The library owns all device memory of a
 * graph; the caller owns every host buffer it passes in.  Every call returns
 * an rtr_status (0 = RTR_OK); on failure rtr_last_error() describes the cause
 * (per calling thread).  Nothing in the library calls exit().  Calls on
 * different graphs may run concurrently from different threads; calls on one
 * graph must not overlap.
 *
 * Array layouts follow the reference:
 *   offsets  int64[n+1], nbors int64[2m]   the symmetric CSR of makeCSR
 *                                           (RTRex_Sequential/Graph.cpp:344-384),
 *                                           rows ascending by neighbour id
 *   perEdge  double[2m]  one cell per directed slot (both copies of an edge
 *                        hold the same value), perVertex double[n]
 *   status   uint8[2m]   'Y' alive / 'N' deleted, as edgeStatus
 *                        (RTRex_Sequential/Escape/Decomposition.h:127)
 *   support  uint32[2m]  live triangles on each slot (integer companion)
 * Inputs must be simple graphs (no self-loops, no repeated pairs) unless
 * RTR_FLAG_SIMPLIFY is passed, which drops them before building the CSR.
 */
#ifndef RTR_H
#define RTR_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rtr_graph rtr_graph;

enum rtr_status {
    RTR_OK = 0,
    RTR_ERR_ARG = 1,     /* null pointer / bad argument */
    RTR_ERR_CUDA = 2,    /* CUDA runtime error or allocation failure */
    RTR_ERR_INPUT = 3,   /* malformed graph: ids out of range, self-loops, duplicates, asymmetric CSR */
    RTR_ERR_LIMIT = 4,   /* size beyond the supported index width (n, 2m < 2^31-1) */
    RTR_ERR_STATE = 5,   /* stage called out of order */
    RTR_ERR_DEVICE = 6,  /* a kernel reported an internal inconsistency (error word) */
    RTR_ERR_IO = 7       /* file could not be read or written / short edge count */
};

enum rtr_flags {
    RTR_FLAG_SIMPLIFY = 1,     /* drop self-loops and duplicate pairs instead of rejecting them */
    RTR_FLAG_RTREX_OUTPUTS = 2, /* rtr_run_file also writes what the sequential RTRex CLI writes besides the
                                   decomposition: connected-components-<name>-* and amazon_cleaned_edges.txt */
    RTR_FLAG_EXPAND = 4         /* rtr_run_file_ex also runs expandClusters (the RTRex driver's mode e) */
};

/* Library version string and the calling thread's last error message. */
const char* rtr_version(void);
const char* rtr_last_error(void);

/* Build a graph on `device` from m undirected pairs (src[i], dst[i]), 0 <= id < n,
 * stored in both directions as loadGraph(.., undirected=1, escape) does, with
 * the CSR built on the device (radix sort, offsets, partner map).
 * Replaces: loadGraph_Escape's edge storage (RTRex_Sequential/GraphIO.cpp:42-63),
 *           makeCSR (RTRex_Sequential/Graph.cpp:344-384),
 *           CGraph::getPartnerMap (RTRex_Sequential/Graph.cpp:320-340) and
 *           transferGraphToDevice (RTRex_CUDA/gpu_graph.cuh:47-52). */
int rtr_graph_create_from_edges(const int64_t* src, const int64_t* dst, int64_t m, int64_t n, int device, int flags,
                                rtr_graph** out);

/* Build an R-MAT graph on `device` without host edge arrays: 2^scale vertices,
 * edge_factor * 2^scale generated pairs (below 2^30) with quadrant
 * probabilities a, b, c (d = 1-a-b-c), symmetrised, self-loops and repeated
 * pairs dropped.  Edge k's bit at level l comes from the splitmix64 output
 * function of seed * 0x9E3779B97F4A7C15 ^ (k << 6 | l): high 32 bits >=
 * floor((a+b) 2^32) sets the source bit, low 32 bits >= floor(a/(a+b) 2^32)
 * (source bit clear) or floor(c/(1-a-b) 2^32) (set) the destination bit, level
 * l giving bit scale-1-l.  For synthetic large-graph workloads; no counterpart
 * in the reference, which reads edge-list files. */
int rtr_graph_create_rmat(int scale, int64_t edge_factor, double a, double b, double c, uint64_t seed, int device,
                          rtr_graph** out);

/* Build a graph from a host CSR (symmetric, rows strictly ascending).
 * Replaces: transferGraphToDevice(h_offsets, h_nbors, nVertices, nEdges, dg)
 *           (RTRex_CUDA/gpu_graph.cuh:47-52) with allocateDeviceState (:57). */
int rtr_graph_create_from_csr(const int64_t* offsets, const int64_t* nbors, int64_t n, int device, rtr_graph** out);

/* Build ONE device graph that holds K independent graphs (their disjoint
 * union) so a single rtr_decompose runs them all: graph k has nverts[k]
 * vertices and the undirected pairs (src[i], dst[i]), i in [eoff[k], eoff[k+1]),
 * in graph-local ids.  Graph k's vertex v becomes union vertex base_k + v with
 * base_k = nverts[0] + ... + nverts[k-1]; clusters, weights and statuses come
 * back in union ids and equal, graph by graph, what a separate decomposition of
 * each graph returns (the extraction hashes graph-local ids, so set-iteration
 * orders match).  No counterpart in the reference, which decomposes one graph
 * per process. */
int rtr_batch_create(const int64_t* src, const int64_t* dst, const int64_t* eoff, const int64_t* nverts, int64_t K,
                     int device, int flags, rtr_graph** out);

/* Clusters per graph of a batch after extraction (counts[K]). */
int rtr_batch_cluster_counts(const rtr_graph* g, int64_t* counts);

/* Release every device buffer of the graph.
 * Replaces: freeDeviceGraph (RTRex_CUDA/gpu_graph.cuh:62). */
int rtr_graph_destroy(rtr_graph* g);

/* n and the number of undirected edges m (nEdges/2 in the reference). */
int rtr_graph_info(const rtr_graph* g, int64_t* n, int64_t* m);

/* Device memory of the graph: bytes it holds between calls (CSR, state,
 * results) and the largest temporary working set any call has needed so far.
 * No counterpart in the reference; used for admission by memory budget. */
int rtr_get_memory(const rtr_graph* g, int64_t* resident_bytes, int64_t* peak_scratch_bytes);

/* Work split of the counting kernels: an intersection gallops the shorter row
 * through the longer when their lengths differ by more than gallop_ratio
 * (otherwise it merges); a vertex of at least heavy_degree neighbours has its
 * perVertex fold done by a whole warp; an edge whose endpoints' degrees sum to
 * at least heavy_edge is intersected by a whole warp.  Defaults 16, 32, 1024.
 * Results are the same bits for every setting; only the time changes.  No
 * counterpart in the reference. */
int rtr_set_tuning(rtr_graph* g, int gallop_ratio, int heavy_degree, int heavy_edge);
int rtr_get_tuning(const rtr_graph* g, int* gallop_ratio, int* heavy_degree, int* heavy_edge);

/* Counting layout.  mode 0 (the default) keeps the per-edge triangle lists
 * (32 B per triangle and edge) when they fit in the device memory that is free
 * beside what the clean needs, and otherwise counts without them; mode 1 always
 * keeps them (RTR_ERR_CUDA when they do not fit); mode 2 never does.  Without
 * them ("rows layout") the count keeps 4-byte per-slot lists of the z > y terms
 * of perVertex instead (taken in windows of whole rows when even those do not
 * fit) and folds perVertex from them -- the same bits; a vertex of at least
 * hub_degree perVertex terms (default 1024) is folded by a warp, the others by
 * a thread.  Those lists (and, on large graphs, the heavy edges' hit masks)
 * stay allocated with the graph for its next count, until a count keeps the
 * triangle lists or rtr_graph_destroy.  The clean and the extraction need the
 * triangle lists, so rtr_clean then returns
 * RTR_ERR_LIMIT.  *lists_kept tells whether the last rtr_count kept them.  No
 * counterpart in the reference, whose commonNbr keeps no lists
 * (RTRex_Sequential/Escape/Decomposition.h:42-117). */
int rtr_set_count_mode(rtr_graph* g, int mode, int hub_degree);
int rtr_get_count_mode(const rtr_graph* g, int* mode, int* hub_degree, int* lists_kept);
/* Rows layout of the last rtr_count: the windows of whole rows its per-slot
 * lists were filled and folded in (1 when they all fit in free device memory)
 * and their total entries (3 per triangle); both 0 when the lists were kept.
 * No counterpart in the reference. */
int rtr_get_count_windows(const rtr_graph* g, int64_t* windows, int64_t* list_entries);
/* At most max_entries per-slot list entries per rows-layout window (0, the
 * default: as many as fit in free device memory).  Results are the same bits
 * for every setting; smaller windows only take more passes (a vertex whose
 * perVertex terms exceed the window is an RTR_ERR_LIMIT).  No counterpart in
 * the reference. */
int rtr_set_count_window(rtr_graph* g, int64_t max_entries);

/* Split of the cascading clean: units (connected components of the
 * triangle-carrying edges) with at least min_seeds seeds and triangle lists of
 * at most max_mean_list entries on average are replayed in parallel rounds by
 * one thread block each -- pops whose cells are disjoint run together,
 * perVertex is folded afterwards in the reference's pop order -- and the other
 * units one warp per unit.  Defaults 2048 and 8.  Results are the same bits
 * for every setting.  No counterpart in the reference. */
int rtr_set_clean_split(rtr_graph* g, int64_t min_seeds, double max_mean_list);
int rtr_get_clean_split(const rtr_graph* g, int64_t* min_seeds, double* max_mean_list);

/* Split of the extraction: components of the cleaned graph with at least
 * min_vertices vertices (default 512) replay their seed loop in a whole thread
 * block -- the two-hop scan's pairs worked out by seven warps ahead of the warp
 * that applies them in order -- and the others in one warp each.  Results are
 * the same bits for every setting.  No counterpart in the reference. */
int rtr_set_extract_split(rtr_graph* g, int64_t min_vertices);

/* Bounds of the clean's device-side self-checks, to test their error reports
 * (no counterpart in the reference).  first_wait_rounds limits the first
 * bounded wait of the warp-per-unit replay on each window's asynchronous copies
 * (0 = the full limit; a lowered limit probes the barrier without blocking);
 * when it runs out the warp reports it and drains the copies under the full
 * limit before it stops.  stack_entries caps the depth of every unit's cascade
 * stack (-1 = bounded only by the unit's own region).  A check that fires makes
 * rtr_clean return RTR_ERR_DEVICE with the condition named in rtr_last_error();
 * the graph's results are then incomplete but the device stays usable. */
int rtr_set_clean_checks(rtr_graph* g, int64_t first_wait_rounds, int64_t stack_entries);

/* Autotuner: times the counting pass on this graph for gallop ratios
 * {4,8,16,32,64}, then heavy degrees {8,16,32,64,128}, then heavy-edge degree
 * sums {128,256,512,1024,4096,off} (coordinate descent, each candidate timed by
 * the kernels' CUDA events), keeps the fastest triple in the graph and returns
 * it.  Leaves the graph counted (as after rtr_count).  Reuse the triple on
 * similar graphs with rtr_set_tuning.  No counterpart in the reference. */
int rtr_autotune(rtr_graph* g, int* gallop_ratio, int* heavy_degree, int* heavy_edge);

/* Weighted triangle counting: perEdge, perVertex, support and the total.
 * Replaces: commonNbr (RTRex_Sequential/Escape/Decomposition.h:42-117) and
 *           gpuCommonNbr (RTRex_CUDA/gpu_triangle_count.cuh:23). */
int rtr_count(rtr_graph* g, int64_t* total_triangles);

/* Initial clean at threshold eps (edges with perEdge < eps/(du*dv) are removed
 * in cascade); returns the triangles left.
 * Replaces: initialClean (Decomposition.h:302-460, deleteAndClean :147-283) and
 *           gpuInitialClean (RTRex_CUDA/gpu_clean.cuh:30). */
int rtr_clean(rtr_graph* g, double eps, int64_t* triangles_left);

/* Cluster extraction from the cleaned graph; returns the number of clusters.
 * Replaces: disjointExtract's seed loop (Decomposition.h:566-919) with
 *           populateStats (:473-491), and disjointExtractCUDA
 *           (RTRex_CUDA/main.cu:130-338) with gpuExtractInner / gpuMarkClusterEdges /
 *           gpuDeleteAndClean (RTRex_CUDA/gpu_extract.cuh:28-59, gpu_clean.cuh:44). */
int rtr_extract(rtr_graph* g, int64_t* n_clusters);

/* rtr_count + rtr_clean(eps) + rtr_extract in one call.
 * Replaces: disjointExtract (Decomposition.h:538-940). */
int rtr_decompose(rtr_graph* g, double eps, int64_t* n_clusters);

/* Copy the CSR to host buffers (offsets[n+1], nbors[2m]). */
int rtr_get_csr(const rtr_graph* g, int64_t* offsets, int64_t* nbors);

/* Copy the current weights (any pointer may be NULL).
 * Replaces: syncWeightsDeviceToHost (RTRex_CUDA/gpu_graph.cuh:69-73). */
int rtr_get_weights(const rtr_graph* g, double* perEdge, double* perVertex, uint32_t* support, int64_t* total);

/* Copy the edge status ('Y' / 'N'; 'S' never remains after a stage).
 * Replaces: syncEdgeStatusDeviceToHost (RTRex_CUDA/gpu_graph.cuh:77). */
int rtr_get_status(const rtr_graph* g, uint8_t* status);

/* Copy the clusters in creation order: cluster k has seed[k], nVertices nv[k],
 * internal edges ne[k], cut edges cut[k], and members vert[off[k] .. off[k+1])
 * in the order the reference's unordered_set iterates them.
 * Sizes: seed/nv/ne/cut[n_clusters], off[n_clusters+1], vert[n].
 * Replaces: the vector<Cluster> returned by disjointExtract (Decomposition.h:538). */
int rtr_get_clusters(const rtr_graph* g, int64_t* seed, int64_t* nv, int64_t* ne, int64_t* cut, int64_t* off,
                     int64_t* vert);

/* Number of clusters produced by the last extraction (0 before one). */
int rtr_num_clusters(const rtr_graph* g, int64_t* n_clusters);

/* cluster_of[v] = index of v's cluster (creation order), the cluster_map of
 * disjointExtract (Decomposition.h:538). */
int rtr_get_cluster_of(const rtr_graph* g, int64_t* cluster_of);

/* Stage times in milliseconds from CUDA events: [build, count, clean, extract];
 * kernel launches issued for this graph so far; diagnostic counter of the
 * reference's residual self-check (Decomposition.h:273-277). */
int rtr_get_stats(const rtr_graph* g, double* ms4, int64_t* launches, int64_t* residual_warnings);

/* Connected components of the original graph, in creation order (ascending
 * smallest vertex), each listing its vertices in breadth-first discovery order.
 * Replaces: connectedComp (RTRex_Sequential/Escape/Decomposition.h:1023-1068). */
int rtr_connected_components(rtr_graph* g, int64_t* n_components);

/* Copy the components: component k has vertices vert[off[k] .. off[k+1]) in
 * discovery order.  Sizes: off[n_components+1], vert[n]. */
int rtr_get_components(const rtr_graph* g, int64_t* off, int64_t* vert);

/* The nucleus (truss-hierarchy) path of the reference's nucleus driver: the
 * graph relabelled by (degree, id), every edge's triangles listed, edges
 * peeled level by level (an edge goes at level c when it is in fewer than c
 * live triangles; kappa = c-1) in the reference's LIFO order, and the edge
 * hierarchy turned into clusters, highest level first.  *n_clusters receives
 * their number.  Results are bit-identical to the reference (its
 * fixed-size arrays overrun on some inputs, e.g. K20, where its output is
 * undefined).
 * Replaces: clustering/nucleus.cpp:12-81 with Escape/Digraph.h:84-134 and
 *           Escape/Nucleus.h:78-565 (betterWedgeEnumerator, storeAllTriangles, nuclei). */
int rtr_nucleus(rtr_graph* g, int64_t* n_clusters);

/* The clusters of the last rtr_nucleus, in the order the driver writes them:
 * cluster k has level c[k], nv[k] vertices, ne[k] edges, parent[k] (-1: none)
 * and members vert[off[k] .. off[k+1]) in original labels, ascending in the
 * relabelled order.  Sizes: c/nv/ne/parent[n_clusters], off[n_clusters+1],
 * vert[n_members]; any pointer may be NULL (call once with NULLs for the sizes). */
int rtr_get_nuclei(const rtr_graph* g, int64_t* n_clusters, int64_t* n_members, int64_t* c, int64_t* nv,
                   int64_t* ne, int64_t* parent, int64_t* off, int64_t* vert);

/* Write the clusters of the last rtr_nucleus to `path` exactly as the nucleus
 * driver writes its output file (nucleus.cpp:62-76). */
int rtr_write_nuclei(const rtr_graph* g, const char* path);

/* Write <name>-decomposition.txt / -stats.txt / -freq.txt / -cut.txt for the
 * connected components, as RTRex.cpp:203-204 prints them through
 * printDecomposition (members in the order the reference's unordered_set
 * iterates them after inserting them in discovery order). */
int rtr_write_components(const rtr_graph* g, const char* name);

/* Device times (ms, CUDA events on the graph's stream) of the last run of the
 * main kernels: ms[0] edge fold, [1] triangle-list fill, [2] vertex fold,
 * [3] unit clean replay, [4] component extraction, [5] whole rtr_decompose.
 * Replaces: the phase timers the reference prints (Decomposition.h:556,563,926;
 *           RTRex_CUDA/gpu_triangle_count.cu:135-139, gpu_clean.cu:206-210). */
int rtr_get_kernel_ms(const rtr_graph* g, double* ms, int n);

/* Weighted triangle counting into caller-provided DEVICE buffers, with no
 * device allocation at all -- for callers that cannot let a library call
 * cudaMalloc (a server that reserves its HBM budget up front and allocates only
 * from its own arena, or a latency-critical path where cudaMalloc/cudaFree may
 * synchronise the device).  No counterpart in the reference: it is an extra
 * entry point of this library.
 *   d_offsets int64[n+1], d_nbors int32[2m]  symmetric CSR on the current device:
 *                                            offsets non-decreasing from 0 to 2m,
 *                                            rows strictly ascending, ids in [0, n),
 *                                            no self-loops
 *   d_perEdge f64[2m], d_perVertex f64[n], d_support u32[2m], d_total int64[1]
 *                                            outputs, bit-identical to rtr_count's
 *   stream    a cudaStream_t (NULL = the default stream); the call is
 *             asynchronous and the outputs are ready when the stream is
 * Every buffer must be non-null when n > 0 (RTR_ERR_ARG otherwise).  Neighbour
 * ids outside [0, n) are skipped, never dereferenced, and make *d_total -1.
 * Working memory is one fixed static device array (about 4.3 MB, held by every
 * GPU that loads librtr.so until exit), so n is limited to 1,048,576 vertices;
 * larger graphs get RTR_ERR_LIMIT.  The first call on each device looks up that
 * array's device address (make it before any stream capture; a failed lookup is
 * retried by the next call, and the address is not valid after a
 * cudaDeviceReset).  All calls share the array, so calls that overlap on the
 * GPU race: serialise them. */
int rtr_count_noalloc(const int64_t* d_offsets, const int32_t* d_nbors, int64_t n, double* d_perEdge,
                      double* d_perVertex, uint32_t* d_support, int64_t* d_total, void* stream);

/* Cluster expansion after rtr_extract: every cluster that has one vertex joins
 * the cluster holding most of its neighbours (the one whose count first
 * reaches the maximum in neighbour order) when that count exceeds `threshold`;
 * its score is that count / its degree.  Votes read the extraction's cluster
 * map; statistics are recomputed.  *num_scores receives the number of scored
 * (moved) vertices.  Not defined for a batch handle (RTR_ERR_ARG).
 * Replaces: expandClusters (RTRex_Sequential/Escape/Decomposition.h:958-1008),
 *           called by the RTRex driver in mode e (clustering/RTRex.cpp:196-201). */
int rtr_expand(rtr_graph* g, int64_t threshold, int64_t* num_scores);

/* Copy the expanded clusters: the extraction's clusters, same count and order,
 * with statistics nv/ne/cut recomputed and members vert[off[k] .. off[k+1]) in
 * the order the reference's unordered_set iterates them after the moves
 * (clusters emptied by a move have nv 0).  cluster_of[v] is v's cluster or -1
 * when v is in none (only possible with threshold <= 0).  Any pointer may be
 * NULL.  Sizes: nv/ne/cut[n_clusters], off[n_clusters+1], vert[n], cluster_of[n].
 * Replaces: the vector<Cluster> returned by expandClusters (Decomposition.h:958). */
int rtr_get_expanded(const rtr_graph* g, int64_t* nv, int64_t* ne, int64_t* cut, int64_t* off, int64_t* vert,
                     int64_t* cluster_of);

/* The scores of the moved vertices in ascending vertex order: *num_scores
 * receives their number; vertices[num_scores] and scores[num_scores] are
 * filled when non-NULL.
 * Replaces: the std::map<VertexIdx,double> scores of expandClusters (Decomposition.h:958). */
int rtr_get_scores(const rtr_graph* g, int64_t* num_scores, int64_t* vertices, double* scores);

/* Write <name>-{decomposition,stats,freq,cut}.txt of the expanded clusters as
 * printDecomposition does and <name>-scores.txt as printScores does
 * (RTRex_Sequential/clustering/RTRex.cpp:19-118, :120-135, :199-200). */
int rtr_write_expanded(const rtr_graph* g, const char* name);

/* ---- Request server (no counterpart in the reference) ----------------------
 * Graphs are registered once (the server keeps a host copy of the edges) and
 * decomposition requests are submitted against them.  Worker threads admit
 * requests continuously: the oldest queued request whose graph is idle and whose
 * device working set fits the HBM budget starts as soon as a worker is free, on
 * its graph's own stream, so requests overlap on the device.  Graphs stay
 * resident in HBM after a request and are evicted least-recently-used when the
 * budget needs room.  Requests for graphs with at most batch_max_edges edges
 * that wait together (same eps and flags, up to batch_max_graphs) run as one
 * batched decomposition.  Every result equals the graph's own rtr_decompose. */
typedef struct rtr_server rtr_server;

typedef struct rtr_request_info {
    int status;              /* rtr_status of the request */
    int batched;             /* graphs decomposed together with it (1 = alone) */
    int64_t n_clusters;      /* clusters extracted */
    int64_t triangles;       /* triangles before the clean */
    int64_t triangles_left;  /* triangles after the clean */
    double t_submit_ms;      /* server clock: submission, */
    double t_start_ms;       /* start of its device work, */
    double t_end_ms;         /* results ready on the host */
    char error[160];         /* message when status != RTR_OK */
} rtr_request_info;

int rtr_server_create(int device, int64_t hbm_budget_bytes, int workers, int64_t batch_max_edges,
                      int batch_max_graphs, rtr_server** out);

/* Register a graph (copied); *graph_id is its handle for rtr_server_submit. */
int rtr_server_add_graph(rtr_server* s, const int64_t* src, const int64_t* dst, int64_t m, int64_t n, int flags,
                         int64_t* graph_id);

/* Queue a decomposition at eps; cluster_of (n entries, or NULL) receives the
 * cluster of every vertex (creation order) and must stay valid until the
 * request is waited for. */
int rtr_server_submit(rtr_server* s, int64_t graph_id, double eps, int64_t* cluster_of, int64_t* request_id);

/* Block until the request is done and release it; info may be NULL. */
int rtr_server_wait(rtr_server* s, int64_t request_id, rtr_request_info* info);

/* stats[0..n): resident graphs, bytes in use (resident + reserved), peak bytes
 * in use, peak requests in flight, evictions, batched launches, requests served
 * in batches, queued requests. */
int rtr_server_stats(rtr_server* s, int64_t* stats, int n);

/* Stop the workers after the requests in flight; queued requests are cancelled
 * (status RTR_ERR_STATE).  Call it after every rtr_server_wait has returned. */
int rtr_server_destroy(rtr_server* s);

/* Write <name>-decomposition.txt, -stats.txt, -freq.txt and -cut.txt exactly as
 * printDecomposition does (RTRex_Sequential/clustering/RTRex.cpp:19-118,
 * RTRex_CUDA/main.cu:57-108), and print its summary lines to stdout. */
int rtr_write_decomposition(const rtr_graph* g, const char* name);

/* Create a graph straight from Escape edge-list text: the bytes go to the
 * device and are parsed there (line rules of rtr_load_escape: '#' comments and
 * blank lines skipped, first data line "n m", then one pair per line, lines past
 * the m-th pair ignored), then the CSR is built on the device.  Errors and
 * messages are rtr_load_escape's (RTR_ERR_IO for malformed or short input).
 * Replaces: loadGraph(path, g, 1, IOFormat::escape) + makeCSR +
 *           transferGraphToDevice (GraphIO.cpp:19-88, Graph.cpp:344-384,
 *           RTRex_CUDA/gpu_graph.cuh:47-60). */
int rtr_graph_create_from_escape_text(const char* text, int64_t len, int device, int flags, rtr_graph** out);

/* The same from a file.  Files above 16 MiB are read in 32 MiB chunks through
 * two pinned staging buffers, each chunk's copy overlapping the next chunk's
 * read; the buffers (64 MiB of pinned host memory) are allocated by the first
 * such call and held until the process exits, and concurrent file parses take
 * turns on them. */
int rtr_graph_create_from_escape_file(const char* path, int device, int flags, rtr_graph** out);

/* Parse an Escape edge-list file (first data line "n m", then m lines "u v";
 * '#' and blank lines skipped) into malloc'ed arrays released with rtr_free.
 * Replaces: loadGraph(path, g, 1, IOFormat::escape) (RTRex_Sequential/GraphIO.cpp:19-88);
 * returns RTR_ERR_IO when fewer than m edges are present (GraphIO.cpp:67-71). */
int rtr_load_escape(const char* path, int64_t* n, int64_t* m, int64_t** src, int64_t** dst);
void rtr_free(void* p);

/* The whole drop-in driver: load, decompose at eps on `device`, and write
 * <prefix><name>-{decomposition,stats,freq,cut}.txt.
 * Replaces: RTRex_CUDA main (RTRex_CUDA/main.cu:343-391) with prefix "RTRex-CUDA-",
 *           and RTRex main's decomposition output (RTRex.cpp:176-194) with "RTRex-". */
int rtr_run_file(const char* graph_path, const char* name, double eps, int device, const char* prefix, int flags);

/* rtr_run_file with the RTRex driver's mode e: with RTR_FLAG_EXPAND in flags it
 * also expands the clusters at `threshold` and writes
 * <prefix>expanded-<name>-{decomposition,stats,freq,cut,scores}.txt.
 * Replaces: RTRex <graph> <name> <eps> e <threshold> (RTRex.cpp:141-206). */
int rtr_run_file_ex(const char* graph_path, const char* name, double eps, int device, const char* prefix,
                    int flags, int64_t threshold);

#ifdef __cplusplus
}
#endif
#endif /* RTR_H */
