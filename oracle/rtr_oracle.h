/* Restated CPU oracle for the RTRExtractor decomposition path.
 *
 * TEST INFRASTRUCTURE ONLY: tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline use this library as the checker / CPU baseline.  The product
 * library (librtr.so) never links or calls it.
 *
 * Each function restates one reference function, in the same floating-point
 * operation order, with plain arrays in place of the ESCAPE structs:
 *   orc_build_csr      makeCSR + sortById        RTRex_Sequential/Graph.cpp:344-384, :201-205
 *   orc_partner        CGraph::getPartnerMap     RTRex_Sequential/Graph.cpp:320-340
 *   orc_count          commonNbr                 RTRex_Sequential/Escape/Decomposition.h:42-117
 *   orc_initial_clean  initialClean (mode s)     Decomposition.h:302-460 (+ deleteAndClean :147-283)
 *   orc_extract        disjointExtract loop      Decomposition.h:566-919 (+ populateStats :473-491)
 *   orc_expand         expandClusters            Decomposition.h:958-1008
 *   orc_cells_*        commonNbr, cell by cell   Decomposition.h:70-115 (rtr_cells.cpp)
 *   orc_nucleus        nucleus driver + nuclei   clustering/nucleus.cpp:12-81, Nucleus.h:125-565 (rtr_nucleus.cpp)
 *
 * Status bytes use the reference's characters: 'Y' alive, 'S' on the
 * deletion stack, 'N' deleted.  support[] is an integer companion the
 * reference does not keep: the number of live triangles on each directed edge.
 */
#ifndef RTR_ORACLE_H
#define RTR_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* makeCSR on the symmetrised list: 2m directed pairs sorted by (src,dst). */
int orc_build_csr(int64_t n, int64_t m, const int64_t* u, const int64_t* v,
                  int64_t* offsets /* n+1 */, int64_t* nbors /* 2m */);

/* Index of the reverse copy of every directed edge; returns the number of
 * edges whose reverse is missing (the reference prints an error for each). */
int64_t orc_partner(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t* partner);

/* Weighted triangle counting; perEdge/perVertex/support are overwritten. */
void orc_count(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
               double* perEdge, double* perVertex, uint32_t* support, int64_t* total);

/* Initial clean; status is written ('Y'/'N'), the weights are updated in place.
 * When trace != NULL, the index of every popped edge is appended to trace[]
 * and *trace_len receives the number of pops (caller sizes trace to m2). */
void orc_initial_clean(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
                       double eps, double* perEdge, double* perVertex, uint32_t* support,
                       int64_t* total, uint8_t* status, int64_t* trace, int64_t* trace_len);

/* Extraction from the cleaned state.  Clusters are reported in creation order:
 * cluster k has seed cl_seed[k], statistics cl_nv/cl_ne/cl_cut[k], and its
 * vertices are cl_vert[cl_off[k] .. cl_off[k+1]) in the order the reference's
 * unordered_set iterates them.  Arrays cl_seed/cl_nv/cl_ne/cl_cut are sized n,
 * cl_off n+1, cl_vert n.  Returns the number of clusters. */
int64_t orc_extract(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
                    double eps, double* perEdge, double* perVertex, uint32_t* support,
                    int64_t* total, uint8_t* status,
                    int64_t* cl_seed, int64_t* cl_nv, int64_t* cl_ne, int64_t* cl_cut,
                    int64_t* cl_off, int64_t* cl_vert);

/* expandClusters (Decomposition.h:958-1008) applied to the clusters of the last
 * orc_extract call (its member sets are kept with their container state).
 * Writes the same number of clusters, in the same order, with statistics
 * recomputed and members in set-iteration order (emptied singletons have no
 * members), and the singleton scores in ascending vertex order
 * (std::map<VertexIdx,double> iteration).  cl_* sized as for orc_extract,
 * sc_* sized n.  Returns the number of clusters. */
int64_t orc_expand(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t threshold,
                   int64_t* cl_nv, int64_t* cl_ne, int64_t* cl_cut, int64_t* cl_off, int64_t* cl_vert,
                   int64_t* n_scores, int64_t* sc_vertex, double* sc_value);

/* Per-cell restatement of commonNbr's folds (rtr_cells.cpp), for graphs too
 * large for orc_count: perEdge and support of the k directed slots slots[],
 * perVertex of the k vertices verts[] (outputs indexed like the samples), and
 * the triangle total.  Multi-threaded (OpenMP). */
void orc_cells_edge(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t k, const int64_t* slots,
                    double* perEdge, uint32_t* support);
void orc_cells_vertex(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t k, const int64_t* verts,
                      double* perVertex);
int64_t orc_count_total(int64_t n, const int64_t* offsets, const int64_t* nbors);

/* The nucleus (truss-hierarchy) path, nucleus.cpp:12-81 (rtr_nucleus.cpp):
 * returns the number of clusters; orc_nucleus_sizes / orc_nucleus_get copy
 * the result out (clusters in output order with id, C, n_vertices, n_edges,
 * parent and members in original labels; kappa per slot of the relabelled
 * CSR; that CSR; new -> old labels; which of the reference's fixed-size
 * arrays the input overruns, where the reference is undefined). */
int64_t orc_nucleus(int64_t n, const int64_t* offsets, const int64_t* nbors);
void orc_nucleus_sizes(int64_t* n_members, int64_t* m2, int64_t* overflow);
void orc_nucleus_get(int64_t* id, int64_t* c, int64_t* nv, int64_t* ne, int64_t* parent, int64_t* voff,
                     int64_t* vert, int64_t* kappa, int64_t* rel_off, int64_t* rel_nb, int64_t* inverse);

/* Counters of the reference's self-checks that print and continue
 * (Decomposition.h:158-170 and :273-277), accumulated since the last reset. */
void orc_selfcheck_counts(int64_t* missing_edge, int64_t* bad_status, int64_t* residual);
void orc_selfcheck_reset(void);

#ifdef __cplusplus
}
#endif
#endif
