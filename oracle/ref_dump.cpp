// Golden-vector dumper for the RTRExtractor decomposition path.
//
// TEST INFRASTRUCTURE ONLY. This harness is compiled against the reference's
// own header-only algorithm (RTRex_Sequential/Escape/Decomposition.h) and its
// loader / CSR builder (RTRex_Sequential/GraphIO.cpp, Graph.cpp) by
// oracle/Makefile, and writes each stage's state as raw little-endian arrays so
// the restated oracle (rtr_oracle.cpp) and the CUDA path can be pinned against
// the reference bit for bit.  It is never linked into the product.
//
// Usage: rtr_ref_dump <escape-graph-file> <eps> <out-dir> [threshold ...]
//
// Files written into <out-dir>:
//   csr_offsets.i64, csr_nbors.i64          makeCSR result  (Graph.cpp:344-384)
//   count_perEdge.f64, count_perVertex.f64  commonNbr        (Decomposition.h:42-117)
//   count_total.i64
//   clean_status.u8, clean_perEdge.f64,     initialClean     (Decomposition.h:302-460)
//   clean_perVertex.f64, clean_total.i64
//   clusters.txt                            disjointExtract  (Decomposition.h:538-940)
//       one line per cluster in creation order:
//       "<nVertices> <nEdges> <cut> : <v> <v> ..."  (vertices in set iteration order)
//   expanded_<t>.txt, scores_<t>.txt        expandClusters   (Decomposition.h:958-1008)
//       for each threshold argument t, as the RTRex driver calls it in mode e
//       (RTRex.cpp:196-201): the expanded clusters in the same line format and
//       the singleton scores as "<v> <score as %a>" in map order
#include "Escape/GraphIO.h"
#include "Escape/Graph.h"
#include "Escape/Decomposition.h"

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include <unistd.h>

using namespace Escape;

static void dump(const std::string& path, const void* p, size_t bytes)
{
    FILE* f = fopen(path.c_str(), "wb");
    if (!f) { fprintf(stderr, "cannot write %s\n", path.c_str()); exit(2); }
    if (bytes && fwrite(p, 1, bytes, f) != bytes) { fprintf(stderr, "short write %s\n", path.c_str()); exit(2); }
    fclose(f);
}

int main(int argc, char** argv)
{
    if (argc < 4) { fprintf(stderr, "usage: %s <graph> <eps> <outdir>\n", argv[0]); return 1; }
    const double eps = atof(argv[2]);
    std::string out(argv[3]);
    std::string graphPath(argv[1]);
    if (graphPath[0] != '/') {
        char cwd[4096];
        if (getcwd(cwd, sizeof cwd)) graphPath = std::string(cwd) + "/" + graphPath;
    }
    // initialClean writes a debug dump into the working directory.
    if (chdir(out.c_str()) != 0) { fprintf(stderr, "cannot chdir %s\n", out.c_str()); return 1; }

    Graph g;
    if (loadGraph(graphPath.c_str(), g, 1, IOFormat::escape)) return 1;
    CGraph cg = makeCSR(g);
    const int64_t n = cg.nVertices, m2 = cg.nEdges;
    dump("csr_offsets.i64", cg.offsets, sizeof(int64_t) * (n + 1));
    dump("csr_nbors.i64", cg.nbors, sizeof(int64_t) * m2);

    // Stage 1: commonNbr.
    WeightedTriangleInfo tri = commonNbr(&cg);
    dump("count_perEdge.f64", tri.perEdge, sizeof(double) * m2);
    dump("count_perVertex.f64", tri.perVertex, sizeof(double) * n);
    dump("count_total.i64", &tri.total, sizeof(int64_t));

    // Stage 2: initialClean (mutates tri in place).
    char* status = initialClean(&cg, &tri, eps, false);
    dump("clean_status.u8", status, m2);
    dump("clean_perEdge.f64", tri.perEdge, sizeof(double) * m2);
    dump("clean_perVertex.f64", tri.perVertex, sizeof(double) * n);
    dump("clean_total.i64", &tri.total, sizeof(int64_t));
    delete[] status;
    delete[] tri.perEdge;
    delete[] tri.perVertex;

    // Stage 3: the full disjointExtract (recounts and recleans internally).
    std::map<VertexIdx, VertexIdx> cmap;
    std::vector<Cluster> dec = disjointExtract(&cg, eps, cmap, false);
    FILE* f = fopen("clusters.txt", "w");
    for (const Cluster& c : dec) {
        fprintf(f, "%" PRId64 " %" PRId64 " %" PRId64 " :", c.nVertices, c.nEdges, c.cut);
        for (VertexIdx v : c.vertices) fprintf(f, " %" PRId64, v);
        fprintf(f, "\n");
    }
    fclose(f);

    for (int a = 4; a < argc; ++a) {
        const int thr = atoi(argv[a]);
        std::map<VertexIdx, double> scores;
        std::vector<Cluster> ex = expandClusters(&cg, dec, cmap, thr, scores);
        FILE* fe = fopen(("expanded_" + std::to_string(thr) + ".txt").c_str(), "w");
        for (const Cluster& c : ex) {
            fprintf(fe, "%" PRId64 " %" PRId64 " %" PRId64 " :", c.nVertices, c.nEdges, c.cut);
            for (VertexIdx v : c.vertices) fprintf(fe, " %" PRId64, v);
            fprintf(fe, "\n");
        }
        fclose(fe);
        FILE* fs = fopen(("scores_" + std::to_string(thr) + ".txt").c_str(), "w");
        for (const auto& e : scores) fprintf(fs, "%" PRId64 " %a\n", e.first, e.second);
        fclose(fs);
    }
    return 0;
}
