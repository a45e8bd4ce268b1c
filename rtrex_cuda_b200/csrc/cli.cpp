// rtrex_b200: drop-in command line for the decomposition path.
//
//   rtrex_b200 <graph_file> <output_name> <eps> [gpu_device] [--prefix P] [--simplify] [--expand T]
//   rtrex_b200 --nucleus <graph_file> <output_file>
//
// Same positional arguments and outputs as RTRex_CUDA (RTRex_CUDA/main.cu:343-391):
// writes <P><output_name>-{decomposition,stats,freq,cut}.txt with P defaulting
// to "RTRex-CUDA-"; pass --prefix RTRex- for the sequential RTRex driver's names
// (RTRex_Sequential/clustering/RTRex.cpp:194); with that prefix the CLI also
// writes the RTRex driver's connected-components-<name>-* files and the
// amazon_cleaned_edges.txt survivor dump (RTRex.cpp:203-204, Decomposition.h:441-452).  --expand T is the
// RTRex driver's mode e with threshold T (RTRex.cpp:196-201): it adds
// <P>expanded-<output_name>-{decomposition,stats,freq,cut,scores}.txt.  Exit code 1 on any failure,
// as the reference exits 1 when the graph cannot be loaded.
#include "../../include/rtr.h"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

// rtrex_b200 --nucleus <graph_file> <output_file>: the reference's nucleus
// driver (RTRex_Sequential/clustering/nucleus.cpp:12-81) -- the truss hierarchy
// written to <output_file> in its format.
static int run_nucleus(const char* graph, const char* out)
{
    rtr_graph* g = nullptr;
    int rc = rtr_graph_create_from_escape_file(graph, 0, 0, &g);
    if (rc) return rc;
    printf("Loaded graph\n");
    int64_t k = 0;
    if (!(rc = rtr_nucleus(g, &k))) {
        printf("Compute nuclei\n%lld clusters\n", (long long)k);
        rc = rtr_write_nuclei(g, out);
    }
    rtr_graph_destroy(g);
    return rc;
}

int main(int argc, char** argv)
{
    if (argc == 4 && !strcmp(argv[1], "--nucleus")) {
        const int rc = run_nucleus(argv[2], argv[3]);
        if (rc != RTR_OK) {
            fprintf(stderr, "Error: %s\n", rtr_last_error());
            return 1;
        }
        return 0;
    }
    std::string prefix = "RTRex-CUDA-";
    int flags = 0;
    long long threshold = 0;
    const char* pos[4] = {nullptr, nullptr, nullptr, nullptr};
    int npos = 0;
    for (int i = 1; i < argc; ++i) {
        if (!strcmp(argv[i], "--prefix") && i + 1 < argc) {
            prefix = argv[++i];
            if (prefix == "RTRex-") flags |= RTR_FLAG_RTREX_OUTPUTS;
        } else if (!strcmp(argv[i], "--simplify")) {
            flags |= RTR_FLAG_SIMPLIFY;
        } else if (!strcmp(argv[i], "--expand") && i + 1 < argc) {
            flags |= RTR_FLAG_EXPAND;
            threshold = atoll(argv[++i]);
        } else if (npos < 4) {
            pos[npos++] = argv[i];
        }
    }
    if (npos < 3) {
        printf("Usage: %s <graph_file> <output_name> <eps> [gpu_device] [--prefix P] [--simplify] [--expand T]\n",
               argv[0]);
        return 1;
    }
    const double eps = atof(pos[2]);
    const int device = npos >= 4 ? atoi(pos[3]) : 0;
    printf("eps = %f\n", eps);
    if (flags & RTR_FLAG_EXPAND) printf("threshold = %lld\n", threshold);
    const int rc = rtr_run_file_ex(pos[0], pos[1], eps, device, prefix.c_str(), flags, threshold);
    if (rc != RTR_OK) {
        fprintf(stderr, "Error: %s\n", rtr_last_error());
        return 1;
    }
    printf("[Main] Done.\n");
    return 0;
}
