// Host side of the drop-in surface: the Escape edge-list parser, the
// decomposition writer and the whole-file driver.
#include "../../include/rtr.h"
#include "escape_text.h"

#include <algorithm>
#include <cerrno>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>

namespace rtr {
void set_error(const char* fmt, ...);
}

namespace {

struct ClusterView {
    int64_t nv, ne, idx;
};

}  // namespace

extern "C" {

// loadGraph_Escape (RTRex_Sequential/GraphIO.cpp:19-74): comment lines start
// with '#', blank lines are skipped, the first data line is "n m", every other
// data line is one undirected pair.
int rtr_load_escape(const char* path, int64_t* n_out, int64_t* m_out, int64_t** src_out, int64_t** dst_out)
{
    if (!path || !n_out || !m_out || !src_out || !dst_out) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    *src_out = *dst_out = nullptr;
    FILE* f = fopen(path, "rb");
    if (!f) {
        rtr::set_error("could not open file %s", path);
        return RTR_ERR_IO;
    }
    std::vector<char> buf;
    {
        fseek(f, 0, SEEK_END);
        long sz = ftell(f);
        fseek(f, 0, SEEK_SET);
        buf.resize(sz > 0 ? (size_t)sz : 0);
        if (sz > 0 && fread(buf.data(), 1, (size_t)sz, f) != (size_t)sz) {
            fclose(f);
            rtr::set_error("short read on %s", path);
            return RTR_ERR_IO;
        }
        fclose(f);
    }
    const char* p = buf.data();
    const char* end = p + buf.size();
    bool have_header = false;
    int64_t n = 0, m = 0, got = 0, lineno = 0;
    int64_t *src = nullptr, *dst = nullptr;
    while (p < end) {
        const char* nl = (const char*)memchr(p, '\n', (size_t)(end - p));
        const char* le = nl ? nl : end;
        ++lineno;
        int64_t a = 0, b = 0;
        const int kind = rtr::esc_line(p, le, &a, &b);
        if (kind != 0) {
            if (kind == 2) {
                free(src);
                free(dst);
                rtr::set_error("%s:%lld: expected two integers", path, (long long)lineno);
                return RTR_ERR_IO;
            }
            if (!have_header) {
                have_header = true;
                n = a;
                m = b;
                if (n < 0 || m < 0) {
                    rtr::set_error("%s: negative header values", path);
                    return RTR_ERR_IO;
                }
                src = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
                dst = (int64_t*)malloc(sizeof(int64_t) * (size_t)(m > 0 ? m : 1));
                if (!src || !dst) {
                    free(src);
                    free(dst);
                    rtr::set_error("host allocation failed for %lld edges", (long long)m);
                    return RTR_ERR_IO;
                }
            } else if (got < m) {
                src[got] = a;
                dst[got] = b;
                ++got;
            }
        }
        p = nl ? nl + 1 : end;
    }
    if (!have_header) {
        rtr::set_error("%s: no header line", path);
        return RTR_ERR_IO;
    }
    if (got < m) {
        free(src);
        free(dst);
        // the reference reports edges counted in both directions (GraphIO.cpp:67-71)
        rtr::set_error("expected %" PRId64 " edges, only got %" PRId64, 2 * m, 2 * got);
        return RTR_ERR_IO;
    }
    *n_out = n;
    *m_out = m;
    *src_out = src;
    *dst_out = dst;
    return RTR_OK;
}

// printDecomposition (RTRex_Sequential/clustering/RTRex.cpp:19-118).  Clusters
// are ranked with std::sort on the size comparator from creation order, as the
// reference does, so equal-size clusters land in the same lines; members are
// written in the reference's set-iteration order.
static int write_clusters(const char* name_c, int64_t n, const std::vector<int64_t>& off,
                          const std::vector<int64_t>& nb, int64_t k, const std::vector<int64_t>& nv,
                          const std::vector<int64_t>& ne, const std::vector<int64_t>& coff,
                          const std::vector<int64_t>& vert, const std::vector<int64_t>& cluster_of)
{
    const std::string name(name_c);
    printf("\n--------------------------------------------\n");
    printf("Generating details of %s decomposition\n", name.c_str());
    FILE* f = fopen((name + "-decomposition.txt").c_str(), "w");
    FILE* fs = fopen((name + "-stats.txt").c_str(), "w");
    FILE* fcut = fopen((name + "-cut.txt").c_str(), "w");
    FILE* ffreq = fopen((name + "-freq.txt").c_str(), "w");
    if (!f || !fs || !fcut || !ffreq) {
        if (f) fclose(f);
        if (fs) fclose(fs);
        if (fcut) fclose(fcut);
        if (ffreq) fclose(ffreq);
        rtr::set_error("could not write the output files for %s", name.c_str());
        return RTR_ERR_IO;
    }
    std::vector<ClusterView> cl(k);
    for (int64_t i = 0; i < k; ++i) cl[i] = ClusterView{nv[i], ne[i], i};
    std::sort(cl.begin(), cl.end(), [](const ClusterView& a, const ClusterView& b) { return a.nv > b.nv; });
    std::vector<int64_t> freq(n + 1, 0);
    int64_t maxsize = 0, total_clustered = 0, total_internal = 0;
    std::string line;
    for (int64_t r = 0; r < k; ++r) {
        const ClusterView& c = cl[r];
        line.clear();
        char tmp[32];
        for (int64_t p = coff[c.idx]; p < coff[c.idx + 1]; ++p) {
            int len = snprintf(tmp, sizeof tmp, "%" PRId64 " ", vert[p]);
            line.append(tmp, (size_t)len);
        }
        line.push_back('\n');
        fwrite(line.data(), 1, line.size(), f);
        if (c.nv > maxsize) maxsize = c.nv;
        freq[c.nv]++;
        if (c.nv != 1) {
            const double density = 2 * (c.ne) / ((double)(c.nv) * (double)(c.nv - 1));
            total_clustered += c.nv;
            total_internal += c.ne;
            fprintf(fs, "%" PRId64 " %.2f\n", c.nv, density);
        }
        for (int64_t p = coff[c.idx]; p < coff[c.idx + 1]; ++p) {
            const int64_t vtx = vert[p];
            for (int64_t j = off[vtx]; j < off[vtx + 1]; ++j) {
                const int64_t nbr = nb[j];
                if (nbr < vtx) continue;
                if (cluster_of[nbr] != c.idx) fprintf(fcut, "%" PRId64 " %" PRId64 "\n", vtx, nbr);
            }
        }
    }
    printf("Non-trivial clustered vertices: %" PRId64 "\n", total_clustered);
    printf("Edges inside clusters: %" PRId64 "\n", total_internal);
    printf("\n--------------------------------------------\n");
    for (int64_t i = 0; i < maxsize + 1; ++i)
        fprintf(ffreq, "Size = %" PRId64 ", freq = %" PRId64 ", total vertices = %" PRId64 "\n", i, freq[i],
                i * freq[i]);
    fclose(fs);
    fclose(ffreq);
    fclose(fcut);
    fclose(f);
    return RTR_OK;
}

int rtr_write_decomposition(const rtr_graph* g, const char* name_c)
{
    if (!g || !name_c) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    int64_t n = 0, m = 0, k = 0;
    int rc = rtr_graph_info(g, &n, &m);
    if (rc) return rc;
    std::vector<int64_t> off(n + 1), nb(2 * m), cluster_of(n);
    if ((rc = rtr_get_csr(g, off.data(), nb.data()))) return rc;
    if ((rc = rtr_get_cluster_of(g, cluster_of.data()))) return rc;
    if ((rc = rtr_num_clusters(g, &k))) return rc;
    std::vector<int64_t> seed(k), nv(k), ne(k), cut(k), coff(k + 1), vert(n);
    if ((rc = rtr_get_clusters(g, seed.data(), nv.data(), ne.data(), cut.data(), coff.data(), vert.data())))
        return rc;
    return write_clusters(name_c, n, off, nb, k, nv, ne, coff, vert, cluster_of);
}

int rtr_write_expanded(const rtr_graph* g, const char* name_c)
{
    if (!g || !name_c) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    int64_t n = 0, m = 0, k = 0;
    int rc = rtr_graph_info(g, &n, &m);
    if (rc) return rc;
    if ((rc = rtr_num_clusters(g, &k))) return rc;
    std::vector<int64_t> off(n + 1), nb(2 * m), cluster_of(n);
    std::vector<int64_t> nv(k), ne(k), cut(k), coff(k + 1), vert(n);
    if ((rc = rtr_get_csr(g, off.data(), nb.data()))) return rc;
    if ((rc = rtr_get_expanded(g, nv.data(), ne.data(), cut.data(), coff.data(), vert.data(), cluster_of.data())))
        return rc;
    if ((rc = write_clusters(name_c, n, off, nb, k, nv, ne, coff, vert, cluster_of))) return rc;
    // printScores (RTRex.cpp:120-135): header line, then the std::map in key order.
    int64_t ns = 0;
    if ((rc = rtr_get_scores(g, &ns, nullptr, nullptr))) return rc;
    std::vector<int64_t> sv(ns);
    std::vector<double> sx(ns);
    if ((rc = rtr_get_scores(g, &ns, sv.data(), sx.data()))) return rc;
    printf("\n--------------------------------------------\n");
    printf("generating singleton scores\n");
    const std::string name(name_c);
    FILE* f = fopen((name + "-scores.txt").c_str(), "w");
    if (!f) {
        rtr::set_error("could not write %s-scores.txt", name.c_str());
        return RTR_ERR_IO;
    }
    fprintf(f, "Vertex,Score\n");
    for (int64_t i = 0; i < ns; ++i) fprintf(f, "%" PRId64 ",%f\n", sv[i], sx[i]);
    fclose(f);
    printf("\n--------------------------------------------\n");
    return RTR_OK;
}

// The components' member order: the reference inserts a component's vertices
// into an unordered_set in discovery order (Decomposition.h:1038-1056) and
// prints them in that set's iteration order, so the writer replays the inserts.
int rtr_write_components(const rtr_graph* g, const char* name_c)
{
    if (!g || !name_c) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    int64_t n = 0, m = 0;
    int rc = rtr_graph_info(g, &n, &m);
    if (rc) return rc;
    std::vector<int64_t> off(n + 1), nb(2 * m), disc(n);
    if ((rc = rtr_get_csr(g, off.data(), nb.data()))) return rc;
    int64_t k = 0;
    {
        // number of components = entries of the offsets array minus one
        std::vector<int64_t> tmp(n + 2, -1);
        if ((rc = rtr_get_components(g, tmp.data(), disc.data()))) return rc;
        while (k < n && tmp[k + 1] > tmp[k]) ++k;
        std::vector<int64_t> coff(tmp.begin(), tmp.begin() + k + 1);
        std::vector<int64_t> nv(k), ne(k), vert(n), cluster_of(n);
        int64_t w = 0;
        for (int64_t c = 0; c < k; ++c) {
            std::unordered_set<int64_t> members;
            for (int64_t p = coff[c]; p < coff[c + 1]; ++p) members.insert(disc[p]);
            int64_t deg_sum = 0;
            const int64_t start = w;
            for (int64_t v : members) {
                vert[w++] = v;
                cluster_of[v] = c;
                deg_sum += off[v + 1] - off[v];
            }
            nv[c] = w - start;
            ne[c] = deg_sum / 2;  // populateStats: every neighbour of a component member is inside it
        }
        return write_clusters(name_c, n, off, nb, k, nv, ne, coff, vert, cluster_of);
    }
}

// The survivor dump initialClean writes into the working directory
// (Decomposition.h:416-455): the 'Y' edges u<v, sorted.
static int write_cleaned_edges(const rtr_graph* g)
{
    int64_t n = 0, m = 0;
    int rc = rtr_graph_info(g, &n, &m);
    if (rc) return rc;
    std::vector<int64_t> off(n + 1), nb(2 * m + 1);
    std::vector<uint8_t> st(2 * m + 1);
    if ((rc = rtr_get_csr(g, off.data(), nb.data()))) return rc;
    if ((rc = rtr_get_status(g, st.data()))) return rc;
    int64_t remaining = 0;
    FILE* f = fopen("amazon_cleaned_edges.txt", "w");
    for (int64_t u = 0; u < n; ++u)
        for (int64_t j = off[u]; j < off[u + 1]; ++j)
            if (st[j] == 'Y') {
                ++remaining;
                if (f && u < nb[j]) fprintf(f, "%" PRId64 " %" PRId64 "\n", u, nb[j]);
            }
    if (f) fclose(f);
    printf("Edges remaining after initialClean (Directed): %" PRId64 "\n", remaining);
    printf("Edges remaining after initialClean (Undirected): %" PRId64 "\n", remaining / 2);
    return RTR_OK;
}

int rtr_run_file(const char* graph_path, const char* name, double eps, int device, const char* prefix, int flags)
{
    return rtr_run_file_ex(graph_path, name, eps, device, prefix, flags & ~RTR_FLAG_EXPAND, 0);
}

int rtr_run_file_ex(const char* graph_path, const char* name, double eps, int device, const char* prefix,
                    int flags, int64_t threshold)
{
    if (!graph_path || !name) {
        rtr::set_error("null argument");
        return RTR_ERR_ARG;
    }
    // the text is parsed on the device and the CSR built there
    rtr_graph* g = nullptr;
    int rc = rtr_graph_create_from_escape_file(graph_path, device, flags, &g);
    if (rc) return rc;
    int64_t n = 0, m = 0;
    rtr_graph_info(g, &n, &m);
    printf("Loaded graph\nVertices = %" PRId64 "\nEdges = %" PRId64 "\n", n, m);
    int64_t total = 0, left = 0, ncl = 0;
    if (!(rc = rtr_count(g, &total))) {
        printf("Total triangles = %" PRId64 "\n", total);
        if (!(rc = rtr_clean(g, eps, &left))) {
            printf("Total triangle count, post cleaning = %" PRId64 "\n", left);
            if (flags & RTR_FLAG_RTREX_OUTPUTS) rc = write_cleaned_edges(g);
            if (!rc) rc = rtr_extract(g, &ncl);
        }
    }
    if (!rc) {
        double ms[4];
        rtr_get_stats(g, ms, nullptr, nullptr);
        printf("Time for getting the weights: %gs \n", ms[1] / 1e3);
        printf("Time for the initial clean: %gs \n", ms[2] / 1e3);
        printf("Time for getting the clusters: %gs \n", ms[3] / 1e3);
        printf("Total clusters extracted: %" PRId64 "\n", ncl);
        rc = rtr_write_decomposition(g, (std::string(prefix ? prefix : "") + name).c_str());
    }
    if (!rc && (flags & RTR_FLAG_EXPAND)) {
        int64_t nsc = 0;
        rc = rtr_expand(g, threshold, &nsc);
        if (!rc) rc = rtr_write_expanded(g, (std::string(prefix ? prefix : "") + "expanded-" + name).c_str());
    }
    if (!rc && (flags & RTR_FLAG_RTREX_OUTPUTS)) {
        int64_t ncomp = 0;
        rc = rtr_connected_components(g, &ncomp);
        if (!rc) rc = rtr_write_components(g, (std::string("connected-components-") + name).c_str());
    }
    rtr_graph_destroy(g);
    return rc;
}

}  // extern "C"
