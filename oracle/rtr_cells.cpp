// Per-cell restatement of commonNbr's folds, for graphs too large to run the
// whole oracle on (R-MAT scale 22 and beyond).
//
// TEST INFRASTRUCTURE ONLY (tests/ and bench.py's checks); the product library
// never links it.
//
// commonNbr (RTRex_Sequential/Escape/Decomposition.h:42-117) meets every
// triangle once, in lexicographic order of its sorted triple, and adds its
// weight 1/double(du*dv*dw) (:97) to the cells of its edges and vertices.  So:
//   perEdge[(u,v)]  = left fold, over z in N(u) & N(v) ascending, of the weight
//   perVertex[x]    = left fold over y in N(x) ascending, then over
//                     z in N(x) & N(y), z > y ascending, of the weight
// which makes every cell a function of the CSR alone: a sample of cells can be
// recomputed without the rest.  orc_count (rtr_oracle.cpp) is the whole-graph
// restatement these are checked against on graphs it can finish.
#include "rtr_oracle.h"

#include <algorithm>
#include <cstdint>
#include <vector>

namespace {

// Common neighbours of two ascending rows in ascending order: f(z).
template <typename F>
void common(const int64_t* a, int64_t la, const int64_t* b, int64_t lb, F&& f)
{
    if (la == 0 || lb == 0) return;
    if (la > lb) {
        std::swap(a, b);
        std::swap(la, lb);
    }
    if (la * 16 < lb) {  // short row looked up in the long one
        const int64_t* lo = b;
        const int64_t* end = b + lb;
        for (int64_t p = 0; p < la && lo < end; ++p) {
            lo = std::lower_bound(lo, end, a[p]);
            if (lo < end && *lo == a[p]) {
                f(a[p]);
                ++lo;
            }
        }
        return;
    }
    int64_t i = 0, j = 0;
    while (i < la && j < lb) {
        if (a[i] < b[j]) ++i;
        else if (a[i] > b[j]) ++j;
        else {
            f(a[i]);
            ++i;
            ++j;
        }
    }
}

}  // namespace

extern "C" {

void orc_cells_edge(int64_t n, const int64_t* off, const int64_t* nb, int64_t k, const int64_t* slots, double* pe,
                    uint32_t* sup)
{
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t s = 0; s < k; ++s) {
        const int64_t i = slots[s];
        const int64_t u = (int64_t)(std::upper_bound(off, off + n + 1, i) - off) - 1;  // the row holding slot i
        const int64_t v = nb[i];
        const int64_t du = off[u + 1] - off[u], dv = off[v + 1] - off[v];
        double acc = 0;
        uint32_t c = 0;
        common(nb + off[u], du, nb + off[v], dv, [&](int64_t z) {
            const int64_t dz = off[z + 1] - off[z];
            acc += 1 / double(du * dv * dz);
            ++c;
        });
        pe[s] = acc;
        sup[s] = c;
    }
}

void orc_cells_vertex(int64_t n, const int64_t* off, const int64_t* nb, int64_t k, const int64_t* verts, double* pv)
{
    (void)n;
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t s = 0; s < k; ++s) {
        const int64_t x = verts[s];
        const int64_t dx = off[x + 1] - off[x];
        double acc = 0;
        for (int64_t i = off[x]; i < off[x + 1]; ++i) {
            const int64_t y = nb[i];
            const int64_t dy = off[y + 1] - off[y];
            // z > y: the part of N(x) after y, against N(y)
            common(nb + i + 1, off[x + 1] - i - 1, nb + off[y], dy, [&](int64_t z) {
                const int64_t dz = off[z + 1] - off[z];
                acc += 1 / double(dx * dy * dz);
            });
        }
        pv[s] = acc;
    }
}

int64_t orc_count_total(int64_t n, const int64_t* off, const int64_t* nb)
{
    // orient every edge from the (degree, id)-smaller end; count each triangle once
    auto before = [&](int64_t a, int64_t b) {
        const int64_t da = off[a + 1] - off[a], db = off[b + 1] - off[b];
        return da < db || (da == db && a < b);
    };
    std::vector<int64_t> ooff(n + 1, 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < n; ++u) {
        int64_t c = 0;
        for (int64_t p = off[u]; p < off[u + 1]; ++p) c += before(u, nb[p]) ? 1 : 0;
        ooff[u + 1] = c;
    }
    for (int64_t u = 0; u < n; ++u) ooff[u + 1] += ooff[u];
    std::vector<int64_t> onb((size_t)std::max<int64_t>(1, ooff[n]));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int64_t u = 0; u < n; ++u) {
        int64_t w = ooff[u];
        for (int64_t p = off[u]; p < off[u + 1]; ++p)
            if (before(u, nb[p])) onb[w++] = nb[p];
    }
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : total)
    for (int64_t u = 0; u < n; ++u)
        for (int64_t p = ooff[u]; p < ooff[u + 1]; ++p) {
            const int64_t v = onb[p];
            common(onb.data() + ooff[u], ooff[u + 1] - ooff[u], onb.data() + ooff[v], ooff[v + 1] - ooff[v],
                   [&](int64_t) { ++total; });
        }
    return total;
}

}  // extern "C"
