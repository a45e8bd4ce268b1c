// Restated CPU oracle for the RTRExtractor decomposition path.
//
// TEST INFRASTRUCTURE ONLY (see rtr_oracle.h).  This is a sequential
// restatement of the reference's algorithm that keeps its floating-point
// operation order, its LIFO deletion stack and its container iteration orders
// (std::set for the two-hop candidates, std::unordered_set for cluster members,
// std::sort for the candidate ranking), so that it produces the reference's
// results bit for bit.  It is pinned against the reference itself
// (oracle/_ref/rtr_ref_dump) by tests/test_oracle.py and the committed
// fixtures under tests/golden/.
#include "rtr_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <set>
#include <stack>
#include <unordered_set>
#include <utility>
#include <vector>

namespace {

struct Csr {
    int64_t n;
    const int64_t* off;
    const int64_t* nb;
    const int64_t* partner;
    int64_t deg(int64_t v) const { return off[v + 1] - off[v]; }
    // CGraph::getEdgeBinary, RTRex_Sequential/Graph.cpp:130-149.
    int64_t find(int64_t v1, int64_t v2) const
    {
        if (v1 >= n) return -1;
        int64_t lo = off[v1], hi = off[v1 + 1] - 1;
        while (lo <= hi) {
            int64_t mid = (lo + hi) / 2;
            if (nb[mid] == v2) return mid;
            if (nb[mid] > v2) hi = mid - 1;
            else lo = mid + 1;
        }
        return -1;
    }
};

struct Pr {
    int64_t first, second;
};

int64_t g_missing = 0, g_badstatus = 0, g_residual = 0;

// The member sets of the last orc_extract call, in creation order, kept as the
// containers themselves: expandClusters continues inserting into them, and the
// iteration order after those inserts depends on each set's bucket state.
std::vector<std::unordered_set<int64_t>> g_last_sets;

// deleteAndClean, Decomposition.h:147-283.  Pops the LIFO stack; every popped
// edge removes its live triangles (no 'N' edge), subtracting the triangle
// weight from the six directed-edge cells and three vertex cells, and pushes
// the (lower,w)/(higher,w) edges that fall below eps * 1/(d*d).
void delete_and_clean(const Csr& g, uint8_t* st, double* pe, double* pv, uint32_t* sup,
                      int64_t* total, std::stack<Pr>& todo, double eps,
                      int64_t* trace, int64_t* trace_len)
{
    while (!todo.empty()) {
        Pr e = todo.top();
        todo.pop();
        const int64_t u = e.first, v = e.second;
        const int64_t loc_uv = g.find(u, v);
        if (loc_uv == -1) { ++g_missing; continue; }
        const int64_t part_uv = g.partner[loc_uv];
        if (st[loc_uv] != 'S' || st[part_uv] != 'S') ++g_badstatus;
        if (trace) trace[(*trace_len)++] = loc_uv;

        const int64_t degu = g.deg(u), degv = g.deg(v);
        const int64_t lower = (degu < degv) ? u : v;
        const int64_t higher = (degu < degv) ? v : u;
        const int64_t deglower = (degu < degv) ? degu : degv;
        const int64_t deghigher = (degu < degv) ? degv : degu;

        for (int64_t j = g.off[lower]; j < g.off[lower + 1]; ++j) {
            if (st[j] == 'N') continue;
            const int64_t w = g.nb[j];
            if (w == u || w == v) continue;
            const int64_t loc_hw = g.find(higher, w);
            if (loc_hw == -1) continue;
            if (st[loc_hw] == 'N') continue;
            const int64_t part_j = g.partner[j];
            const int64_t part_hw = g.partner[loc_hw];
            const int64_t degw = g.deg(w);
            const double wgt = 1 / double(degu * degv * degw);
            pe[loc_uv] -= wgt;
            pe[j] -= wgt;
            pe[loc_hw] -= wgt;
            pe[part_uv] -= wgt;
            pe[part_j] -= wgt;
            pe[part_hw] -= wgt;
            pv[u] -= wgt;
            pv[v] -= wgt;
            pv[w] -= wgt;
            sup[loc_uv]--; sup[j]--; sup[loc_hw]--;
            sup[part_uv]--; sup[part_j]--; sup[part_hw]--;
            (*total)--;
            double ew = 1 / double(deglower * degw);
            if (st[j] != 'S' && pe[j] < eps * ew) {
                todo.push(Pr{lower, w});
                st[j] = 'S';
                st[part_j] = 'S';
            }
            ew = 1 / double(deghigher * degw);
            if (st[loc_hw] != 'S' && pe[loc_hw] < eps * ew) {
                todo.push(Pr{higher, w});
                st[loc_hw] = 'S';
                st[part_hw] = 'S';
            }
        }
        if (std::fabs(pe[loc_uv]) > 1 / double(g.n) || std::fabs(pe[part_uv]) > 1 / double(g.n))
            ++g_residual;
        st[loc_uv] = 'N';
        st[part_uv] = 'N';
    }
}

}  // namespace

extern "C" {

// makeCSR, Graph.cpp:344-384: sort the (src,dst) pairs of the symmetrised list,
// compress the sources into offsets, then sort each adjacency list.
int orc_build_csr(int64_t n, int64_t m, const int64_t* u, const int64_t* v, int64_t* offsets, int64_t* nbors)
{
    std::vector<std::pair<int64_t, int64_t>> e;
    e.reserve(2 * m);
    for (int64_t i = 0; i < m; ++i) {  // GraphIO.cpp:53-62 stores (u,v) then (v,u)
        e.push_back({u[i], v[i]});
        e.push_back({v[i], u[i]});
    }
    std::sort(e.begin(), e.end());
    for (int64_t i = 0; i < 2 * m; ++i) {
        if (e[i].first < 0 || e[i].first >= n || e[i].second < 0 || e[i].second >= n) return -1;
        nbors[i] = e[i].second;
    }
    int64_t cv = 0;
    for (int64_t i = 0; i < 2 * m; ++i)
        while (cv <= e[i].first) offsets[cv++] = i;
    while (cv <= n) offsets[cv++] = 2 * m;
    return 0;
}

// CGraph::getPartnerMap, Graph.cpp:320-340.
int64_t orc_partner(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t* partner)
{
    Csr g{n, offsets, nbors, nullptr};
    int64_t bad = 0;
    for (int64_t u = 0; u < n; ++u)
        for (int64_t i = offsets[u]; i < offsets[u + 1]; ++i) {
            partner[i] = g.find(nbors[i], u);
            if (partner[i] == -1) ++bad;
        }
    return bad;
}

// commonNbr, Decomposition.h:42-117.  Each triangle is found once, from its
// smallest vertex u and edge (u,v) with v the middle vertex, scanning the
// lower-degree endpoint's list and binary-searching the other.
void orc_count(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
               double* pe, double* pv, uint32_t* sup, int64_t* total)
{
    Csr g{n, offsets, nbors, partner};
    const int64_t m2 = offsets[n];
    for (int64_t v = 0; v < n; ++v) pv[v] = 0;
    for (int64_t j = 0; j < m2; ++j) { pe[j] = 0; sup[j] = 0; }
    *total = 0;
    for (int64_t u = 0; u < n; ++u)
        for (int64_t i = offsets[u]; i < offsets[u + 1]; ++i) {
            const int64_t v = nbors[i];
            const int64_t degu = g.deg(u), degv = g.deg(v);
            if (u > v) continue;
            const int64_t lower = (degu < degv) ? u : v;
            const int64_t higher = (degu < degv) ? v : u;
            for (int64_t j = offsets[lower]; j < offsets[lower + 1]; ++j) {
                const int64_t w = nbors[j];
                if (w <= u || w <= v) continue;
                const int64_t loc = g.find(higher, w);
                if (loc == -1) continue;
                const int64_t degw = g.deg(w);
                const double wgt = 1 / double(degu * degv * degw);
                (*total)++;
                pe[i] += wgt;
                pe[partner[i]] += wgt;
                pe[j] += wgt;
                pe[partner[j]] += wgt;
                pe[loc] += wgt;
                pe[partner[loc]] += wgt;
                pv[u] += wgt;
                pv[v] += wgt;
                pv[w] += wgt;
                sup[i]++; sup[partner[i]]++; sup[j]++; sup[partner[j]]++; sup[loc]++; sup[partner[loc]]++;
            }
        }
}

// initialClean, Decomposition.h:302-460 (sequential seeding, :378-405).
void orc_initial_clean(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
                       double eps, double* pe, double* pv, uint32_t* sup, int64_t* total,
                       uint8_t* st, int64_t* trace, int64_t* trace_len)
{
    Csr g{n, offsets, nbors, partner};
    const int64_t m2 = offsets[n];
    for (int64_t j = 0; j < m2; ++j) st[j] = 'Y';
    if (trace_len) *trace_len = 0;
    std::stack<Pr> todo;
    for (int64_t u = 0; u < n; ++u)
        for (int64_t i = offsets[u]; i < offsets[u + 1]; ++i) {
            const int64_t v = nbors[i];
            const int64_t degu = g.deg(u), degv = g.deg(v);
            if (u > v) continue;
            const double ew = 1 / double(degu * degv);
            if (st[i] != 'S' && pe[i] < eps * ew) {
                todo.push(Pr{u, v});
                st[i] = 'S';
                st[partner[i]] = 'S';
            }
        }
    delete_and_clean(g, st, pe, pv, sup, total, todo, eps, trace, trace_len);
}

// disjointExtract's seed loop, Decomposition.h:566-919 (sequential inner loop,
// :728-805), with populateStats (:473-491) for the cluster statistics.
int64_t orc_extract(int64_t n, const int64_t* offsets, const int64_t* nbors, const int64_t* partner,
                    double eps, double* pe, double* pv, uint32_t* sup, int64_t* total, uint8_t* st,
                    int64_t* cl_seed, int64_t* cl_nv, int64_t* cl_ne, int64_t* cl_cut,
                    int64_t* cl_off, int64_t* cl_vert)
{
    Csr g{n, offsets, nbors, partner};
    // Seeds by (degree asc, id asc): pairCompareSecond, Graph.cpp:40-45.
    std::vector<Pr> order(n);
    for (int64_t i = 0; i < n; ++i) order[i] = Pr{i, g.deg(i)};
    std::sort(order.begin(), order.end(), [](const Pr& a, const Pr& b) {
        if (a.second != b.second) return a.second < b.second;
        return a.first < b.first;
    });
    std::vector<double> triwgt(n, 0.0);
    std::vector<char> nbd(n, 0), clustered(n, 0);
    struct Cand {
        int64_t vertex;
        double wgt;
    };
    int64_t ncl = 0, nout = 0;
    cl_off[0] = 0;
    g_last_sets.clear();
    for (int64_t i = 0; i < n; ++i) {
        const int64_t u = order[i].first;
        const int64_t degu = order[i].second;
        if (clustered[u]) continue;
        std::unordered_set<int64_t> members;
        members.insert(u);
        clustered[u] = 1;
        std::set<int64_t> two_hop;
        double internal = 0;
        for (int64_t j = offsets[u]; j < offsets[u + 1]; ++j) {
            const int64_t v = nbors[j];
            if (st[j] == 'N') continue;
            members.insert(v);
            nbd[v] = 1;
            clustered[v] = 1;
        }
        for (int64_t j = offsets[u]; j < offsets[u + 1]; ++j) {
            const int64_t v = nbors[j];
            if (st[j] == 'N') continue;
            const int64_t degv = g.deg(v);
            if ((double)degv > (double)degu / eps) continue;
            for (int64_t k = j; k < offsets[u + 1]; ++k) {  // k starts at j: w == v included
                const int64_t w = nbors[k];
                if (st[k] == 'N') continue;
                const int64_t degw = g.deg(w);
                if ((double)degw > (double)degu / eps) continue;
                const int64_t loc = g.find(u, w);
                if (loc == -1 || st[loc] == 'N') continue;
                internal += 1.0 / double(degu * degv * degw);
                const int64_t lower = (degv < degw) ? v : w;
                const int64_t higher = (degv < degw) ? w : v;
                for (int64_t l = offsets[lower]; l < offsets[lower + 1]; ++l) {
                    if (st[l] == 'N') continue;
                    const int64_t x = nbors[l];
                    const int64_t degx = g.deg(x);
                    if (x == lower || x == higher || x == u) continue;
                    const int64_t loc_hx = g.find(higher, x);
                    if (loc_hx == -1 || st[loc_hx] == 'N') continue;
                    const double wgt = 1.0 / double(degx * degv * degw);
                    if (nbd[x]) {
                        if (x > v && x > w) internal += wgt;
                        continue;
                    }
                    two_hop.insert(x);
                    triwgt[x] += wgt;
                }
            }
        }
        std::vector<Cand> cand;
        cand.reserve(two_hop.size());
        double potential = 0;
        for (int64_t x : two_hop) {
            cand.push_back(Cand{x, triwgt[x]});
            potential += triwgt[x];
            triwgt[x] = 0;
        }
        std::sort(cand.begin(), cand.end(), [](const Cand& a, const Cand& b) { return a.wgt > b.wgt; });
        double ratio = internal / (internal + potential);
        int64_t maxind = -1;
        double num = 0, den = 0;
        for (int64_t c = 0; c < (int64_t)cand.size(); ++c) {
            num += cand[c].wgt;
            den += pv[cand[c].vertex];
            const double nr = (internal + num) / (internal + potential + den);
            if (nr > ratio) {
                ratio = nr;
                maxind = c;
            }
        }
        for (int64_t c = 0; c <= maxind; ++c) {
            members.insert(cand[c].vertex);
            clustered[cand[c].vertex] = 1;
        }
        for (int64_t j = offsets[u]; j < offsets[u + 1]; ++j) nbd[nbors[j]] = 0;

        // populateStats over the original adjacency.
        int64_t ne = 0, cut = 0;
        for (int64_t z : members)
            for (int64_t j = offsets[z]; j < offsets[z + 1]; ++j) {
                if (members.count(nbors[j])) ++ne;
                else ++cut;
            }
        cl_seed[ncl] = u;
        cl_nv[ncl] = (int64_t)members.size();
        cl_ne[ncl] = ne / 2;
        cl_cut[ncl] = cut;
        for (int64_t z : members) cl_vert[nout++] = z;
        cl_off[ncl + 1] = nout;
        ++ncl;
        g_last_sets.push_back(members);  // decomposition.push_back(next_clus): a copy

        std::stack<Pr> todo;
        for (int64_t z : members)
            for (int64_t j = offsets[z]; j < offsets[z + 1]; ++j) {
                if (st[j] != 'Y') continue;
                todo.push(Pr{z, nbors[j]});
                st[j] = 'S';
                st[partner[j]] = 'S';
            }
        delete_and_clean(g, st, pe, pv, sup, total, todo, eps, nullptr, nullptr);
    }
    return ncl;
}

int64_t orc_expand(int64_t n, const int64_t* offsets, const int64_t* nbors, int64_t threshold,
                   int64_t* cl_nv, int64_t* cl_ne, int64_t* cl_cut, int64_t* cl_off, int64_t* cl_vert,
                   int64_t* n_scores, int64_t* sc_vertex, double* sc_value)
{
    // expandClusters, Decomposition.h:958-1008.  The decomposition and the
    // cluster map arrive by value: the sets are copies of the extraction's
    // (copies keep iteration order and bucket count) and the map is never
    // updated, so every vote reads the extraction's assignment.
    std::vector<std::unordered_set<int64_t>> dec = g_last_sets;
    const int64_t k = (int64_t)dec.size();
    std::vector<int64_t> cmap(n, -1);
    std::vector<int64_t> nv0(k);
    for (int64_t c = 0; c < k; ++c) {
        nv0[c] = (int64_t)dec[c].size();  // nVertices as populateStats left it
        for (int64_t z : dec[c]) cmap[z] = c;
    }
    std::map<int64_t, double> scores;
    for (int64_t i = 0; i < k; ++i) {
        if (nv0[i] > 1) continue;
        const int64_t v = *dec[i].cbegin();
        std::map<int64_t, int64_t> counts;
        int64_t best = -1;
        int64_t max_score = threshold;
        const int64_t deg = offsets[v + 1] - offsets[v];
        for (int64_t j = offsets[v]; j < offsets[v + 1]; ++j) {
            const int64_t u = nbors[j];
            if (cmap[u] == -1) continue;
            const int64_t c = cmap[u];
            const int64_t cnt = ++counts[c];
            if (cnt > max_score) {
                best = c;
                max_score = cnt;
            }
        }
        if (best == -1) continue;
        dec[best].insert(v);
        dec[i].erase(v);
        scores[v] = (double)max_score / deg;
    }
    int64_t nout = 0;
    cl_off[0] = 0;
    for (int64_t c = 0; c < k; ++c) {
        int64_t ne = 0, cut = 0;
        for (int64_t z : dec[c])
            for (int64_t j = offsets[z]; j < offsets[z + 1]; ++j) {
                if (dec[c].count(nbors[j])) ++ne;
                else ++cut;
            }
        cl_nv[c] = (int64_t)dec[c].size();
        cl_ne[c] = ne / 2;
        cl_cut[c] = cut;
        for (int64_t z : dec[c]) cl_vert[nout++] = z;
        cl_off[c + 1] = nout;
    }
    int64_t ns = 0;
    for (const auto& e : scores) {
        sc_vertex[ns] = e.first;
        sc_value[ns] = e.second;
        ++ns;
    }
    *n_scores = ns;
    return k;
}

void orc_selfcheck_counts(int64_t* missing_edge, int64_t* bad_status, int64_t* residual)
{
    *missing_edge = g_missing;
    *bad_status = g_badstatus;
    *residual = g_residual;
}

void orc_selfcheck_reset(void)
{
    g_missing = g_badstatus = g_residual = 0;
}

}  // extern "C"
