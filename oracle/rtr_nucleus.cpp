// Restated nucleus (truss-hierarchy) path of the reference, for parity tests.
//
// TEST INFRASTRUCTURE ONLY (tests/ and the bench's CPU leg); the product
// library never links it.
//
// Follows RTRex_Sequential/clustering/nucleus.cpp:12-81 step by step:
//   relabel by (degree, id)        CGraph::renameByDegreeOrderMapping, Graph.cpp:261-310
//   per-edge triangle lists        storeAllTriangles, Escape/Nucleus.h:125-163
//   integer peel and hierarchy     nuclei, Nucleus.h:306-565, with
//                                  findConnectedComponent :169-242 and completeCluster :246-301
// (betterWedgeEnumerator, Nucleus.h:78-119, only supplies the triangle total
// that sizes the lists; the lists' length is that total times three.)
// Edge ids are slots of the relabelled CSR; every container keeps the
// reference's order (LIFO deletion stack, neighbour lists in discovery order,
// the depth-first stacks of the hierarchy walk, std::set member order).
#include "rtr_oracle.h"

#include <algorithm>
#include <cstdint>
#include <set>
#include <vector>

namespace {

struct NucleusResult {
    std::vector<int64_t> id, c, nv, ne, parent, voff, vert;  // vert in original labels
    std::vector<int64_t> kappa;                               // per slot of the relabelled CSR (-1: backward slot)
    std::vector<int64_t> rel_off, rel_nb, inverse;            // the relabelled CSR and new -> old labels
    int64_t overflow = 0;  // bits: arrays of the reference's fixed sizes this input overruns (see orc_nucleus_sizes)
};

NucleusResult g_last;

struct Rel {
    int64_t n;
    std::vector<int64_t> off, nb;
    int64_t slot(int64_t a, int64_t b) const  // CGraph::getEdgeBinary
    {
        int64_t lo = off[a], hi = off[a + 1] - 1;
        while (lo <= hi) {
            const int64_t mid = (lo + hi) / 2;
            if (nb[mid] == b) return mid;
            if (nb[mid] > b) hi = mid - 1;
            else lo = mid + 1;
        }
        return -1;
    }
    int64_t deg(int64_t a) const { return off[a + 1] - off[a]; }
};

struct Clus {
    int64_t id = 0, c = 0, nv = 0, ne = 0, parent = -1;
    std::set<int64_t> verts;
};

}  // namespace

extern "C" {

int64_t orc_nucleus(int64_t n, const int64_t* off, const int64_t* nb)
{
    NucleusResult& R = g_last;
    R = NucleusResult();
    // relabel: new label = rank of (degree, old id)
    std::vector<int64_t> order(n), newid(n);
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order.begin(), order.end(), [&](int64_t a, int64_t b) {
        const int64_t da = off[a + 1] - off[a], db = off[b + 1] - off[b];
        return da != db ? da < db : a < b;
    });
    for (int64_t r = 0; r < n; ++r) newid[order[r]] = r;
    Rel g;
    g.n = n;
    g.off.assign(n + 1, 0);
    g.nb.resize(off[n]);
    for (int64_t r = 0; r < n; ++r) {
        const int64_t old = order[r];
        g.off[r + 1] = g.off[r] + (off[old + 1] - off[old]);
        for (int64_t p = off[old]; p < off[old + 1]; ++p) g.nb[g.off[r] + (p - off[old])] = newid[nb[p]];
        std::sort(g.nb.begin() + g.off[r], g.nb.begin() + g.off[r + 1]);
    }
    const int64_t m2 = g.off[n];
    std::vector<int64_t> src(m2);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t p = g.off[i]; p < g.off[i + 1]; ++p) src[p] = i;

    // triangle lists of the edges whose far end is later in degree order
    std::vector<int64_t> trioff(m2 + 1, 0), tris;
    for (int64_t i = 0; i < n; ++i) {
        const int64_t di = g.deg(i);
        for (int64_t p = g.off[i]; p < g.off[i + 1]; ++p) {
            const int64_t j = g.nb[p];
            const int64_t dj = g.deg(j);
            trioff[p] = (int64_t)tris.size();
            if (dj < di || (dj == di && j <= i)) continue;
            for (int64_t q = g.off[i]; q < g.off[i + 1]; ++q)
                if (g.slot(g.nb[q], j) != -1) tris.push_back(g.nb[q]);
        }
    }
    trioff[m2] = (int64_t)tris.size();

    // level-by-level integer peel
    std::vector<int64_t> tri_count(m2 + 1, 0), kappa(m2 + 1, -1), dtime(m2 + 1, 0);
    std::vector<char> deleted(m2 + 1, 0);
    for (int64_t p = 0; p < m2; ++p)
        if (src[p] <= g.nb[p]) tri_count[p] = trioff[p + 1] - trioff[p];
    std::vector<int64_t> nbr_list, nbr_off(m2 + 2, 0);
    std::vector<int64_t> del_edges, del_off(m2 + 2, 0);
    std::vector<int64_t> stack;
    int64_t ndel = 0, total = 0, c = 1;
    // The reference holds these in fixed arrays: the neighbour lists in
    // 3T+1 entries (Nucleus.h:320), the deletion stack and the two depth-first
    // stacks in 2m+1 (Nucleus.h:310, :177, :259).  Inputs that need more are
    // undefined behaviour there; they are flagged so no test compares them.
    const int64_t nbr_cap = (int64_t)tris.size() + 1, stack_cap = m2 + 1;
    auto note_stack = [&](size_t depth, int64_t bit) {
        if ((int64_t)depth > stack_cap) R.overflow |= bit;
    };
    while (total < m2 / 2) {
        for (int64_t p = 0; p < m2; ++p)
            if (src[p] <= g.nb[p] && !deleted[p] && tri_count[p] < c) stack.push_back(p);
        while (!stack.empty()) {
            const int64_t e = stack.back();
            stack.pop_back();
            if (deleted[e]) continue;
            note_stack(stack.size() + 1, 2);
            const int64_t i = src[e], j = g.nb[e];
            deleted[e] = 1;
            kappa[e] = c - 1;
            dtime[e] = ndel++;
            del_edges.push_back(e);
            ++total;
            for (int64_t t = trioff[e]; t < trioff[e + 1]; ++t) {
                const int64_t k = tris[t];
                const int64_t eik = i < k ? g.slot(i, k) : g.slot(k, i);
                const int64_t ejk = j < k ? g.slot(j, k) : g.slot(k, j);
                if (!deleted[eik]) nbr_list.push_back(eik);
                if (!deleted[ejk]) nbr_list.push_back(ejk);
                if (deleted[eik] || deleted[ejk]) continue;
                if (--tri_count[eik] < c) stack.push_back(eik);
                if (--tri_count[ejk] < c) stack.push_back(ejk);
                note_stack(stack.size(), 2);
            }
            nbr_off[ndel] = (int64_t)nbr_list.size();
            if ((int64_t)nbr_list.size() > nbr_cap) R.overflow |= 1;
        }
        del_off[c] = (int64_t)del_edges.size();
        ++c;
    }
    const int64_t max_c = c - 2;

    // hierarchy of edge trees, highest level first
    std::vector<int64_t> parent(m2 + 1), cparent(m2 + 1), ptime(m2 + 1, 0), children, child_off(m2 + 2, 0);
    std::vector<char> in_cluster(m2 + 1, 0);
    for (int64_t p = 0; p <= m2; ++p) parent[p] = cparent[p] = p;
    std::vector<int64_t> roots, root_off(std::max<int64_t>(max_c, 0) + 2, 0);
    int64_t pt = 0;
    auto grow = [&](int64_t e) {  // findConnectedComponent
        std::vector<int64_t> st(nbr_list.begin() + nbr_off[dtime[e]], nbr_list.begin() + nbr_off[dtime[e] + 1]);
        in_cluster[e] = 1;
        while (!st.empty()) {
            const int64_t x = st.back();
            st.pop_back();
            if (cparent[x] == e) continue;
            if (in_cluster[x]) {
                int64_t top = x;
                while (cparent[top] != top) {
                    const int64_t up = cparent[top];
                    cparent[top] = e;
                    top = up;
                }
                if (top != e) {
                    parent[top] = e;
                    cparent[top] = e;
                    children.push_back(top);
                }
                continue;
            }
            parent[x] = e;
            cparent[x] = e;
            children.push_back(x);
            in_cluster[x] = 1;
            st.insert(st.end(), nbr_list.begin() + nbr_off[dtime[x]], nbr_list.begin() + nbr_off[dtime[x] + 1]);
            note_stack(st.size(), 4);
        }
    };
    for (int64_t lv = max_c; lv > 0; --lv) {
        for (int64_t q = del_off[lv]; q < del_off[lv + 1]; ++q) {
            const int64_t e = del_edges[q];
            ptime[e] = pt;
            child_off[pt] = (int64_t)children.size();
            ++pt;
            if (!in_cluster[e]) grow(e);
        }
        root_off[max_c - lv] = (int64_t)roots.size();
        for (int64_t q = del_off[lv]; q < del_off[lv + 1]; ++q) {
            const int64_t e = del_edges[q];
            if (parent[e] == e || kappa[parent[e]] < lv) roots.push_back(e);
        }
    }
    if (max_c >= 0) root_off[max_c] = (int64_t)roots.size();
    if (max_c >= 0)
        for (int64_t q = del_off[0]; q < del_off[1]; ++q) {
            ptime[del_edges[q]] = pt;
            child_off[pt] = (int64_t)children.size();
            ++pt;
        }
    child_off[pt] = (int64_t)children.size();

    // clusters, highest level first, each root's tree walked depth first
    std::vector<Clus> cl;
    std::vector<int64_t> root_to_cluster(m2 + 1, -1);
    for (int64_t lv = max_c; lv > 0; --lv) {
        for (int64_t q = root_off[max_c - lv]; q < root_off[max_c - lv + 1]; ++q) {
            const int64_t root = roots[q];
            Clus k;
            k.id = (int64_t)cl.size();
            k.c = lv;
            root_to_cluster[root] = k.id;
            std::vector<int64_t> st{root};
            while (!st.empty()) {
                const int64_t e = st.back();
                st.pop_back();
                if (kappa[e] > lv) {
                    Clus& inner = cl[root_to_cluster[e]];
                    k.ne += inner.ne;
                    inner.parent = k.id;
                    for (int64_t v : inner.verts)
                        if (k.verts.insert(v).second) ++k.nv;
                } else {
                    ++k.ne;
                    if (k.verts.insert(src[e]).second) ++k.nv;
                    if (k.verts.insert(g.nb[e]).second) ++k.nv;
                    for (int64_t t = child_off[ptime[e]]; t < child_off[ptime[e] + 1]; ++t) st.push_back(children[t]);
                    note_stack(st.size(), 8);
                }
            }
            cl.push_back(std::move(k));
        }
    }
    R.voff.push_back(0);
    for (const Clus& k : cl) {
        R.id.push_back(k.id);
        R.c.push_back(k.c);
        R.nv.push_back(k.nv);
        R.ne.push_back(k.ne);
        R.parent.push_back(k.parent);
        for (int64_t v : k.verts) R.vert.push_back(order[v]);
        R.voff.push_back((int64_t)R.vert.size());
    }
    R.kappa.assign(kappa.begin(), kappa.begin() + m2);
    R.rel_off = g.off;
    R.rel_nb = g.nb;
    R.inverse = order;
    return (int64_t)cl.size();
}

/* Sizes of the last orc_nucleus result: member entries over all clusters, 2m,
 * and the reference's fixed arrays the input overruns (bit 0 the neighbour
 * lists, 1 the deletion stack, 2 and 3 the two depth-first stacks; 0 = none,
 * so the reference's output is defined and comparable). */
void orc_nucleus_sizes(int64_t* n_members, int64_t* m2, int64_t* overflow)
{
    *n_members = (int64_t)g_last.vert.size();
    *m2 = (int64_t)g_last.kappa.size();
    *overflow = g_last.overflow;
}

/* Copy the last result out: per cluster id/c/nv/ne/parent, member offsets and
 * members (original labels, in the reference's set order of relabelled ids),
 * and kappa per slot of the relabelled CSR (-1 on slots whose source is the
 * later end).  Any pointer may be NULL. */
void orc_nucleus_get(int64_t* id, int64_t* c, int64_t* nv, int64_t* ne, int64_t* parent, int64_t* voff,
                     int64_t* vert, int64_t* kappa, int64_t* rel_off, int64_t* rel_nb, int64_t* inverse)
{
    const NucleusResult& R = g_last;
    auto put = [](const std::vector<int64_t>& a, int64_t* out) {
        if (out) std::copy(a.begin(), a.end(), out);
    };
    put(R.id, id);
    put(R.c, c);
    put(R.nv, nv);
    put(R.ne, ne);
    put(R.parent, parent);
    put(R.voff, voff);
    put(R.vert, vert);
    put(R.kappa, kappa);
    put(R.rel_off, rel_off);
    put(R.rel_nb, rel_nb);
    put(R.inverse, inverse);
}

}  // extern "C"
