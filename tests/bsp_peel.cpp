// Bulk-synchronous peel used by tests/test_oracle.py to show that a case is
// order-sensitive: every round recomputes each alive edge's triangle weight
// from scratch and removes all edges below eps/(du*dv) at once, until no edge
// is removed.  Prints one 0/1 alive flag per directed CSR slot.
// Usage: bsp_peel <escape-graph> <eps>
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

int main(int argc, char** argv)
{
    if (argc < 3) return 2;
    FILE* f = fopen(argv[1], "r");
    const double eps = atof(argv[2]);
    long n, m;
    if (!f || fscanf(f, "%ld %ld", &n, &m) != 2) return 1;
    std::vector<std::pair<long, long>> e;
    for (long i = 0; i < m; ++i) {
        long a, b;
        if (fscanf(f, "%ld %ld", &a, &b) != 2) return 1;
        e.push_back({a, b});
        e.push_back({b, a});
    }
    std::sort(e.begin(), e.end());
    const long m2 = (long)e.size();
    std::vector<long> off(n + 1, 0), nb(m2);
    for (long i = 0; i < m2; ++i) {
        nb[i] = e[i].second;
        off[e[i].first + 1]++;
    }
    for (long i = 0; i < n; ++i) off[i + 1] += off[i];
    auto deg = [&](long v) { return off[v + 1] - off[v]; };
    auto find = [&](long a, long b) -> long {
        long lo = off[a], hi = off[a + 1] - 1;
        while (lo <= hi) {
            long md = (lo + hi) / 2;
            if (nb[md] == b) return md;
            if (nb[md] > b) hi = md - 1;
            else lo = md + 1;
        }
        return -1;
    };
    std::vector<long> part(m2);
    for (long u = 0; u < n; ++u)
        for (long i = off[u]; i < off[u + 1]; ++i) part[i] = find(nb[i], u);
    std::vector<char> alive(m2, 1);
    while (true) {
        std::vector<double> w(m2, 0.0);
        for (long u = 0; u < n; ++u)
            for (long i = off[u]; i < off[u + 1]; ++i) {
                const long v = nb[i];
                if (!alive[i] || u > v) continue;
                for (long j = off[u]; j < off[u + 1]; ++j) {
                    const long x = nb[j];
                    if (!alive[j] || x <= v) continue;
                    const long l = find(v, x);
                    if (l < 0 || !alive[l]) continue;
                    const double t = 1 / double(deg(u) * deg(v) * deg(x));
                    w[i] += t;
                    w[j] += t;
                    w[l] += t;
                }
            }
        long removed = 0;
        for (long u = 0; u < n; ++u)
            for (long i = off[u]; i < off[u + 1]; ++i) {
                const long v = nb[i];
                if (!alive[i] || u > v) continue;
                if (w[i] < eps * (1 / double(deg(u) * deg(v)))) {
                    alive[i] = alive[part[i]] = 0;
                    ++removed;
                }
            }
        if (!removed) break;
    }
    for (long i = 0; i < m2; ++i) printf("%d\n", (int)alive[i]);
    return 0;
}
