// Pins rtrex_cuda_b200/csrc/stl_order.cuh against the host C++ library it
// restates: std::sort's permutation on tie-heavy candidate arrays (the
// reference's wgtCompareDecreasing ranking) and std::unordered_set<int64_t>'s
// iteration order after arbitrary insert sequences.  Built and run by
// tests/test_stl_order.py; prints "OK <cases>" or the first mismatch.
#include "../rtrex_cuda_b200/csrc/stl_order.cuh"

#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <random>
#include <unordered_set>
#include <vector>

struct Cand {
    int32_t vertex;
    double wgt;
};

static bool by_wgt_desc(const Cand& a, const Cand& b) { return a.wgt > b.wgt; }

static int check_sort(std::vector<Cand> v, long* cases)
{
    std::vector<Cand> ref = v;
    std::sort(ref.begin(), ref.end(), by_wgt_desc);
    rtr::introsort(v.data(), v.data() + v.size(), [](const Cand& a, const Cand& b) { return a.wgt > b.wgt; });
    ++*cases;
    for (size_t i = 0; i < v.size(); ++i)
        if (v[i].vertex != ref[i].vertex || v[i].wgt != ref[i].wgt) {
            printf("SORT MISMATCH n=%zu at %zu\n", v.size(), i);
            return 1;
        }
    return 0;
}

static int check_uset(const std::vector<int32_t>& ins, long* cases)
{
    std::unordered_set<int64_t> ref;
    size_t cap = ins.size() + 1;
    std::vector<int32_t> key(cap), nxt(cap), bkt(rtr::uset_buckets_after((int64_t)cap) + 1);
    rtr::UsetOrder s;
    s.init(key.data(), nxt.data(), bkt.data());
    for (int32_t k : ins) {
        bool a = ref.insert(k).second;
        bool b = s.insert(k);
        if (a != b) {
            printf("USET INSERT RESULT MISMATCH\n");
            return 1;
        }
        if ((int64_t)ref.bucket_count() != s.nbuckets) {
            printf("USET BUCKETS MISMATCH %zu vs %ld at size %zu\n", ref.bucket_count(), (long)s.nbuckets,
                   ref.size());
            return 1;
        }
    }
    ++*cases;
    int32_t p = s.head;
    for (int64_t x : ref) {
        if (p == -1 || key[p] != x) {
            printf("USET ORDER MISMATCH size=%zu\n", ref.size());
            return 1;
        }
        p = nxt[p];
    }
    if (p != -1) {
        printf("USET LENGTH MISMATCH\n");
        return 1;
    }
    return 0;
}

static int same_order(const std::unordered_set<int64_t>& ref, const rtr::UsetOrder& s, const char* what)
{
    int32_t p = s.head;
    for (int64_t x : ref) {
        if (p == -1 || s.key[p] != x) {
            printf("USET %s ORDER MISMATCH size=%zu\n", what, ref.size());
            return 1;
        }
        p = s.next[p];
    }
    if (p != -1 || (int64_t)ref.size() != s.size || (int64_t)ref.bucket_count() != s.nbuckets) {
        printf("USET %s SIZE/BUCKETS MISMATCH %zu/%zu vs %d/%ld\n", what, ref.size(), ref.bucket_count(), s.size,
               (long)s.nbuckets);
        return 1;
    }
    return 0;
}

// A set built by inserts, copied (the copy keeps iteration order and bucket
// count), then driven by a mix of inserts and erases: the state rebuilt from the
// copy's iteration order (init_from_list) follows the library through every step.
static int check_uset_mixed(const std::vector<int32_t>& base, const std::vector<std::pair<int, int32_t>>& ops,
                            long* cases)
{
    std::unordered_set<int64_t> built;
    for (int32_t k : base) built.insert(k);
    std::unordered_set<int64_t> ref = built;
    size_t cap = built.size() + ops.size() + 1;
    std::vector<int32_t> key(cap), nxt(cap), bkt(rtr::uset_buckets_after((int64_t)cap) + 1);
    int32_t cnt = 0;
    for (int64_t x : built) key[cnt++] = (int32_t)x;
    rtr::UsetOrder s;
    s.init_from_list(key.data(), nxt.data(), bkt.data(), cnt);
    if (same_order(ref, s, "REBUILT")) return 1;
    for (const auto& op : ops) {
        bool a, b;
        if (op.first) {
            a = ref.insert(op.second).second;
            b = s.insert(op.second);
        } else {
            a = ref.erase(op.second) == 1;
            b = s.erase(op.second);
        }
        if (a != b) {
            printf("USET %s RESULT MISMATCH\n", op.first ? "INSERT" : "ERASE");
            return 1;
        }
        if (same_order(ref, s, op.first ? "INSERT" : "ERASE")) return 1;
    }
    ++*cases;
    return 0;
}

// McIlroy's adversary ("A killer adversary for quicksort", 1999): values are
// fixed lazily during a sort so that every partition is maximally unbalanced.
// Sorting the resulting input again drives introsort into its heapsort branch.
static std::vector<int> adversarial_input(int n)
{
    std::vector<int> val(n), ptr(n);
    const int gas = n;
    int nsolid = 0, candidate = 0;
    for (int i = 0; i < n; ++i) {
        val[i] = gas;
        ptr[i] = i;
    }
    auto cmp = [&](int x, int y) {
        if (val[x] == gas && val[y] == gas) {
            if (x == candidate) val[x] = nsolid++;
            else val[y] = nsolid++;
        }
        if (val[x] == gas) candidate = x;
        else if (val[y] == gas) candidate = y;
        return val[x] < val[y];
    };
    std::sort(ptr.begin(), ptr.end(), cmp);
    for (int i = 0; i < n; ++i)
        if (val[i] == gas) val[i] = nsolid++;
    return val;
}

int main()
{
    std::mt19937_64 rng(12345);
    long cases = 0;
    for (int n : {64, 500, 3000, 50000}) {
        std::vector<int> a = adversarial_input(n);
        std::vector<Cand> v(n);
        for (int i = 0; i < n; ++i) v[i] = Cand{i, -(double)a[i]};  // weight desc == value asc
        if (check_sort(v, &cases)) return 1;
        for (int i = 0; i < n; ++i) v[i] = Cand{i, -(double)(a[i] / 3)};  // with ties
        if (check_sort(v, &cases)) return 1;
    }
    // Random tie-heavy candidate arrays in ascending-vertex order.
    for (int rep = 0; rep < 4000; ++rep) {
        int n = (rep < 300) ? rep : (int)(rng() % (rep < 3000 ? 200 : 6000));
        int distinct = 1 + (int)(rng() % 12);
        std::vector<Cand> v(n);
        for (int i = 0; i < n; ++i) {
            v[i].vertex = i * 3 + 1;
            v[i].wgt = 1.0 / (double)(1 + rng() % distinct);
        }
        if (check_sort(v, &cases)) return 1;
    }
    // Structured inputs: sorted, reversed, organ pipe, sawtooth, all equal.
    for (int n : {17, 33, 100, 257, 1000, 4097, 20000}) {
        for (int pat = 0; pat < 6; ++pat) {
            std::vector<Cand> v(n);
            for (int i = 0; i < n; ++i) {
                double w;
                switch (pat) {
                case 0: w = i; break;
                case 1: w = n - i; break;
                case 2: w = i < n / 2 ? i : n - i; break;
                case 3: w = i % 7; break;
                case 4: w = 1.0; break;
                default: w = (i * 2654435761u) % 97; break;
                }
                v[i] = Cand{i, w};
            }
            if (check_sort(v, &cases)) return 1;
        }
    }
    // unordered_set: random inserts with repeats, sizes across several rehashes.
    for (int rep = 0; rep < 600; ++rep) {
        int n = (rep < 200) ? rep : (int)(rng() % (rep < 550 ? 3000 : 200000));
        int range = 1 + (int)(rng() % (rep % 3 == 0 ? 100 : 10000000));
        std::vector<int32_t> ins(n);
        for (int i = 0; i < n; ++i) ins[i] = (int32_t)(rng() % range);
        if (check_uset(ins, &cases)) return 1;
    }
    // Rebuilt sets under inserts and erases (cluster expansion: absorbed
    // singletons join clusters, emptied singletons lose their vertex).
    for (int rep = 0; rep < 400; ++rep) {
        int n = 1 + (int)(rng() % (rep < 300 ? 40 : 3000));
        int range = 1 + (int)(rng() % (rep % 2 ? 64 : 1000000));
        std::vector<int32_t> base(n);
        for (int i = 0; i < n; ++i) base[i] = (int32_t)(rng() % range);
        std::vector<std::pair<int, int32_t>> ops(1 + rng() % (rep < 300 ? 60 : 5000));
        for (auto& op : ops) {
            op.first = (rng() % 3) != 0;
            op.second = (op.first || base.empty()) ? (int32_t)(rng() % range) : base[rng() % base.size()];
        }
        if (check_uset_mixed(base, ops, &cases)) return 1;
    }
    printf("OK %ld\n", cases);
    return 0;
}
