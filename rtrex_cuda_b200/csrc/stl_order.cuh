// Order-faithful restatements of the two GNU libstdc++ (GCC 13) behaviours the
// reference's results depend on, usable from host and device code:
//
//  * std::sort's permutation (introsort: median-of-three quicksort with an
//    unguarded partition, heapsort below depth 2*floor(log2 n), final insertion
//    sort with a 16-element threshold).  The reference ranks the two-hop
//    candidates with std::sort(.., wgtCompareDecreasing) (Decomposition.h:829,
//    ClusterStructures.h:44-47); equal weights keep whatever order introsort
//    leaves them in, and that order decides which vertices enter a cluster.
//
//  * std::unordered_set<int64_t> iteration order (identity hash, unique keys,
//    max load factor 1).  The reference pushes a cluster's edges onto the
//    deletion stack while iterating its member set (Decomposition.h:898-914), so
//    the LIFO cascade order, and with it every later floating-point decision,
//    follows this order.  It is also the order the decomposition file lists a
//    cluster's vertices in (RTRex.cpp:63-65).
//
// Both are written from the published algorithms, not copied; they are pinned
// against the real std::sort / std::unordered_set by tests/test_stl_order.py.
#pragma once

#include <cstdint>

#ifdef __CUDACC__
#define RTR_HD __host__ __device__
#else
#define RTR_HD
#endif

namespace rtr {

// ------------------------------------------------------------------ introsort

template <typename T>
RTR_HD inline void swap_elems(T* a, T* b)
{
    T t = *a;
    *a = *b;
    *b = t;
}

template <typename T, typename Comp>
RTR_HD inline void heap_sift(T* first, int64_t hole, int64_t len, T value, Comp comp)
{
    // Move the larger child up until the hole reaches a leaf, then push value up.
    const int64_t top = hole;
    int64_t child = hole;
    while (child < (len - 1) / 2) {
        child = 2 * (child + 1);
        if (comp(first[child], first[child - 1])) child--;
        first[hole] = first[child];
        hole = child;
    }
    if ((len & 1) == 0 && child == (len - 2) / 2) {
        child = 2 * (child + 1);
        first[hole] = first[child - 1];
        hole = child - 1;
    }
    int64_t parent = (hole - 1) / 2;
    while (hole > top && comp(first[parent], value)) {
        first[hole] = first[parent];
        hole = parent;
        parent = (hole - 1) / 2;
    }
    first[hole] = value;
}

template <typename T, typename Comp>
RTR_HD inline void heap_sort_range(T* first, T* last, Comp comp)
{
    const int64_t len = last - first;
    if (len >= 2) {  // build the heap bottom-up
        int64_t parent = (len - 2) / 2;
        while (true) {
            T v = first[parent];
            heap_sift(first, parent, len, v, comp);
            if (parent == 0) break;
            parent--;
        }
    }
    while (last - first > 1) {  // repeatedly move the top to the end
        --last;
        T v = *last;
        *last = *first;
        heap_sift(first, (int64_t)0, (int64_t)(last - first), v, comp);
    }
}

template <typename T, typename Comp>
RTR_HD inline void median_to_first(T* result, T* a, T* b, T* c, Comp comp)
{
    if (comp(*a, *b)) {
        if (comp(*b, *c)) swap_elems(result, b);
        else if (comp(*a, *c)) swap_elems(result, c);
        else swap_elems(result, a);
    } else if (comp(*a, *c)) {
        swap_elems(result, a);
    } else if (comp(*b, *c)) {
        swap_elems(result, c);
    } else {
        swap_elems(result, b);
    }
}

// Hoare partition around *pivot without bounds checks in the original; the
// guards below never fire for a consistent comparator and only keep a broken
// one from walking out of the range.
template <typename T, typename Comp>
RTR_HD inline T* partition_unguarded(T* first, T* last, T* pivot, T* lo, T* hi, Comp comp)
{
    while (true) {
        while (first < hi && comp(*first, *pivot)) ++first;
        --last;
        while (last > lo && comp(*pivot, *last)) --last;
        if (!(first < last)) return first;
        swap_elems(first, last);
        ++first;
    }
}

template <typename T, typename Comp>
RTR_HD inline void linear_insert(T* pos, T* lo, Comp comp)
{
    T val = *pos;
    T* next = pos - 1;
    while (pos > lo && comp(val, *next)) {
        *pos = *next;
        pos = next;
        --next;
    }
    *pos = val;
}

template <typename T, typename Comp>
RTR_HD inline void insertion_sort(T* first, T* last, Comp comp)
{
    if (first == last) return;
    for (T* i = first + 1; i != last; ++i) {
        if (comp(*i, *first)) {
            T val = *i;
            for (T* p = i; p != first; --p) *p = *(p - 1);
            *first = val;
        } else {
            linear_insert(i, first, comp);
        }
    }
}

RTR_HD inline int floor_log2(int64_t n)
{
    int r = -1;
    while (n > 0) {
        n >>= 1;
        ++r;
    }
    return r;
}

// std::sort(first, last, comp): same sequence of comparisons and moves, so the
// same final permutation for any comparator (including ties).
template <typename T, typename Comp>
RTR_HD inline void introsort(T* first, T* last, Comp comp)
{
    constexpr int64_t kThreshold = 16;
    const int64_t n = last - first;
    if (n <= 0) return;
    // The quicksort recursion handles [cut,last) then continues on [first,cut);
    // the two ranges are disjoint, so an explicit stack gives the same result.
    struct Range {
        T* f;
        T* l;
        int depth;
    };
    Range stack[128];
    int sp = 0;
    stack[sp++] = Range{first, last, 2 * floor_log2(n)};
    while (sp > 0) {
        Range r = stack[--sp];
        T* f = r.f;
        T* l = r.l;
        int depth = r.depth;
        while (l - f > kThreshold) {
            if (depth == 0) {
                heap_sort_range(f, l, comp);
                break;
            }
            --depth;
            T* mid = f + (l - f) / 2;
            median_to_first(f, f + 1, mid, l - 1, comp);
            T* cut = partition_unguarded(f + 1, l, f, f, l, comp);
            if (sp < 128) stack[sp++] = Range{cut, l, depth};
            l = cut;
        }
    }
    if (n > kThreshold) {
        insertion_sort(first, first + kThreshold, comp);
        for (T* i = first + kThreshold; i != last; ++i) linear_insert(i, first, comp);
    } else {
        insertion_sort(first, last, comp);
    }
}

// ------------------------------------------------------ unordered_set order

// Bucket count after the insert that brings the set to `size` elements, for a
// default-constructed std::unordered_set<int64_t> (probed through the public
// bucket_count() of GCC 13's libstdc++): the set starts with 1 bucket, and the
// insert that makes size exceed the bucket count rehashes to the next entry.
struct RehashStep {
    int64_t at_size;
    int64_t buckets;
};
constexpr int kRehashSteps = 23;
RTR_HD inline int64_t uset_buckets_after(int64_t size)
{
    const RehashStep t[kRehashSteps] = {
        {1, 13},
        {14, 29},
        {30, 59},
        {60, 127},
        {128, 257},
        {258, 541},
        {542, 1109},
        {1110, 2357},
        {2358, 5087},
        {5088, 10273},
        {10274, 20753},
        {20754, 42043},
        {42044, 85229},
        {85230, 172933},
        {172934, 351061},
        {351062, 712697},
        {712698, 1447153},
        {1447154, 2938679},
        {2938680, 5967347},
        {5967348, 12117689},
        {12117690, 24607243},
        {24607244, 49969847},
        {49969848, 101473717},
    };
    int64_t b = 1;
    for (int i = 0; i < kRehashSteps; ++i)
        if (size >= t[i].at_size) b = t[i].buckets;
    return b;
}
constexpr int64_t kUsetMaxSize = 101473717;

// The set's nodes live in caller-provided arrays: node i holds key[i] and the
// index of the next node in iteration order (-1 ends the list).  bucket[b] names
// the node *before* bucket b's first node (kBeforeBegin for the list head) or
// kEmpty.  Node ids are assigned in insertion order (an erased node's id is not
// reused).  The table grows when an insert takes the size above the current
// bucket count (max_load_factor 1: the rehash policy's next-resize mark equals
// the bucket count) and never shrinks, as in the library: after erases, inserts
// up to the previous size do not rehash.
struct UsetOrder {
    static constexpr int32_t kEmpty = -1;
    static constexpr int32_t kBeforeBegin = -2;
    int32_t* key;
    int32_t* next;
    int32_t* bucket;
    int64_t nbuckets;
    int32_t head;
    int32_t size;
    int32_t used;  // node ids handed out

    RTR_HD void init(int32_t* k, int32_t* nx, int32_t* b)
    {
        key = k;
        next = nx;
        bucket = b;
        nbuckets = 1;
        head = -1;
        size = 0;
        used = 0;
        bucket[0] = kEmpty;
    }

    // The state of a set built by `cnt` inserts of distinct keys (no erase),
    // given its keys in iteration order in key[0..cnt): nodes in list order,
    // bucket count from the growth schedule, bucket heads from the list (the
    // list keeps each bucket's nodes together).
    RTR_HD void init_from_list(int32_t* k, int32_t* nx, int32_t* b, int32_t cnt)
    {
        key = k;
        next = nx;
        bucket = b;
        size = used = cnt;
        nbuckets = cnt ? uset_buckets_after(cnt) : 1;
        head = cnt ? 0 : -1;
        for (int64_t i = 0; i < nbuckets; ++i) bucket[i] = kEmpty;
        int32_t prev = kBeforeBegin;
        for (int32_t p = 0; p < cnt; ++p) {
            next[p] = p + 1 < cnt ? p + 1 : -1;
            const int64_t bk = bkt(key[p]);
            if (bucket[bk] == kEmpty) bucket[bk] = prev;
            prev = p;
        }
    }
    RTR_HD int32_t after(int32_t p) const { return p == kBeforeBegin ? head : next[p]; }
    RTR_HD void set_after(int32_t p, int32_t v)
    {
        if (p == kBeforeBegin) head = v;
        else next[p] = v;
    }
    RTR_HD int64_t bkt(int32_t k) const { return (int64_t)(uint64_t)(int64_t)k % nbuckets; }

    RTR_HD bool contains(int32_t k) const
    {
        if (size == 0) return false;
        const int64_t b = bkt(k);
        const int32_t prev = bucket[b];
        if (prev == kEmpty) return false;
        for (int32_t p = after(prev); p != -1; p = next[p]) {
            if (key[p] == k) return true;
            if (next[p] == -1 || bkt(key[next[p]]) != b) break;
        }
        return false;
    }

    RTR_HD void rehash(int64_t nb)
    {
        for (int64_t b = 0; b < nb; ++b) bucket[b] = kEmpty;
        int32_t p = head;
        head = -1;
        int64_t bbegin = 0;
        const int64_t old = nbuckets;
        nbuckets = nb;
        (void)old;
        while (p != -1) {
            const int32_t nx = next[p];
            const int64_t b = bkt(key[p]);
            if (bucket[b] == kEmpty) {
                next[p] = head;
                head = p;
                bucket[b] = kBeforeBegin;
                if (next[p] != -1) bucket[bbegin] = p;
                bbegin = b;
            } else {
                next[p] = after(bucket[b]);
                set_after(bucket[b], p);
            }
            p = nx;
        }
    }

    // insert(k); returns false when k was already present.
    RTR_HD bool insert(int32_t k)
    {
        if (contains(k)) return false;
        const int64_t nb = uset_buckets_after((int64_t)size + 1);
        if (nb > nbuckets) rehash(nb);
        const int32_t id = used++;
        key[id] = k;
        const int64_t b = bkt(k);
        if (bucket[b] != kEmpty) {
            next[id] = after(bucket[b]);
            set_after(bucket[b], id);
        } else {
            next[id] = head;
            head = id;
            if (next[id] != -1) bucket[bkt(key[next[id]])] = id;
            bucket[b] = kBeforeBegin;
        }
        ++size;
        return true;
    }

    // erase(k): unlink k's node, keeping every bucket's before-node valid
    // (the hashtable's _M_erase / _M_remove_bucket_begin).  Returns false when
    // k is absent.
    RTR_HD bool erase(int32_t k)
    {
        if (size == 0) return false;
        const int64_t b = bkt(k);
        int32_t prev = bucket[b];
        if (prev == kEmpty) return false;
        int32_t p = after(prev);
        while (p != -1 && key[p] != k) {
            if (next[p] == -1 || bkt(key[next[p]]) != b) return false;
            prev = p;
            p = next[p];
        }
        if (p == -1) return false;
        const int32_t nx = next[p];
        if (prev == bucket[b]) {  // p begins its bucket
            const int64_t nb = nx != -1 ? bkt(key[nx]) : 0;
            if (nx == -1 || nb != b) {  // the bucket becomes empty
                if (nx != -1) bucket[nb] = bucket[b];
                bucket[b] = kEmpty;
            }
        } else if (nx != -1) {
            const int64_t nb = bkt(key[nx]);
            if (nb != b) bucket[nb] = prev;
        }
        set_after(prev, nx);
        --size;
        return true;
    }
};

}  // namespace rtr
