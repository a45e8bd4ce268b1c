// Hash sets of long CSR rows, for membership lookups that cost about one
// memory transaction instead of a binary search's chain of dependent loads.
// Built by build_row_sets (count_rows.cu) for every vertex of at least
// kSetDegree neighbours: buckets of 8 keys (one 32-byte sector), a power-of-two
// number of them with at least 4 slots per key, linear probing over buckets;
// -1 marks an empty slot and a bucket's keys fill its slots from the first, so
// a lookup ends at the first bucket that still has an empty slot.  Rows hold
// distinct ids, so a set answers exactly "is z a neighbour of w"; the counting
// folds only need that (the weight of a common neighbour z depends on z alone).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "intersect.cuh"

namespace rtr {

// rows of at least this many entries get a hash set
constexpr int kSetDegree = 256;
constexpr int kBucketKeys = 8;

struct RowSets {
    const int32_t* tab;    // vertex -> its table, -1 for rows without one (null: no tables at all)
    const int64_t* toff;   // table -> first slot (a multiple of kBucketKeys)
    const int32_t* tbits;  // table -> log2 of its bucket count
    const int32_t* slot;   // the keys, -1 for empty slots
};

__device__ __forceinline__ int32_t rs_table(const RowSets& r, int32_t w) { return r.tab ? r.tab[w] : -1; }

__device__ __forceinline__ uint32_t rs_hash(int32_t z, int bits)
{
    return bits == 0 ? 0u : ((uint32_t)z * 2654435761u) >> (32 - bits);
}

__device__ __forceinline__ bool rs_member(const RowSets& r, int32_t t, int32_t z)
{
    const int4* tb = reinterpret_cast<const int4*>(r.slot + r.toff[t]);
    const int bits = r.tbits[t];
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t b = rs_hash(z, bits);
    while (true) {
        const int4 k0 = __ldg(tb + 2 * b), k1 = __ldg(tb + 2 * b + 1);
        if (k0.x == z || k0.y == z || k0.z == z || k0.w == z || k1.x == z || k1.y == z || k1.z == z || k1.w == z)
            return true;
        if (k1.w < 0) return false;  // the bucket is not full: z would be in it
        b = (b + 1u) & mask;
    }
}

// Warp-cooperative scan of the ascending range [s0, s1) 32 elements at a
// time, lane k holding element base+k: chunk(hit, x) with hit = pred(x), called
// by every lane (warp-uniform control flow); hits come in ascending order.  The
// scan stops at the first chunk whose elements all exceed zmax (no hits can
// follow: the caller passes the largest element of the row it looks up in).
template <typename Pred, typename F>
__device__ __forceinline__ void warp_scan(const int32_t* __restrict__ nb, int64_t s0, int64_t s1, int32_t zmax,
                                          int lane, Pred&& pred, F&& chunk)
{
    int32_t xn = s0 + lane < s1 ? nb[s0 + lane] : 0x7fffffff;
    for (int64_t base = s0; base < s1; base += 32) {
        const int32_t x = xn;
        const int64_t pn = base + 32 + lane;
        xn = pn < s1 ? nb[pn] : 0x7fffffff;  // the next chunk, loaded ahead of this one's lookups
        if (__all_sync(0xffffffffu, x > zmax)) break;
        const bool hit = base + lane < s1 && x <= zmax && pred(x);
        chunk(hit, x);
    }
}

// Batched form of a warp_scan through table t of the longer row (whose
// largest element is zmax): each step takes B chunks of 32 elements of S =
// [s0, s1), with the next step's elements loaded ahead and the first bucket of
// all 32*B lookups in flight at once; on_step(hit, x) then sees the step's B
// chunks (lane k of chunk b holds element base + 32b + k), every lane, in
// ascending order.  The walk stops at the first step whose first chunk lies
// wholly above zmax.
template <int B, typename F>
__device__ __forceinline__ void warp_probe_walk(const RowSets& rs, int32_t t, const int32_t* __restrict__ nb,
                                                int64_t s0, int64_t s1, int32_t zmax, int lane, F&& on_step)
{
    const int4* tb = reinterpret_cast<const int4*>(rs.slot + rs.toff[t]);
    const int bits = rs.tbits[t];
    const uint32_t mask = (1u << bits) - 1u;
    int32_t xn[B];
#pragma unroll
    for (int b = 0; b < B; ++b) {
        const int64_t p = s0 + 32 * b + lane;
        xn[b] = p < s1 ? nb[p] : 0x7fffffff;
    }
    for (int64_t base = s0; base < s1; base += 32 * B) {
        int32_t x[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            x[b] = xn[b];
            const int64_t p = base + 32 * (B + b) + lane;
            xn[b] = p < s1 ? nb[p] : 0x7fffffff;  // the next step, ahead of this one's lookups
        }
        if (__all_sync(0xffffffffu, x[0] > zmax)) break;
        uint32_t bk[B];
        int4 k0[B], k1[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            bk[b] = rs_hash(x[b], bits);
            if (x[b] <= zmax) {
                k0[b] = __ldg(tb + 2 * bk[b]);
                k1[b] = __ldg(tb + 2 * bk[b] + 1);
            } else {
                k0[b] = k1[b] = make_int4(-1, -1, -1, -1);
            }
        }
        bool hit[B];
#pragma unroll
        for (int b = 0; b < B; ++b) {
            const int32_t z = x[b];
            auto match = [&](const int4& p, const int4& q) {
                return p.x == z || p.y == z || p.z == z || p.w == z || q.x == z || q.y == z || q.z == z || q.w == z;
            };
            bool h = z <= zmax && match(k0[b], k1[b]);
            bool more = z <= zmax && !h && k1[b].w >= 0;  // the bucket is full: z may sit further on
            uint32_t c = bk[b];
            while (more) {
                c = (c + 1u) & mask;
                const int4 p = __ldg(tb + 2 * c), q = __ldg(tb + 2 * c + 1);
                h = match(p, q);
                more = !h && q.w >= 0;
            }
            hit[b] = h;
        }
        on_step(hit, x);
    }
}

// Common neighbours z >= from of the rows of a and b, ascending: f(z).  One
// thread.  The shorter row is walked and its elements looked up in the longer
// row's hash set when that row has one; otherwise the rows merge or gallop
// (intersect_rows).  from = INT32_MIN visits every common neighbour.
template <typename F>
__device__ __forceinline__ void thread_common(const RowSets& rs, const int64_t* __restrict__ off,
                                              const int32_t* __restrict__ nb, int32_t a, int32_t b, int32_t from,
                                              int gallop, F&& f)
{
    int64_t a0 = off[a], a1 = off[a + 1], b0 = off[b], b1 = off[b + 1];
    if (a0 == a1 || b0 == b1) return;
    const bool a_short = a1 - a0 <= b1 - b0;
    const int32_t t = rs_table(rs, a_short ? b : a);
    const bool cut = from != INT32_MIN;
    if (t >= 0) {
        int64_t s0 = a_short ? a0 : b0;
        const int64_t s1 = a_short ? a1 : b1;
        if (cut) s0 = lower_bound_row(nb, s0, s1, from);
        const int32_t zmax = nb[(a_short ? b1 : a1) - 1];
        for (int64_t p = s0; p < s1; ++p) {
            const int32_t z = nb[p];
            if (z > zmax) break;
            if (rs_member(rs, t, z)) f(z);
        }
        return;
    }
    if (cut) {
        a0 = lower_bound_row(nb, a0, a1, from);
        b0 = lower_bound_row(nb, b0, b1, from);
    }
    intersect_rows(nb, a0, a1, b0, b1, gallop, [&](int32_t z, int64_t, int64_t) { f(z); });
}

// The warp's hits of the ascending range S = [s0, s1) in the row of w, whose
// range is [l0, l1): chunk(hit, z) per 32 elements of S (every lane, warp-
// uniform control flow), hits ascending.  Through w's hash set when it has one
// (the caller passes w's whole row, or a part of it holding every element of S
// that is in the row), else by binary search in [l0, l1).
template <typename F>
__device__ __forceinline__ void warp_walk(const RowSets& rs, const int64_t* __restrict__ off,
                                          const int32_t* __restrict__ nb, int64_t s0, int64_t s1, int32_t w,
                                          int64_t l0, int64_t l1, int lane, F&& chunk)
{
    if (s0 >= s1 || l0 >= l1) return;
    const int32_t t = rs_table(rs, w);
    if (t >= 0) {
        const int32_t zmax = nb[off[w + 1] - 1];
        warp_scan(nb, s0, s1, zmax, lane, [&](int32_t z) { return rs_member(rs, t, z); }, chunk);
    } else {
        warp_chunks(nb, s0, s1, l0, l1, lane,
                    [&](int64_t lo, int64_t hi, int32_t v) { return lower_bound_row(nb, lo, hi, v); }, chunk);
    }
}

}  // namespace rtr
