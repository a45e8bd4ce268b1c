// Hash sets of long CSR rows, for membership lookups that cost one or two
// independent loads instead of a binary search's chain of dependent ones.
// Built by build_row_sets (count_rows.cu) for every vertex of at least a given
// degree: open addressing with linear probing over a power-of-two table of at
// least twice the row's length (so every probe sequence ends), keys the
// neighbour ids, -1 empty.  Rows hold distinct ids, so a set answers exactly
// "is z a neighbour of w"; the counting folds only need that (the weight of a
// common neighbour z depends on z alone), not z's slot.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtr {

// rows of at least this many entries get a hash set
constexpr int kSetDegree = 256;

struct RowSets {
    const int32_t* tab;    // vertex -> its table, -1 for rows without one (null: no tables at all)
    const int64_t* toff;   // table -> first slot
    const int32_t* tbits;  // table -> log2 of its slot count
    const int32_t* slot;   // the keys, -1 for empty slots
};

__device__ __forceinline__ int32_t rs_table(const RowSets& r, int32_t w) { return r.tab ? r.tab[w] : -1; }

__device__ __forceinline__ uint32_t rs_hash(int32_t z, int bits)
{
    return ((uint32_t)z * 2654435761u) >> (32 - bits);
}

__device__ __forceinline__ bool rs_member(const RowSets& r, int32_t t, int32_t z)
{
    const int64_t base = r.toff[t];
    const int bits = r.tbits[t];
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t h = rs_hash(z, bits);
    while (true) {
        const int32_t k = r.slot[base + h];
        if (k == z) return true;
        if (k < 0) return false;
        h = (h + 1u) & mask;
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
    for (int64_t base = s0; base < s1; base += 32) {
        const int64_t p = base + lane;
        const bool valid = p < s1;
        const int32_t x = valid ? nb[p] : 0x7fffffff;
        if (__all_sync(0xffffffffu, x > zmax)) break;
        const bool hit = valid && x <= zmax && pred(x);
        chunk(hit, x);
    }
}

}  // namespace rtr
