// Sorted-row intersection helpers shared by the counting kernels
// (count.cu, count_rows.cu, noalloc.cu).  Rows of the CSR hold neighbour ids
// strictly ascending (makeCSR + sortById, RTRex_Sequential/Graph.cpp:344-384),
// so every helper visits common neighbours in ascending order -- the order in
// which commonNbr (RTRex_Sequential/Escape/Decomposition.h:70-115) meets the
// triangles of an edge -- which is what the ordered folds need.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtr {

__device__ __forceinline__ int64_t lower_bound_row(const int32_t* __restrict__ nb, int64_t lo, int64_t hi, int32_t x)
{
    while (lo < hi) {
        const int64_t mid = (lo + hi) >> 1;
        if (nb[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Visit common neighbours of rows [a0,a1) and [b0,b1) in ascending order:
// f(z, slot_in_a, slot_in_b).  Skewed pairs (lengths differing by more than
// `gallop`) binary-search the short row's elements in the long row; the others
// merge.  One thread.
template <typename F>
__device__ __forceinline__ void intersect_rows(const int32_t* __restrict__ nb, int64_t a0, int64_t a1, int64_t b0,
                                               int64_t b1, int gallop, F&& f)
{
    const int64_t la = a1 - a0, lb = b1 - b0;
    if (la <= 0 || lb <= 0) return;
    if (la * gallop < lb || lb * gallop < la) {
        const bool a_short = la <= lb;
        const int64_t s0 = a_short ? a0 : b0, s1 = a_short ? a1 : b1;
        int64_t lo = a_short ? b0 : a0;
        const int64_t l1 = a_short ? b1 : a1;
        for (int64_t p = s0; p < s1 && lo < l1; ++p) {
            const int32_t x = nb[p];
            lo = lower_bound_row(nb, lo, l1, x);
            if (lo < l1 && nb[lo] == x) {
                if (a_short) f(x, p, lo);
                else f(x, lo, p);
                ++lo;
            }
        }
        return;
    }
    int64_t i = a0, j = b0;
    int32_t x = nb[i], y = nb[j];
    while (true) {
        if (x < y) {
            if (++i >= a1) break;
            x = nb[i];
        } else if (x > y) {
            if (++j >= b1) break;
            y = nb[j];
        } else {
            f(x, i, j);
            if (++i >= a1 || ++j >= b1) break;
            x = nb[i];
            y = nb[j];
        }
    }
}

// Lane `lane`'s share of the common neighbours of rows A=[a0,a1) and B=[b0,b1),
// visited in ascending order: f(z, slot_in_a, slot_in_b).  The shorter row is
// cut into 32 contiguous pieces and the lane takes piece `lane` together with
// the part of the longer row between its piece's first value and the next
// piece's first value, so lane l's common neighbours all precede lane l+1's.
// Within its part a lane merges, or -- when the rows' lengths differ by more
// than `gallop` -- binary-searches each of its elements.
template <typename F>
__device__ __forceinline__ void warp_intersect_part(const int32_t* __restrict__ nb, int64_t a0, int64_t a1, int64_t b0,
                                                    int64_t b1, int gallop, int lane, F&& f)
{
    const int64_t la = a1 - a0, lb = b1 - b0;
    if (la <= 0 || lb <= 0) return;
    const bool a_short = la <= lb;
    const int64_t s0 = a_short ? a0 : b0, s1 = a_short ? a1 : b1;
    const int64_t l0 = a_short ? b0 : a0, l1 = a_short ? b1 : a1;
    const int64_t ls = s1 - s0, ll = l1 - l0;
    const int64_t piece = (ls + 31) / 32;
    const int64_t p0 = s0 + (int64_t)lane * piece;
    const int64_t p1 = p0 + piece < s1 ? p0 + piece : s1;
    if (p0 >= p1) return;
    int64_t lo = lower_bound_row(nb, l0, l1, nb[p0]);
    const int64_t hi = p1 < s1 ? lower_bound_row(nb, lo, l1, nb[p1]) : l1;
    if (ls * gallop < ll) {
        for (int64_t p = p0; p < p1 && lo < hi; ++p) {
            const int32_t x = nb[p];
            lo = lower_bound_row(nb, lo, hi, x);
            if (lo < hi && nb[lo] == x) {
                if (a_short) f(x, p, lo);
                else f(x, lo, p);
                ++lo;
            }
        }
        return;
    }
    int64_t i = p0, j = lo;
    if (j >= hi) return;
    int32_t x = nb[i], y = nb[j];
    while (true) {
        if (x < y) {
            if (++i >= p1) break;
            x = nb[i];
        } else if (x > y) {
            if (++j >= hi) break;
            y = nb[j];
        } else {
            if (a_short) f(x, i, j);
            else f(x, j, i);
            if (++i >= p1 || ++j >= hi) break;
            x = nb[i];
            y = nb[j];
        }
    }
}

// Warp-cooperative ordered intersection of a short row S=[s0,s1) with a long
// row L=[l0,l1) (both ascending): the warp walks S 32 elements at a time, lane k
// holding S[base+k]; every lane looks its element up in L with
// search(lo, l1, x) (a lower bound at or after the cursor lo), and
// chunk(hit, x) is called by all lanes with hit = whether the lane's element is
// in L.  Across and within chunks the hits come in ascending order of x, so a
// caller that folds the hits of each chunk in lane order folds them in
// ascending order overall.  Control flow is warp-uniform.
template <typename Search, typename F>
__device__ __forceinline__ void warp_chunks(const int32_t* __restrict__ nb, int64_t s0, int64_t s1, int64_t l0,
                                            int64_t l1, int lane, Search&& search, F&& chunk)
{
    int64_t lo = l0;
    for (int64_t base = s0; base < s1; base += 32) {
        const int64_t p = base + lane;
        const bool valid = p < s1;
        const int32_t x = valid ? nb[p] : 0x7fffffff;
        const int64_t pos = valid ? search(lo, l1, x) : l1;
        const bool hit = valid && pos >= l0 && pos < l1 && nb[pos] == x;
        chunk(hit, x);
        const int last = (s1 - base >= 32) ? 31 : (int)(s1 - base - 1);
        lo = __shfl_sync(0xffffffffu, pos, last);
        if (lo >= l1) break;
    }
}

// Ordered fold of the chunk's hits: the lanes with hit place w at their rank
// among the hits in the warp's shared-memory slots s (32 doubles), and every
// lane then adds them in rank order -- ascending x -- to acc; lanes whose rank
// is below `from` are left out of acc2 (both chains are optional: pass
// nullptr).  Returns the number of hits.
__device__ __forceinline__ int fold_hits(bool hit, double w, double* s, int lane, double* acc, double* acc2, int from2)
{
    const unsigned mask = __ballot_sync(0xffffffffu, hit);
    const int cnt = __popc(mask);
    if (cnt == 0) return 0;
    if (hit) s[__popc(mask & ((1u << lane) - 1u))] = w;
    __syncwarp();
    if (acc && acc2) {
        for (int j = 0; j < cnt; ++j) {
            const double v = s[j];
            *acc += v;
            if (j >= from2) *acc2 += v;
        }
    } else if (acc) {
        for (int j = 0; j < cnt; ++j) *acc += s[j];
    } else if (acc2) {
        for (int j = from2; j < cnt; ++j) *acc2 += s[j];
    }
    __syncwarp();
    return cnt;
}

}  // namespace rtr
