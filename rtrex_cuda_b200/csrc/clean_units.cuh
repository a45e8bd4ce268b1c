// Types shared by the two replays of the cascading clean: the warp-per-unit
// replay (clean.cu) and the round-parallel replay of large units
// (clean_rounds.cu).
#pragma once

#include "rtr_graph.cuh"

namespace rtr {

// One unit of the clean: a connected component of the triangle-carrying
// edges, with its seeds (sorted seed range) and its cascade-stack region.
struct UnitDesc {
    int64_t seed_begin;
    int64_t seed_end;
    int64_t stack_base;
    int64_t stack_cap;
    int64_t root;  // the unit's union-find root (smallest vertex id)
};

// One cascade-stack entry: the pair as deleteAndClean pushed it plus the
// static data its pop needs (degrees, triangle-list bounds), so a pop issues
// no lookups before its first dynamic load.  Seeds use the same descriptor.
struct StackEntry {
    int32_t e;        // forward rank of the edge
    int32_t first;    // Pair.first  (deleteAndClean's u)
    int32_t second;   // Pair.second (deleteAndClean's v)
    int32_t dfirst;   // deg(first)
    int32_t dsecond;  // deg(second)
    int32_t cnt;      // triangle-list length
    int64_t t0;       // triangle-list start
};
static_assert(sizeof(StackEntry) == 32, "StackEntry is 32 bytes");

// Streaming read of a triangle-list entry: the clean reads each list once, so
// entries are loaded evict-first and do not displace the edge records in L2.
__device__ __forceinline__ TriEntry ld_entry(const TriEntry* p)
{
    TriEntry t;
    int4* d = reinterpret_cast<int4*>(&t);
    d[0] = __ldcs(reinterpret_cast<const int4*>(p));
    d[1] = __ldcs(reinterpret_cast<const int4*>(p) + 1);
    return t;
}

// Orientation of a popped pair (u, v) as deleteAndClean sees it
// (Decomposition.h:178-186): the lower-degree endpoint's list is scanned.
struct PairSide {
    bool lower_is_a;  // lower == the smaller vertex id (the forward edge's a)
    int32_t lower, higher, dlow, dhigh;
};

__device__ __forceinline__ PairSide pair_side(const StackEntry& c)
{
    const bool lo_is_u = c.dfirst < c.dsecond;
    PairSide s;
    s.lower = lo_is_u ? c.first : c.second;
    s.higher = lo_is_u ? c.second : c.first;
    s.dlow = lo_is_u ? c.dfirst : c.dsecond;
    s.dhigh = lo_is_u ? c.dsecond : c.dfirst;
    s.lower_is_a = s.lower == (c.first < c.second ? c.first : c.second);
    return s;
}

// Round-parallel replay of the units order[0, nbig) (clean_rounds.cu): one
// thread block per unit on the stream `side`, concurrently with whatever the
// caller launches on the graph's stream; the per-vertex weights of those
// units are folded in afterwards, in the reference's order, by
// clean_rounds_finish on the graph's stream (after `side` is joined).
struct RoundReplay {
    int64_t nbig = 0;
    EdgeRec* rec = nullptr;
    const StackEntry* seeds = nullptr;
    const UnitDesc* units = nullptr;
    const uint64_t* order = nullptr;
    int32_t *nx = nullptr, *nx2 = nullptr, *dd = nullptr, *dd2 = nullptr, *inv = nullptr;
    int32_t* pop_wcnt = nullptr;
    uint32_t *logcnt = nullptr, *logoff = nullptr, *logtmp = nullptr;
    double* wbuf = nullptr;
    int32_t* zbuf = nullptr;
    int64_t *len = nullptr, *ubase = nullptr, *tmp = nullptr;
};
int clean_rounds_launch(rtr_graph* g, Scratch& sc, cudaStream_t side, EdgeRec* rec, const StackEntry* seeds,
                        const UnitDesc* units, const uint64_t* order, int64_t nbig, StackEntry* stacks,
                        RoundReplay* rr);
int clean_rounds_finish(rtr_graph* g, Scratch& sc, RoundReplay* rr);

}  // namespace rtr
