// Weighted triangle counting without TriEntry lists ("rows" layout), for
// graphs whose 32-byte-per-entry triangle lists do not fit in HBM (R-MAT
// scale 22 has 2.1 G triangles, ~200 GB of lists; scale 24 10.3 G).
// commonNbr itself keeps no lists (RTRex_Sequential/Escape/Decomposition.h:
// 70-115); its two ordered folds are
//   perEdge[(x,y)] = left fold over z in N(x) & N(y) ascending of w(x,y,z)
//   perVertex[x]   = left fold over y in N(x) ascending, then over
//                    z in N(x) & N(y), z > y ascending, of w(x,y,z)
// with w(x,y,z) = 1/double(dx*dy*dz).
//
// What runs before this (count.cu): one intersection per undirected edge
// gives support, the triangle total, perEdge (light edges by a thread, heavy
// ones by a warp walking the shorter row in order) and, for every directed
// slot (x,y), cgt = #{z in N(x) & N(y) : z > y} -- the number of terms slot
// (x,y) adds to perVertex[x].  This file makes perVertex from that:
//   lists     the exclusive scan of cgt gives every slot a list of its z > y,
//             4 bytes each (3 per triangle: ~124 GB at R-MAT scale 24); an
//             entry holds deg z, all that the fold needs of z.
//             Slots are taken in windows of whole rows that fit in the free
//             HBM (one window when everything fits).
//   fill      one more pass per edge (u < v), restricted to z > u, writes
//             both slots' lists in ascending z: deg z for z > u to slot (v,u),
//             for z > v to slot (u,v).  k_fill_light: a thread per light edge
//             (the intersection again); k_fill_heavy: a warp per heavy edge,
//             which reads the count's hit masks (one 32-bit word per 32
//             elements of the shorter row) instead of repeating the lookups,
//             hits ranked by ballot.
//   fold      perVertex[x] = the left fold of x's slots' lists in slot order
//             (y ascending), each in z order -- exactly commonNbr's order.
//             k_vfold_thread: a thread per vertex of fewer than warp_min terms;
//             k_vfold_warp: a warp per vertex of fewer than 64 x warp_min, the
//             weights of 32 terms computed by the lanes (each term's slot by a
//             shuffle search over 32 slot ends) and added in lane order;
//             k_vfold_block: a thread block per larger vertex, seven warps
//             producing weights into shared memory and one warp running the
//             add chain -- the one sequential part (~10^8 dependent adds for
//             the largest R-MAT scale-24 vertex).  Vertices are dealt from
//             queues in descending term count.
// Membership lookups use the hash sets of the long rows (rowsets.cuh,
// build_row_sets below).  The lists (and the hit masks) are graph-owned
// buffers that later counts reuse.
#include "intersect.cuh"
#include "primitives.cuh"
#include "rowsets.cuh"
#include "rtr_graph.cuh"

namespace rtr {

namespace {

constexpr int kFillBlock = 256;
constexpr int kHeavyBlock = 128;
constexpr int kFoldBlock = 256;

struct FillArgs {
    const int64_t* off;
    const int32_t* nb;
    const int32_t* esrc;
    const int32_t* partner;
    const int32_t* deg;
    const int32_t* fwd;
    int64_t m;
    int heavy_edge;
    int gallop;
    RowSets rs;
    const int64_t* lpos;  // [m2+1] first list entry of every slot (all windows numbered together)
    int64_t p0, p1;       // the window's slots
    int64_t e0;           // lpos[p0]: entry e of the window lives at lists[e - e0]
    int32_t* lists;
    const int64_t* moff;    // heavy edge h's hit masks: masks[moff[h] .. moff[h+1]) (null: none)
    const uint32_t* masks;  // bit k of word j: element 32j + k of the shorter row is common
};

__device__ __forceinline__ bool in_window(const FillArgs& a, int64_t p) { return p >= a.p0 && p < a.p1; }

// Light edges (deg u + deg v below heavy_edge), a thread each.
__global__ void __launch_bounds__(kFillBlock) k_fill_light(FillArgs a)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < a.m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = a.fwd[k];
        const int32_t u = a.esrc[i], v = a.nb[i];
        if (a.deg[u] + a.deg[v] >= a.heavy_edge) continue;
        const int64_t r = a.partner[i];
        const bool wi = in_window(a, i), wr = in_window(a, r);
        if (!wi && !wr) continue;
        // each slot's list ends where the next begins: the writes stay inside it
        int64_t qi = a.lpos[i] - a.e0, qr = a.lpos[r] - a.e0;
        const int64_t qi1 = a.lpos[i + 1] - a.e0, qr1 = a.lpos[r + 1] - a.e0;
        thread_common(a.rs, a.off, a.nb, u, v, wr ? u + 1 : v + 1, a.gallop, [&](int32_t z) {
            const int32_t dz = a.deg[z];
            if (wr && qr < qr1) a.lists[qr++] = dz;
            if (wi && z > v && qi < qi1) a.lists[qi++] = dz;
        });
    }
}

// Heavy edges, a warp each, from the count's heavy-edge list.
__global__ void __launch_bounds__(kHeavyBlock, 8) k_fill_heavy(FillArgs a, const int32_t* __restrict__ heavy_list,
                                                             const unsigned* __restrict__ nheavy)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const int64_t nh = *nheavy;
    const int64_t nwarps = (int64_t)gridDim.x * (kHeavyBlock / 32);
    for (int64_t h = (int64_t)blockIdx.x * (kHeavyBlock / 32) + (threadIdx.x >> 5); h < nh; h += nwarps) {
        const int64_t i = a.fwd[heavy_list[h]];
        const int32_t u = a.esrc[i], v = a.nb[i];
        const int64_t r = a.partner[i];
        const bool wi = in_window(a, i), wr = in_window(a, r);
        if (!wi && !wr) continue;  // uniform across the warp
        int64_t qi = a.lpos[i] - a.e0, qr = a.lpos[r] - a.e0;
        const int64_t qi1 = a.lpos[i + 1] - a.e0, qr1 = a.lpos[r + 1] - a.e0;  // the writes stay inside each list
        const int32_t from = wr ? u + 1 : v + 1;
        const int64_t u0 = a.off[u], u1 = a.off[u + 1], v0 = a.off[v], v1 = a.off[v + 1];
        const bool u_short = u1 - u0 <= v1 - v0;
        const int64_t s1 = u_short ? u1 : v1;
        const int64_t s0 = lower_bound_row(a.nb, u_short ? u0 : v0, s1, from);
        auto emit = [&](bool hit, int32_t z, int32_t dz) {
            const bool to_r = hit && wr, to_i = hit && wi && z > v;
            const unsigned mr = __ballot_sync(0xffffffffu, to_r);
            const unsigned mi = __ballot_sync(0xffffffffu, to_i);
            const int64_t wr_at = qr + __popc(mr & lt), wi_at = qi + __popc(mi & lt);
            if (to_r && wr_at < qr1) a.lists[wr_at] = dz;
            if (to_i && wi_at < qi1) a.lists[wi_at] = dz;
            qr += __popc(mr);
            qi += __popc(mi);
        };
        const int32_t t = rs_table(a.rs, u_short ? v : u);
        if (t >= 0 && a.masks) {
            // the count's hit masks: only chunks with hits are read, no lookups
            const int64_t w0 = a.moff[h], nw = a.moff[h + 1] - w0;
            const int64_t sa = u_short ? u0 : v0;  // where the count's walk began
            for (int64_t cb = (s0 - sa) / 32; cb < nw; cb += 32) {
                const int64_t cc = cb + lane;
                const uint32_t mw = cc < nw ? __ldg(a.masks + w0 + cc) : 0u;
                unsigned nz = __ballot_sync(0xffffffffu, mw != 0u);
                while (nz) {  // uniform across the warp
                    // up to four chunks with hits at a time: their element loads, then their
                    // degree loads, in flight together; emitted in chunk order
                    constexpr int Q = 4;
                    int js[Q];
                    uint32_t ms[Q];
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        js[q] = -1;
                        ms[q] = 0u;
                        if (nz) {
                            js[q] = __ffs(nz) - 1;
                            nz &= nz - 1u;
                            ms[q] = __shfl_sync(0xffffffffu, mw, js[q]);
                        }
                    }
                    bool hit[Q];
                    int32_t z[Q], dz[Q];
#pragma unroll
                    for (int q = 0; q < Q; ++q) {
                        const int64_t p = sa + (cb + js[q]) * 32 + lane;
                        hit[q] = js[q] >= 0 && ((ms[q] >> lane) & 1u) && p >= s0;  // before s0: z < from
                        z[q] = hit[q] ? a.nb[p] : 0;
                    }
#pragma unroll
                    for (int q = 0; q < Q; ++q) dz[q] = hit[q] ? a.deg[z[q]] : 0;
#pragma unroll
                    for (int q = 0; q < Q; ++q)
                        if (js[q] >= 0) emit(hit[q], z[q], dz[q]);
                }
            }
        } else if (t >= 0) {
            constexpr int B = 4;  // 4 chunks per step, their lookups (then degrees) in flight together
            warp_probe_walk<B>(a.rs, t, a.nb, s0, s1, a.nb[(u_short ? v1 : u1) - 1], lane,
                               [&](const bool (&hit)[B], const int32_t (&x)[B]) {
                                   int32_t dz[B];
#pragma unroll
                                   for (int b = 0; b < B; ++b) dz[b] = hit[b] ? a.deg[x[b]] : 0;
#pragma unroll
                                   for (int b = 0; b < B; ++b) emit(hit[b], x[b], dz[b]);
                               });
        } else {
            warp_walk(a.rs, a.off, a.nb, s0, s1, u_short ? v : u, u_short ? v0 : u0, u_short ? v1 : u1, lane,
                      [&](bool hit, int32_t z) { emit(hit, z, hit ? a.deg[z] : 0); });
        }
    }
}

struct FoldArgs {
    const int64_t* off;
    const int32_t* nb;
    const int32_t* deg;
    const int64_t* lpos;
    int64_t e0;
    const int32_t* lists;
    double* pv;
    int64_t x0, x1;  // the window's vertices
    int64_t warp_min;
};

__device__ __forceinline__ int64_t terms_of(const FoldArgs& a, int64_t x)
{
    return a.lpos[a.off[x + 1]] - a.lpos[a.off[x]];
}

__global__ void __launch_bounds__(kFoldBlock) k_vfold_thread(FoldArgs a)
{
    for (int64_t x = a.x0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; x < a.x1;
         x += (int64_t)gridDim.x * blockDim.x) {
        const int64_t q0 = a.off[x], q1 = a.off[x + 1];
        int64_t e = a.lpos[q0];
        if (a.lpos[q1] - e >= a.warp_min) continue;  // k_vfold_warp
        const int64_t dx = a.deg[x];
        double acc = 0.0;
        for (int64_t p = q0; p < q1; ++p) {
            const int64_t e1 = a.lpos[p + 1];
            if (e1 == e) continue;
            const int64_t dxy = dx * (int64_t)a.deg[a.nb[p]];
            for (; e < e1; ++e) acc += 1.0 / (double)(dxy * (int64_t)a.lists[e - a.e0]);
        }
        a.pv[x] = acc;
    }
}

// Vertices of at least warp_min terms, big[] in descending term count, dealt
// to warps by an atomic counter.  A warp takes 32 slots at a time: lane j holds
// slot j's term count, an inclusive scan across lanes gives each term of the
// group its slot (a five-step search over the lanes), the lanes compute 32
// weights at once and the warp adds them in lane order.
__global__ void __launch_bounds__(kFoldBlock) k_vfold_warp(FoldArgs a, const int32_t* __restrict__ big,
                                                            int64_t nbig, unsigned long long* __restrict__ next)
{
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned long long b = 0;
        if (lane == 0) b = atomicAdd(next, 1ull);
        b = __shfl_sync(0xffffffffu, b, 0);
        if ((int64_t)b >= nbig) break;
        const int64_t x = big[b];
        if (x < a.x0 || x >= a.x1) continue;  // another window's vertex
        const int64_t dx = a.deg[x];
        const int64_t q0 = a.off[x], q1 = a.off[x + 1];
        double acc = 0.0;
        for (int64_t g0 = q0; g0 < q1; g0 += 32) {
            const int64_t p = g0 + lane;
            const bool valid = p < q1;
            const int64_t len = valid ? a.lpos[p + 1] - a.lpos[p] : 0;
            int64_t inc = len;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int64_t t = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += t;
            }
            const int64_t G = __shfl_sync(0xffffffffu, inc, 31);
            if (G == 0) continue;
            const int64_t dxy = (valid && len > 0) ? dx * (int64_t)a.deg[a.nb[p]] : 0;
            const int64_t base = a.lpos[g0] - a.e0;
            // Software pipeline over blocks of 4 chunks (128 terms): the lanes' terms
            // (the degrees of their z) are loaded one block ahead of the add chain.
            auto dload = [&](int64_t k0) -> int32_t {
                const int64_t e = k0 + lane;
                return e < G ? __ldg(a.lists + base + e) : 1;
            };
            int32_t dA[4];
#pragma unroll
            for (int c = 0; c < 4; ++c) dA[c] = dload(32 * c);
            for (int64_t b0 = 0; b0 < G; b0 += 128) {
                int32_t dB[4];
#pragma unroll
                for (int c = 0; c < 4; ++c) dB[c] = dload(b0 + 128 + 32 * c);
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int64_t k0 = b0 + 32 * c;
                    if (k0 < G) {  // uniform across the warp
                        const int64_t e = k0 + lane;
                        // slot of term e: the number of lanes whose inclusive count is <= e
                        int q = 0;
#pragma unroll
                        for (int step = 16; step > 0; step >>= 1) {
                            const int64_t cq = __shfl_sync(0xffffffffu, inc, q + step - 1);
                            if (cq <= e) q += step;
                        }
                        const int64_t dq = __shfl_sync(0xffffffffu, dxy, q & 31);
                        const double w = e < G ? 1.0 / (double)(dq * (int64_t)dA[c]) : 0.0;
                        const int cnt = G - k0 < 32 ? (int)(G - k0) : 32;
#pragma unroll
                        for (int t = 0; t < 32; ++t) {
                            const double v = __shfl_sync(0xffffffffu, w, t);
                            if (t < cnt) acc += v;
                        }
                    }
                }
#pragma unroll
                for (int c = 0; c < 4; ++c) dA[c] = dB[c];
            }
        }
        if (lane == 0) a.pv[x] = acc;
    }
}

// The largest vertices (at least block_min terms), a thread block each, from
// the front of big[] (descending term count), two blocks per SM: one warp runs
// the add chain and nothing else, the other seven produce the weights.  The terms of
// x are cut into segments of kSeg, whose first slots k_seg_slots finds ahead of
// time; round r gives the producers the next 7 segments, each lane loading 12
// terms and their degrees at a time with all loads in flight at once and
// writing the weights to the segment's shared-memory buffer (set r&1), while
// the chain warp adds the previous round's 7 segments in order, from 16-byte
// shared-memory loads issued ahead of the adds.  One block barrier per round;
// the chain costs about one double add latency per term.
constexpr int kSeg = 768;
constexpr int kHalfChunks = kSeg / 64;  // a producer takes its segment in two halves of 12 chunks
constexpr int kProducers = kFoldBlock / 32 - 1;
constexpr size_t kBlockFoldSmem = sizeof(double) * 2 * kProducers * kSeg;

__global__ void __launch_bounds__(kFoldBlock, 2)
    k_vfold_block(FoldArgs a, const int32_t* __restrict__ huge, int64_t nhuge, const int64_t* __restrict__ segoff,
                  const int32_t* __restrict__ segslot, unsigned long long* __restrict__ next)
{
    extern __shared__ double s_buf[];  // [2][kProducers][kSeg]
    __shared__ int64_t s_h;
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    // the chain warp: picked by block index, so that the chains of the blocks an SM holds tend to
    // sit on different schedulers; the other warps are producers 0..6 (pid < 0: the chain warp)
    const int chain = (int)(blockIdx.x & 3);
    const int pid = wib == chain ? -1 : (wib < chain ? wib : wib - 1);
    while (true) {
        if (threadIdx.x == 0) {
            const unsigned long long b = atomicAdd(next, 1ull);
            s_h = (int64_t)b < nhuge ? (int64_t)b : -1;
        }
        __syncthreads();
        const int64_t h = s_h;
        if (h < 0) break;  // uniform across the block
        const int64_t x = huge[h];
        if (x >= a.x0 && x < a.x1) {
            const int64_t q0 = a.off[x], q1 = a.off[x + 1];
            const int64_t E0 = a.lpos[q0], T = a.lpos[q1] - E0;
            const int64_t dx = a.deg[x];
            const int64_t nseg = (T + kSeg - 1) / kSeg;
            const int64_t rounds = (nseg + kProducers - 1) / kProducers;
            const int32_t* sslot = segslot + segoff[h];
            // producer pid (0..6): the weights of segment sg into set `set`.  Lane j
            // holds the term end and dx*dy of slot gp+j; a term's slot is the number of
            // lanes whose end is <= it (a five-step shuffle search).
            auto produce = [&](int64_t sg, int set) {
                double* buf = s_buf + ((int64_t)set * kProducers + pid) * kSeg;
                const int64_t t0 = sg * kSeg;
                if (t0 >= T) return;  // uniform across the warp
                const int64_t t1 = t0 + kSeg < T ? t0 + kSeg : T;
                int64_t gp = q0 + sslot[sg];  // the slot of term t0
                int64_t endj = 0, dyj = 0, gend = 0;
                auto load_group = [&]() {
                    const int64_t sl = gp + lane;
                    endj = sl < q1 ? a.lpos[sl + 1] - E0 : 0x7fffffffffffffffll;
                    dyj = sl < q1 ? dx * (int64_t)a.deg[a.nb[sl]] : 0;
                    gend = __shfl_sync(0xffffffffu, endj, 31);  // the group holds the terms below gend
                };
                load_group();
#pragma unroll 1
                for (int half = 0; half < 2; ++half) {
                    const int64_t h0 = t0 + half * (kSeg / 2);
                    int32_t dz[kHalfChunks];
#pragma unroll
                    for (int c = 0; c < kHalfChunks; ++c) {
                        const int64_t e = h0 + 32 * c + lane;
                        dz[c] = e < t1 ? __ldg(a.lists + (E0 + e - a.e0)) : 1;
                    }
#pragma unroll
                    for (int c = 0; c < kHalfChunks; ++c) {
                        const int64_t e = h0 + 32 * c + lane;
                        double w = 0.0;
                        bool need = e < t1;
                        while (__any_sync(0xffffffffu, need)) {  // ends: the last slot's end is T
                            int q = 0;
#pragma unroll
                            for (int step = 16; step > 0; step >>= 1) {
                                const int64_t cq = __shfl_sync(0xffffffffu, endj, q + step - 1);
                                if (cq <= e) q += step;
                            }
                            const int64_t dq = __shfl_sync(0xffffffffu, dyj, q & 31);
                            if (need && e < gend) {
                                w = 1.0 / (double)(dq * (int64_t)dz[c]);
                                need = false;
                            }
                            if (__any_sync(0xffffffffu, need)) {
                                gp += 32;
                                load_group();
                            }
                        }
                        buf[half * (kSeg / 2) + 32 * c + lane] = w;
                    }
                }
            };
            double acc = 0.0;  // meaningful in the chain warp
            if (pid >= 0) produce(pid, 0);
            __syncthreads();
            for (int64_t r = 0; r < rounds; ++r) {
                const int set = (int)(r & 1);
                if (pid < 0) {
                    // 16-byte broadcast loads, issued ahead of the adds (no shuffles: a double
                    // shuffle is two instructions)
                    for (int w = 0; w < kProducers; ++w) {
                        const int64_t t0 = (r * kProducers + w) * kSeg;
                        if (t0 >= T) break;
                        const int cnt = T - t0 < kSeg ? (int)(T - t0) : kSeg;
                        const double* bb = s_buf + ((int64_t)set * kProducers + w) * kSeg;
                        const double2* b2 = reinterpret_cast<const double2*>(bb);
                        int k = 0;
#pragma unroll 4
                        for (; k + 8 <= cnt; k += 8) {
                            const double2 p0 = b2[k / 2], p1 = b2[k / 2 + 1], p2 = b2[k / 2 + 2], p3 = b2[k / 2 + 3];
                            acc += p0.x;
                            acc += p0.y;
                            acc += p1.x;
                            acc += p1.y;
                            acc += p2.x;
                            acc += p2.y;
                            acc += p3.x;
                            acc += p3.y;
                        }
                        for (; k < cnt; ++k) acc += bb[k];
                    }
                } else if (r + 1 < rounds) {
                    produce((r + 1) * kProducers + pid, set ^ 1);
                }
                __syncthreads();
            }
            if (pid < 0 && lane == 0) a.pv[x] = acc;
        }
        __syncthreads();  // s_h is rewritten next
    }
}

// Segments of the block-folded vertices: how many each has, and the slot (from
// the row's start) that holds each segment's first term.
__global__ void k_seg_counts(const int64_t* __restrict__ off, const int64_t* __restrict__ lpos,
                             const int32_t* __restrict__ huge, int64_t nhuge, int64_t* __restrict__ cnt)
{
    for (int64_t h = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; h <= nhuge; h += (int64_t)gridDim.x * blockDim.x) {
        if (h == nhuge) {
            cnt[h] = 0;
            continue;
        }
        const int64_t x = huge[h];
        const int64_t T = lpos[off[x + 1]] - lpos[off[x]];
        cnt[h] = (T + kSeg - 1) / kSeg;
    }
}

__global__ void k_seg_slots(const int64_t* __restrict__ off, const int64_t* __restrict__ lpos,
                            const int32_t* __restrict__ huge, int64_t nhuge, const int64_t* __restrict__ segoff,
                            int32_t* __restrict__ segslot)
{
    for (int64_t h = blockIdx.x; h < nhuge; h += gridDim.x) {
        const int64_t x = huge[h];
        const int64_t q0 = off[x], q1 = off[x + 1], E0 = lpos[q0];
        const int64_t ns = segoff[h + 1] - segoff[h];
        for (int64_t sg = threadIdx.x; sg < ns; sg += blockDim.x) {
            const int64_t target = E0 + sg * kSeg;
            int64_t lo = q0, hi = q1 - 1;  // the last p with lpos[p] <= target
            while (lo < hi) {
                const int64_t mid = (lo + hi + 1) >> 1;
                if (lpos[mid] <= target) lo = mid;
                else hi = mid - 1;
            }
            segslot[segoff[h] + sg] = (int32_t)(lo - q0);
        }
    }
}

// Vertices of at least warp_min terms, keyed for a descending sort by term count.
__global__ void k_big_keys(const int64_t* __restrict__ off, const int64_t* __restrict__ lpos, int64_t n,
                           int64_t warp_min, int64_t block_min, uint64_t* __restrict__ keys,
                           unsigned* __restrict__ nbig)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int64_t t = lpos[off[v + 1]] - lpos[off[v]];
        if (t >= block_min) atomicAdd(nbig + 1, 1u);
        if (t >= warp_min) {
            const uint64_t tc = t < 0xffffffffll ? (uint64_t)t : 0xffffffffull;
            keys[atomicAdd(nbig, 1u)] = ((0xffffffffull - tc) << 32) | (uint64_t)v;
        }
    }
}

__global__ void k_low_ids(const uint64_t* __restrict__ keys, int64_t nk, int32_t* __restrict__ ids)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nk; i += (int64_t)gridDim.x * blockDim.x)
        ids[i] = (int32_t)(keys[i] & 0xffffffffu);
}

// The largest x1 in (x0, n] whose window [x0, x1) holds at most `limit` list
// entries (x0 + 1 when vertex x0 alone holds more: the caller reports that).
__global__ void k_window_end(const int64_t* __restrict__ off, const int64_t* __restrict__ lpos, int64_t n, int64_t x0,
                             int64_t limit, int64_t* __restrict__ out)
{
    const int64_t base = lpos[off[x0]];
    int64_t lo = x0 + 1, hi = n;  // answer in [lo, hi]
    while (lo < hi) {
        const int64_t mid = (lo + hi + 1) >> 1;
        if (lpos[off[mid]] - base <= limit) lo = mid;
        else hi = mid - 1;
    }
    *out = lo;
}

// Row sets: the vertices of at least min_deg neighbours, numbered in id order
// (flag + scan), each with a power-of-two number of 8-key buckets, >= 4 slots
// per key.
__global__ void k_rs_flags(const int32_t* __restrict__ deg, int64_t n, int min_deg, int64_t* __restrict__ flag)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v <= n; v += (int64_t)gridDim.x * blockDim.x)
        flag[v] = (v < n && deg[v] >= min_deg) ? 1 : 0;
}

__global__ void k_rs_sizes(const int32_t* __restrict__ deg, int64_t n, const int64_t* __restrict__ num,
                           int32_t* __restrict__ tab, int32_t* __restrict__ owner, int32_t* __restrict__ tbits,
                           int64_t* __restrict__ tsize)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        if (num[v + 1] == num[v]) {
            tab[v] = -1;
            continue;
        }
        const int32_t t = (int32_t)num[v];
        int bits = 0;
        while ((int64_t)kBucketKeys << bits < 4ll * deg[v]) ++bits;
        tab[v] = t;
        owner[t] = (int32_t)v;
        tbits[t] = bits;
        tsize[t] = (int64_t)kBucketKeys << bits;
    }
}

// A warp per table (dealt modulo the warp count) inserts its row: each key
// takes the first empty slot of the first bucket, from its own, that has one
// (the table is at most a quarter full, so every key finds one).
__global__ void k_rs_insert(const int32_t* __restrict__ owner, int64_t nt, const int64_t* __restrict__ off,
                            const int32_t* __restrict__ nb, const int64_t* __restrict__ toff,
                            const int32_t* __restrict__ tbits, int32_t* __restrict__ slot)
{
    const int lane = threadIdx.x & 31;
    const int64_t nwarps = (int64_t)gridDim.x * (blockDim.x / 32);
    for (int64_t t = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) / 32; t < nt; t += nwarps) {
        const int32_t v = owner[t];
        const int bits = tbits[t];
        const uint32_t mask = (1u << bits) - 1u;
        int32_t* tb = slot + toff[t];
        for (int64_t p = off[v] + lane; p < off[v + 1]; p += 32) {
            const int32_t z = nb[p];
            bool placed = false;
            for (uint32_t b = rs_hash(z, bits); !placed; b = (b + 1u) & mask)
                for (int k = 0; k < kBucketKeys && !placed; ++k)
                    placed = atomicCAS(&tb[(int64_t)b * kBucketKeys + k], -1, z) == -1;
        }
    }
}

}  // namespace

// Hash sets of every row of at least min_deg entries, in scratch (live until
// sc is released); *out stays empty when no row qualifies.
int build_row_sets(rtr_graph* g, Scratch& sc, int min_deg, RowSets* out)
{
    *out = RowSets{nullptr, nullptr, nullptr, nullptr};
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    int64_t* flag = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    int64_t* num = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    int64_t* tmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(n + 1));
    int32_t* tab = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    if (!flag || !num || !tmp || !tab) {
        set_error("device allocation failed (row sets)");
        return RTR_ERR_CUDA;
    }
    k_rs_flags<<<grid_for(n + 1, 256), 256, 0, s>>>(g->deg, n, min_deg, flag);
    exclusive_scan_i64(flag, num, n + 1, nullptr, tmp, s);
    int64_t nt = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nt, num + n, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->launches += 2;
    if (nt == 0) return RTR_OK;
    int32_t* owner = (int32_t*)sc.get(sizeof(int32_t) * (nt + 1));
    int32_t* tbits = (int32_t*)sc.get(sizeof(int32_t) * (nt + 1));
    int64_t* tsize = (int64_t*)sc.get(sizeof(int64_t) * (nt + 1));
    int64_t* toff = (int64_t*)sc.get(sizeof(int64_t) * (nt + 1));
    int64_t* ltmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nt + 1));
    if (!owner || !tbits || !tsize || !toff || !ltmp) {
        set_error("device allocation failed (row sets)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(tsize + nt, 0, sizeof(int64_t), s));
    k_rs_sizes<<<grid_for(n, 256), 256, 0, s>>>(g->deg, n, num, tab, owner, tbits, tsize);
    exclusive_scan_i64(tsize, toff, nt + 1, nullptr, ltmp, s);
    int64_t total = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&total, toff + nt, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    int32_t* slot = (int32_t*)sc.get(sizeof(int32_t) * (total + 1));
    if (!slot) {
        set_error("device allocation failed (row sets: %lld slots)", (long long)total);
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(slot, 0xff, sizeof(int32_t) * (total + 1), s));
    k_rs_insert<<<grid_for(1ll << 40, 256, 8), 256, 0, s>>>(owner, nt, g->offsets, g->nbors, toff, tbits, slot);
    g->launches += 3;
    RTR_CUDA_TRY(cudaGetLastError());
    *out = RowSets{tab, toff, tbits, slot};
    return RTR_OK;
}

// perVertex of every vertex from per-slot lists; the caller has run the edge
// pass (support, total, perEdge of all edges, cgt).  Synchronises the graph's
// stream.
int count_rows(rtr_graph* g, Scratch& sc, const RowSets& rs, const int64_t* cgt, int64_t* lpos,
               const int32_t* heavy_list, const unsigned* nheavy, const int64_t* moff, const uint32_t* masks)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m2 = g->m2, m = g->m;
    if (!cgt) {
        set_error("rows layout without per-slot term counts (count mode 1 keeps the lists)");
        return RTR_ERR_STATE;
    }
    int64_t* tmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(m2 + 1));
    uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    unsigned* d_nbig = (unsigned*)sc.get(sizeof(unsigned) * 2);  // [0] warp or block folds, [1] block folds
    unsigned long long* next = (unsigned long long*)sc.get(sizeof(unsigned long long) * 2);  // [0] warps [1] blocks
    int64_t* d_x1 = (int64_t*)sc.get(sizeof(int64_t) * 2);
    if (!tmp || !keys || !alt || !d_nbig || !next || !d_x1) {
        set_error("device allocation failed (rows layout)");
        return RTR_ERR_CUDA;
    }
    exclusive_scan_i64(cgt, lpos, m2 + 1, nullptr, tmp, s);
    // a warp from warp_min terms, a thread block from 64 x warp_min
    const int64_t warp_min = g->count_hub;
    const int64_t block_min = 64 * warp_min;
    RTR_CUDA_TRY(cudaMemsetAsync(d_nbig, 0, 2 * sizeof(unsigned), s));
    k_big_keys<<<grid_for(n, 256), 256, 0, s>>>(g->offsets, lpos, n, warp_min, block_min, keys, d_nbig);
    int64_t want = 0;
    unsigned nb2[2] = {0, 0};
    RTR_CUDA_TRY(cudaMemcpyAsync(&want, lpos + m2, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(nb2, d_nbig, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->launches += 2;
    const unsigned nbig = nb2[0], nhuge = nb2[1];  // big[0, nhuge) take a block, the rest a warp
    int32_t* big = nullptr;
    if (nbig > 0) {
        void* rtmp = sc.get(radix_temp_bytes(nbig));
        big = (int32_t*)sc.get(sizeof(int32_t) * (nbig + 1));
        if (!rtmp || !big) {
            set_error("device allocation failed (rows layout)");
            return RTR_ERR_CUDA;
        }
        uint64_t* sorted = radix_sort_u64(keys, alt, nbig, 64, rtmp, s);
        k_low_ids<<<grid_for(nbig, 256), 256, 0, s>>>(sorted, nbig, big);
        g->launches += 1 + 3 * 8;
    }
    // the block-folded vertices' segments and the slot each one starts in
    int64_t* segoff = nullptr;
    int32_t* segslot = nullptr;
    if (nhuge > 0) {
        int64_t* scnt = (int64_t*)sc.get(sizeof(int64_t) * (nhuge + 1));
        segoff = (int64_t*)sc.get(sizeof(int64_t) * (nhuge + 1));
        int64_t* stmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nhuge + 1));
        if (!scnt || !segoff || !stmp) {
            set_error("device allocation failed (rows layout)");
            return RTR_ERR_CUDA;
        }
        k_seg_counts<<<grid_for(nhuge + 1, 256), 256, 0, s>>>(g->offsets, lpos, big, nhuge, scnt);
        exclusive_scan_i64(scnt, segoff, nhuge + 1, nullptr, stmp, s);
        int64_t nseg = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nseg, segoff + nhuge, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        segslot = (int32_t*)sc.get(sizeof(int32_t) * (nseg + 1));
        if (!segslot) {
            set_error("device allocation failed (rows layout)");
            return RTR_ERR_CUDA;
        }
        k_seg_slots<<<grid_for(1ll << 40, 256, 4), 256, 0, s>>>(g->offsets, lpos, big, nhuge, segoff, segslot);
        g->launches += 3;
    }
    // the lists: all of them when they fit in the free HBM (less 1 GiB), else windows of whole
    // rows; a graph-owned buffer, reused by later counts of the graph
    const int64_t margin = 1ll << 30;
    int64_t room = 0;
    int32_t* lists = nullptr;
    if (g->rows_lists_cap >= (int64_t)sizeof(int32_t) * (want + 1)) {
        room = want;
        lists = (int32_t*)g->rows_lists;
    } else {
        const int64_t avail = (int64_t)device_avail_bytes(g) + g->rows_lists_cap;
        const int64_t fit = avail > margin ? (avail - margin) / (int64_t)sizeof(int32_t) - 1 : 0;
        room = want < fit ? want : fit;
        // the estimate counts the pool's cached blocks; halve until an allocation succeeds
        for (int attempt = 0; attempt < 8 && !lists && room >= 0; ++attempt) {
            lists = (int32_t*)grow_owned(g, &g->rows_lists, &g->rows_lists_cap,
                                         (int64_t)sizeof(int32_t) * (room + 1));
            if (!lists) room /= 2;
        }
        cudaGetLastError();  // a failed attempt's allocation error is not the caller's
    }
    if (!lists) {
        set_error("device allocation failed (rows layout: %lld list entries)", (long long)(room + 1));
        return RTR_ERR_CUDA;
    }
    if (g->rows_window_cap > 0 && room > g->rows_window_cap) room = g->rows_window_cap;
    if (!g->side) RTR_CUDA_TRY(cudaStreamCreateWithFlags(&g->side, cudaStreamNonBlocking));
    cudaEvent_t ready = nullptr, joined = nullptr;
    RTR_CUDA_TRY(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
    RTR_CUDA_TRY(cudaEventCreateWithFlags(&joined, cudaEventDisableTiming));
    float ms_fill = 0, ms_fold = 0, ms_warp = 0, ms_fill_l = 0, ms_fill_h = 0, ms_block = 0;
    // block folds: two per SM (kBlockFoldSmem of shared memory each)
    int hub_grid = 148;
    cudaDeviceGetAttribute(&hub_grid, cudaDevAttrMultiProcessorCount, g->device);
    hub_grid *= 2;
    if (nhuge > 0) RTR_CUDA_TRY(cudaFuncSetAttribute(k_vfold_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                     (int)kBlockFoldSmem));
    int rc = RTR_OK;
    g->rows_windows = 0;
    g->rows_entries = want;
    for (int64_t x0 = 0; x0 < n && rc == RTR_OK;) {
        ++g->rows_windows;
        int64_t x1 = n;
        if (want > room) {
            k_window_end<<<1, 1, 0, s>>>(g->offsets, lpos, n, x0, room, d_x1);
            g->launches += 1;
            if (cudaMemcpyAsync(&x1, d_x1, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                cudaStreamSynchronize(s) != cudaSuccess) {
                rc = cuda_fail(cudaGetLastError(), "rows-layout window", __FILE__, __LINE__);
                break;
            }
        }
        int64_t p01[2] = {0, 0}, e01[2] = {0, 0};
        if (cudaMemcpyAsync(&p01[0], g->offsets + x0, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&p01[1], g->offsets + x1, sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess ||
            cudaMemcpyAsync(&e01[0], lpos + p01[0], sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaMemcpyAsync(&e01[1], lpos + p01[1], sizeof(int64_t), cudaMemcpyDeviceToHost, s) != cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "rows-layout window", __FILE__, __LINE__);
            break;
        }
        if (e01[1] - e01[0] > room) {
            set_error("rows layout: vertex %lld alone has %lld perVertex terms, more than the %lld list entries "
                      "that fit in free device memory",
                      (long long)x0, (long long)(e01[1] - e01[0]), (long long)room);
            rc = RTR_ERR_LIMIT;
            break;
        }
        FillArgs fa{g->offsets, g->nbors, g->esrc, g->partner, g->deg, g->fwd, m, g->tune_edge, g->tune_gallop,
                    rs, lpos, p01[0], p01[1], e01[0], lists, moff, masks};
        ktime_begin(g, KT_TRI_FILL);
        ktime_begin(g, KT_FILL_LIGHT);
        k_fill_light<<<grid_for(m, kFillBlock), kFillBlock, 0, s>>>(fa);
        ktime_end(g, KT_FILL_LIGHT);
        ktime_begin(g, KT_FILL_HEAVY);
        k_fill_heavy<<<grid_for(1ll << 40, kHeavyBlock, 16), kHeavyBlock, 0, s>>>(fa, heavy_list, nheavy);
        ktime_end(g, KT_FILL_HEAVY);
        ktime_end(g, KT_TRI_FILL);
        FoldArgs fo{g->offsets, g->nbors, g->deg, lpos, e01[0], lists, g->pv, x0, x1, warp_min};
        cudaMemsetAsync(next, 0, 2 * sizeof(unsigned long long), s);
        ktime_begin(g, KT_VERTEX_FOLD);
        // block folds on the second stream, concurrent with the warp and thread folds
        cudaEventRecord(ready, s);
        cudaStreamWaitEvent(g->side, ready, 0);
        ktime_begin(g, KT_FOLD_BLOCK, g->side);
        if (nhuge > 0)
            k_vfold_block<<<(int)(nhuge < (unsigned)hub_grid ? nhuge : (unsigned)hub_grid), kFoldBlock,
                            kBlockFoldSmem, g->side>>>(fo, big, nhuge, segoff, segslot, next + 1);
        ktime_end(g, KT_FOLD_BLOCK, g->side);
        cudaEventRecord(joined, g->side);
        ktime_begin(g, KT_FOLD_WARP);
        if (nbig > nhuge)
            k_vfold_warp<<<grid_for(1ll << 40, kFoldBlock, 8), kFoldBlock, 0, s>>>(fo, big + nhuge, nbig - nhuge, next);
        ktime_end(g, KT_FOLD_WARP);
        k_vfold_thread<<<grid_for(x1 - x0, kFoldBlock), kFoldBlock, 0, s>>>(fo);
        cudaStreamWaitEvent(s, joined, 0);
        ktime_end(g, KT_VERTEX_FOLD);
        g->launches += 1 + (nbig > nhuge ? 1 : 0) + (nhuge > 0 ? 1 : 0) + 2;
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) {
            rc = cuda_fail(e, "rows-layout fill / fold launch", __FILE__, __LINE__);
            break;
        }
        if (cudaStreamSynchronize(s) != cudaSuccess) {
            rc = cuda_fail(cudaGetLastError(), "rows-layout fill / fold", __FILE__, __LINE__);
            break;
        }
        ktime_read(g, KT_TRI_FILL);
        ktime_read(g, KT_VERTEX_FOLD);
        ktime_read(g, KT_FOLD_WARP);
        ktime_read(g, KT_FOLD_BLOCK);
        ms_block += g->kms[KT_FOLD_BLOCK];
        ktime_read(g, KT_FILL_LIGHT);
        ktime_read(g, KT_FILL_HEAVY);
        ms_fill_l += g->kms[KT_FILL_LIGHT];
        ms_fill_h += g->kms[KT_FILL_HEAVY];
        ms_fill += g->kms[KT_TRI_FILL];
        ms_fold += g->kms[KT_VERTEX_FOLD];
        ms_warp += g->kms[KT_FOLD_WARP];
        x0 = x1;
    }
    cudaStreamSynchronize(g->side);  // scratch is freed on return
    cudaEventDestroy(ready);
    cudaEventDestroy(joined);
    g->kms[KT_TRI_FILL] = ms_fill;
    g->kms[KT_VERTEX_FOLD] = ms_fold;
    g->kms[KT_FOLD_WARP] = ms_warp;
    g->kms[KT_FILL_LIGHT] = ms_fill_l;
    g->kms[KT_FILL_HEAVY] = ms_fill_h;
    g->kms[KT_FOLD_BLOCK] = ms_block;
    return rc;
}

}  // namespace rtr
