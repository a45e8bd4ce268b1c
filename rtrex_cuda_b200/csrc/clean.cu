// Cascading clean, order-faithful to initialClean + deleteAndClean
// (RTRex_Sequential/Escape/Decomposition.h:302-460 and :147-283).
//
// The reference seeds every u<v edge below eps * 1/(du*dv) in slot order onto a
// LIFO stack and then pops: a popped edge removes each of its live triangles
// (no 'N' edge), subtracting the triangle weight from the two other edges and
// the three vertices, and pushes the other edges that fall below threshold.
// Floating-point sums make the survivor set depend on that exact order (a
// bulk-synchronous peel differs on the bundled email / astro graphs), so the
// device replays the same order -- but only where order can matter:
//
//  * a seed with no triangles is a no-op pop: it is marked 'N' directly;
//  * edges with triangles split into vertex-disjoint units (connected
//    components of the graph of triangle-carrying edges, by union-find with
//    hooking to the smaller root).  Every cell a pop touches (the popped edge,
//    the two other edges of each triangle, the three vertices) lies in the
//    popped edge's unit, and a cascade never leaves its unit, so each unit can
//    replay its own seeds (in slot order, popped last-first) and cascades
//    independently and still perform the reference's operations, in the
//    reference's order, on every cell;
//  * one warp replays one unit: per popped edge the lanes take 32 triangles of
//    the edge's triangle list at a time, update the distinct per-triangle
//    cells in parallel, fold the shared cells (the popped edge, its two
//    endpoints) in triangle order, and append pushes in the reference's push
//    order (triangle order, (lower,w) before (higher,w)).
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>
#include <vector>

namespace rtr {

namespace {

constexpr int kBlock = 256;

__global__ void k_seed(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                       const int32_t* __restrict__ deg, const int32_t* __restrict__ fwd, int64_t m, double eps,
                       const double* __restrict__ pe, const uint32_t* __restrict__ sup, uint8_t* __restrict__ st,
                       uint32_t* __restrict__ is_seed)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        const int64_t du = deg[esrc[i]], dv = deg[nb[i]];
        const double ew = 1 / (double)(du * dv);
        const bool below = pe[i] < eps * ew;
        uint8_t s = ST_Y;
        uint32_t seed = 0;
        if (below) {
            if (sup[i] > 0) {
                s = ST_S;
                seed = 1;
            } else {
                s = ST_N;  // a pop with no triangle changes nothing but its own status
            }
        }
        st[i] = s;
        is_seed[k] = seed;
    }
}

__device__ __forceinline__ int32_t uf_find(int32_t* p, int32_t x)
{
    while (true) {
        const int32_t px = p[x];
        if (px == x) return x;
        const int32_t ppx = p[px];
        if (ppx != px) atomicCAS(&p[x], px, ppx);
        x = px;
    }
}

__device__ __forceinline__ void uf_unite(int32_t* p, int32_t a, int32_t b)
{
    while (true) {
        a = uf_find(p, a);
        b = uf_find(p, b);
        if (a == b) return;
        if (a > b) {
            const int32_t t = a;
            a = b;
            b = t;
        }
        // hook the larger root under the smaller: the final root is the minimum id
        const int32_t old = atomicCAS(&p[b], b, a);
        if (old == b) return;
        b = old;
    }
}

__global__ void k_uf_init(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = (int32_t)v;
}

__global__ void k_uf_hook_support(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                                  const int32_t* __restrict__ fwd, int64_t m, const uint32_t* __restrict__ sup,
                                  int32_t* __restrict__ p)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (sup[i] > 0) uf_unite(p, esrc[i], nb[i]);
    }
}

__global__ void k_uf_flatten(int32_t* __restrict__ p, int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        p[v] = uf_find(p, (int32_t)v);
}

// Per-unit capacity of the cascade stack: the unit's triangle-carrying edges.
__global__ void k_unit_edges(const int32_t* __restrict__ esrc, const int32_t* __restrict__ fwd, int64_t m,
                             const uint32_t* __restrict__ sup, const int32_t* __restrict__ root,
                             uint32_t* __restrict__ ecount)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        if (sup[i] > 0) atomicAdd(&ecount[root[esrc[i]]], 1u);
    }
}

__global__ void k_seed_keys(const int32_t* __restrict__ fwd, const int32_t* __restrict__ esrc,
                            const uint32_t* __restrict__ is_seed, const uint32_t* __restrict__ pos, int64_t m,
                            const int32_t* __restrict__ root, int sbits, uint64_t* __restrict__ keys)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x)
        if (is_seed[k]) {
            const int64_t i = fwd[k];
            keys[pos[k]] = ((uint64_t)root[esrc[i]] << sbits) | (uint64_t)i;
        }
}

__global__ void k_unit_heads(const uint64_t* __restrict__ keys, int64_t ns, int sbits, uint32_t* __restrict__ head)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x)
        head[j] = (j == 0 || (keys[j] >> sbits) != (keys[j - 1] >> sbits)) ? 1u : 0u;
}

struct UnitDesc {
    int64_t seed_begin;
    int64_t seed_end;
    int64_t stack_base;
    int64_t stack_cap;
};

__global__ void k_unit_desc(const uint64_t* __restrict__ keys, int64_t ns, int sbits,
                            const uint32_t* __restrict__ head, const uint32_t* __restrict__ hpos,
                            const uint32_t* __restrict__ ecount, UnitDesc* __restrict__ units,
                            int64_t* __restrict__ cap)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < ns; j += (int64_t)gridDim.x * blockDim.x) {
        if (!head[j]) continue;
        const uint32_t u = hpos[j];
        units[u].seed_begin = j;
        const uint32_t r = (uint32_t)(keys[j] >> sbits);
        cap[u] = ecount[r];
    }
}

__global__ void k_unit_finish(UnitDesc* __restrict__ units, const int64_t* __restrict__ cap,
                              const int64_t* __restrict__ capoff, int64_t nu, int64_t ns,
                              uint64_t* __restrict__ order_keys)
{
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < nu; u += (int64_t)gridDim.x * blockDim.x) {
        units[u].seed_end = (u + 1 < nu) ? units[u + 1].seed_begin : ns;
        units[u].stack_base = capoff[u];
        units[u].stack_cap = cap[u];
        // schedule units with the most seeds first
        const uint64_t work = (uint64_t)(units[u].seed_end - units[u].seed_begin);
        order_keys[u] = ((uint64_t)(0xffffffffu - (uint32_t)(work < 0xffffffffull ? work : 0xffffffffull)) << 32) | (uint64_t)u;
    }
}

struct StackEntry {
    int32_t e;      // forward slot of the edge
    int32_t first;  // Pair.first  (deleteAndClean's u)
    int32_t second; // Pair.second (deleteAndClean's v)
    int32_t pad;
};

struct CleanArgs {
    const int64_t* off;
    const int32_t* nb;
    const int32_t* esrc;
    const int32_t* deg;
    const int64_t* tl_off;
    const TriEntry* tl;
    double* pe;
    double* pv;
    uint32_t* sup;
    uint8_t* st;
    double eps;
    double inv_n;
};

// Pop one edge: deleteAndClean's loop body (Decomposition.h:152-281) for the
// whole warp.  Returns the number of triangles removed.
__device__ __forceinline__ int pop_edge(const CleanArgs& a, int32_t e, int32_t u, int32_t v, StackEntry* stack,
                                        int64_t& top, int64_t cap, unsigned* err, unsigned long long* diag)
{
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t s_e = a.sup[e];
    if (s_e == 0) {
        __syncwarp();
        if (lane == 0) {
            if (fabs(a.pe[e]) > a.inv_n) atomicAdd(&diag[0], 1ull);
            a.st[e] = ST_N;
        }
        __syncwarp();
        return 0;
    }
    const int64_t du = a.deg[u], dv = a.deg[v];
    const bool lo_is_u = du < dv;
    const int32_t lower = lo_is_u ? u : v;
    const int32_t higher = lo_is_u ? v : u;
    const int64_t dlow = lo_is_u ? du : dv;
    const int64_t dhigh = lo_is_u ? dv : du;
    const bool lower_is_a = lower == a.esrc[e];  // a = smaller endpoint of the forward slot
    const int64_t t0 = a.tl_off[e], t1 = a.tl_off[e + 1];
    double acc_e = a.pe[e], acc_u = a.pv[u], acc_v = a.pv[v];
    const int64_t duv = du * dv;
    int removed = 0;
    for (int64_t base = t0; base < t1; base += 32) {
        const int64_t idx = base + lane;
        const bool valid = idx < t1;
        TriEntry t = {0, 0, 0, 1};
        if (valid) t = a.tl[idx];
        const int32_t elw = lower_is_a ? t.eaz : t.ebz;
        const int32_t ehw = lower_is_a ? t.ebz : t.eaz;
        uint8_t slw = ST_N, shw = ST_N;
        if (valid) {
            slw = a.st[elw];
            shw = a.st[ehw];
        }
        const bool live = valid && slw != ST_N && shw != ST_N;
        double wgt = 0.0;
        bool p1 = false, p2 = false;
        if (live) {
            wgt = 1 / (double)(duv * (int64_t)t.dz);
            const double x1 = a.pe[elw] - wgt;
            const double x2 = a.pe[ehw] - wgt;
            a.pe[elw] = x1;
            a.pe[ehw] = x2;
            a.sup[elw] -= 1u;
            a.sup[ehw] -= 1u;
            a.pv[t.z] -= wgt;
            p1 = slw != ST_S && x1 < a.eps * (1 / (double)(dlow * (int64_t)t.dz));
            p2 = shw != ST_S && x2 < a.eps * (1 / (double)(dhigh * (int64_t)t.dz));
            if (p1) a.st[elw] = ST_S;
            if (p2) a.st[ehw] = ST_S;
        }
        const unsigned lm = __ballot_sync(0xffffffffu, live);
        const unsigned b1 = __ballot_sync(0xffffffffu, p1);
        const unsigned b2 = __ballot_sync(0xffffffffu, p2);
        // the popped edge and its endpoints accumulate in triangle order
        for (unsigned mm = lm; mm; mm &= mm - 1) {
            const double w = __shfl_sync(0xffffffffu, wgt, __ffs(mm) - 1);
            acc_e -= w;
            acc_u -= w;
            acc_v -= w;
        }
        const int np = __popc(b1) + __popc(b2);
        if (top + np > cap) {
            if (lane == 0) atomicOr(err, (unsigned)DEV_ERR_STACK_OVERFLOW);
            return -1;
        }
        const int before = __popc(b1 & lt) + __popc(b2 & lt);
        if (p1) stack[top + before] = StackEntry{elw, lower, t.z, 0};
        if (p2) stack[top + before + (p1 ? 1 : 0)] = StackEntry{ehw, higher, t.z, 0};
        top += np;
        removed += __popc(lm);
    }
    __syncwarp();
    if (lane == 0) {
        a.pe[e] = acc_e;
        a.pv[u] = acc_u;
        a.pv[v] = acc_v;
        a.sup[e] = s_e - (uint32_t)removed;
        if (fabs(acc_e) > a.inv_n) atomicAdd(&diag[0], 1ull);
        a.st[e] = ST_N;
    }
    __syncwarp();
    return removed;
}

__global__ void __launch_bounds__(kBlock)
    k_clean_units(CleanArgs a, const uint64_t* __restrict__ seed_keys, uint64_t slot_mask,
                  const UnitDesc* __restrict__ units, const uint64_t* __restrict__ order, int64_t nu,
                  StackEntry* __restrict__ stacks, unsigned* __restrict__ next_unit, unsigned* __restrict__ err,
                  unsigned long long* __restrict__ total, unsigned long long* __restrict__ diag)
{
    const int lane = threadIdx.x & 31;
    while (true) {
        unsigned ui = 0;
        if (lane == 0) ui = atomicAdd(next_unit, 1u);
        ui = __shfl_sync(0xffffffffu, ui, 0);
        if ((int64_t)ui >= nu) break;
        const UnitDesc ud = units[(uint32_t)order[ui]];
        StackEntry* stack = stacks + ud.stack_base;
        int64_t top = 0;
        int64_t sp = ud.seed_end;
        unsigned long long removed = 0;
        while (true) {
            int32_t e, u, v;
            if (top > 0) {
                --top;
                const StackEntry se = stack[top];
                e = se.e;
                u = se.first;
                v = se.second;
            } else if (sp > ud.seed_begin) {
                --sp;
                e = (int32_t)(seed_keys[sp] & slot_mask);
                u = a.esrc[e];  // seeds are pushed as (u, v) with u < v
                v = a.nb[e];
            } else {
                break;
            }
            const int r = pop_edge(a, e, u, v, stack, top, ud.stack_cap, err, diag);
            if (r < 0) break;
            removed += (unsigned long long)r;
        }
        if (lane == 0 && removed) atomicAdd(total, (unsigned long long)(-(long long)removed));
    }
}

}  // namespace

int initial_clean(rtr_graph* g, double eps)
{
    if (g->stage < 2) {
        set_error("clean called before count");
        return RTR_ERR_STATE;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m = g->m, m2 = g->m2;
    g->eps = eps;
    Scratch sc(g);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);

    uint32_t* is_seed = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    uint32_t* spos = (uint32_t*)sc.get(sizeof(uint32_t) * (m + 1));
    uint32_t* stmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(m + 1));
    uint32_t* d_ns = (uint32_t*)sc.get(sizeof(uint32_t) * 2);
    int32_t* root = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    uint32_t* ecount = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    if (!is_seed || !spos || !stmp || !d_ns || !root || !ecount) {
        set_error("device allocation failed (clean)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr + 1, 0, 2 * sizeof(unsigned long long), s));
    RTR_CUDA_TRY(cudaMemsetAsync(g->st, ST_N, m2 + 16, s));  // backward slots are never read
    const int gm = grid_for(m, kBlock), gn = grid_for(n, kBlock);
    k_seed<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->deg, g->fwd, m, eps, g->pe, g->sup, g->st, is_seed);
    k_uf_init<<<gn, kBlock, 0, s>>>(root, n);
    k_uf_hook_support<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->fwd, m, g->sup, root);
    k_uf_flatten<<<gn, kBlock, 0, s>>>(root, n);
    RTR_CUDA_TRY(cudaMemsetAsync(ecount, 0, sizeof(uint32_t) * (n + 1), s));
    k_unit_edges<<<gm, kBlock, 0, s>>>(g->esrc, g->fwd, m, g->sup, root, ecount);
    exclusive_scan_u32(is_seed, spos, m, d_ns, stmp, s);
    g->launches += 8;
    RTR_CUDA_TRY(cudaGetLastError());
    uint32_t ns = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&ns, d_ns, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->kms[KT_CLEAN_UNITS] = 0;
    // an empty timer pair keeps the reading defined when no unit exists
    ktime_begin(g, KT_CLEAN_UNITS);
    ktime_end(g, KT_CLEAN_UNITS);

    if (ns > 0) {
        const int sbits = bits_for((uint64_t)m2);
        uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * (ns + 1));
        uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * (ns + 1));
        void* rtmp = sc.get(radix_temp_bytes(ns));
        uint32_t* head = (uint32_t*)sc.get(sizeof(uint32_t) * (ns + 1));
        uint32_t* hpos = (uint32_t*)sc.get(sizeof(uint32_t) * (ns + 1));
        uint32_t* htmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(ns + 1));
        if (!keys || !alt || !rtmp || !head || !hpos || !htmp) {
            set_error("device allocation failed (clean seeds)");
            return RTR_ERR_CUDA;
        }
        k_seed_keys<<<gm, kBlock, 0, s>>>(g->fwd, g->esrc, is_seed, spos, m, root, sbits, keys);
        uint64_t* sorted = radix_sort_u64(keys, alt, ns, sbits + bits_for((uint64_t)n), rtmp, s);
        const int gs = grid_for(ns, kBlock);
        k_unit_heads<<<gs, kBlock, 0, s>>>(sorted, ns, sbits, head);
        exclusive_scan_u32(head, hpos, ns, d_ns + 1, htmp, s);
        g->launches += 3 + 3 * ((sbits + bits_for((uint64_t)n) + 7) / 8);
        uint32_t nu = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nu, d_ns + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        UnitDesc* units = (UnitDesc*)sc.get(sizeof(UnitDesc) * (nu + 1));
        int64_t* cap = (int64_t*)sc.get(sizeof(int64_t) * (nu + 1));
        int64_t* capoff = (int64_t*)sc.get(sizeof(int64_t) * (nu + 1));
        int64_t* ctmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(nu + 1));
        int64_t* d_cap_total = (int64_t*)sc.get(sizeof(int64_t));
        uint64_t* okeys = (uint64_t*)sc.get(sizeof(uint64_t) * (nu + 1));
        uint64_t* oalt = (uint64_t*)sc.get(sizeof(uint64_t) * (nu + 1));
        void* otmp = sc.get(radix_temp_bytes(nu));
        unsigned* next_unit = (unsigned*)sc.get(sizeof(unsigned) * 2);
        if (!units || !cap || !capoff || !ctmp || !d_cap_total || !okeys || !oalt || !otmp || !next_unit) {
            set_error("device allocation failed (clean units)");
            return RTR_ERR_CUDA;
        }
        k_unit_desc<<<gs, kBlock, 0, s>>>(sorted, ns, sbits, head, hpos, ecount, units, cap);
        exclusive_scan_i64(cap, capoff, nu, d_cap_total, ctmp, s);
        k_unit_finish<<<grid_for(nu, kBlock), kBlock, 0, s>>>(units, cap, capoff, nu, ns, okeys);
        uint64_t* order = radix_sort_u64(okeys, oalt, nu, 64, otmp, s);
        g->launches += 5 + 24;
        int64_t cap_total = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&cap_total, d_cap_total, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaMemsetAsync(next_unit, 0, sizeof(unsigned) * 2, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        StackEntry* stacks = (StackEntry*)sc.get(sizeof(StackEntry) * (cap_total + 1));
        if (!stacks) {
            set_error("device allocation failed (clean stacks)");
            return RTR_ERR_CUDA;
        }
        CleanArgs ca{g->offsets, g->nbors, g->esrc, g->deg, g->tl_off, g->tl, g->pe, g->pv, g->sup, g->st, eps,
                     1 / (double)n};
        const uint64_t slot_mask = (1ull << sbits) - 1;
        // one warp per unit, persistent over the unit list
        const int warps_per_block = kBlock / 32;
        int blocks = (int)std::min<int64_t>((nu + warps_per_block - 1) / warps_per_block,
                                            (int64_t)grid_for(1 << 30, kBlock, 8));
        blocks = std::max(blocks, 1);
        ktime_begin(g, KT_CLEAN_UNITS);
        k_clean_units<<<blocks, kBlock, 0, s>>>(ca, sorted, slot_mask, units, order, nu, stacks, next_unit,
                                                (unsigned*)(g->ctr + 1), g->ctr, g->ctr + 2);
        ktime_end(g, KT_CLEAN_UNITS);
        g->launches += 1;
        RTR_CUDA_TRY(cudaGetLastError());
    }
    cudaEventRecord(e1, s);
    RTR_CUDA_TRY(cudaEventSynchronize(e1));
    cudaEventElapsedTime(&g->ms_clean, e0, e1);
    if (g->kms[KT_CLEAN_UNITS] >= 0) ktime_read(g, KT_CLEAN_UNITS);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    unsigned long long h[3];
    RTR_CUDA_TRY(cudaMemcpy(h, g->ctr, sizeof h, cudaMemcpyDeviceToHost));
    if (h[1] != 0) {
        set_error("device error word 0x%llx during the clean", h[1]);
        return RTR_ERR_DEVICE;
    }
    g->diag_residual = (long long)h[2];
    g->stage = 3;
    return RTR_OK;
}

}  // namespace rtr
