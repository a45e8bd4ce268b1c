// Connected components in the reference's BFS discovery order
// (connectedComp, RTRex_Sequential/Escape/Decomposition.h:1023-1068).
//
// The reference starts a BFS at every still-unvisited vertex in id order and
// inserts vertices into the component's set in the order its FIFO queue
// discovers them: a vertex is discovered by the earliest-dequeued vertex that
// has it as a neighbour, at that vertex's row position.  The device runs all
// components' BFS together, level by level:
//   * the frontier array is component-major and in discovery order;
//   * every frontier vertex offers key (frontier index, row position) to each
//     unvisited neighbour and the neighbour keeps the minimum (atomicMin);
//   * a frontier row's winning slots, taken in row order and frontier order,
//     are exactly the next level's discoveries in sequential BFS order, so the
//     next frontier is built by count / scan / write with no sort.
// Components come out in creation order (ascending minimum vertex id, which is
// where the reference's BFS starts, since the union-find roots are minima).
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>
#include <vector>

namespace rtr {

namespace {

constexpr int kBlock = 256;

__device__ __forceinline__ int32_t cc_find(int32_t* p, int32_t x)
{
    while (true) {
        const int32_t px = p[x];
        if (px == x) return x;
        const int32_t ppx = p[px];
        if (ppx != px) atomicCAS(&p[x], px, ppx);
        x = px;
    }
}

__global__ void k_cc_init(int32_t* __restrict__ p, unsigned long long* __restrict__ key, uint8_t* __restrict__ vis,
                          int64_t n)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        p[v] = (int32_t)v;
        key[v] = ~0ull;
        vis[v] = 0;
    }
}

__global__ void k_cc_hook(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb,
                          const int32_t* __restrict__ fwd, int64_t m, int32_t* __restrict__ p)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < m; k += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = fwd[k];
        int32_t a = esrc[i], b = nb[i];
        while (true) {
            a = cc_find(p, a);
            b = cc_find(p, b);
            if (a == b) break;
            if (a > b) {
                const int32_t t = a;
                a = b;
                b = t;
            }
            const int32_t old = atomicCAS(&p[b], b, a);
            if (old == b) break;
            b = old;
        }
    }
}

__global__ void k_cc_flatten(int32_t* __restrict__ p, int64_t n, uint32_t* __restrict__ is_root)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        const int32_t r = cc_find(p, (int32_t)v);
        p[v] = r;
        is_root[v] = r == v ? 1u : 0u;
    }
}

// Level 0: the roots, ascending (component creation order).
__global__ void k_cc_roots(const uint32_t* __restrict__ is_root, const uint32_t* __restrict__ pos, int64_t n,
                           int32_t* __restrict__ frontier, uint8_t* __restrict__ vis, int64_t* __restrict__ seq)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        if (is_root[v]) {
            frontier[pos[v]] = (int32_t)v;
            vis[v] = 1;
            seq[v] = pos[v];
        }
}

__global__ void k_cc_offer(const int32_t* __restrict__ frontier, int64_t nf, const int64_t* __restrict__ off,
                           const int32_t* __restrict__ nb, const uint8_t* __restrict__ vis,
                           unsigned long long* __restrict__ key)
{
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = frontier[f];
        const int64_t r0 = off[x];
        for (int64_t j = r0; j < off[x + 1]; ++j) {
            const int32_t y = nb[j];
            if (!vis[y]) atomicMin(&key[y], ((unsigned long long)f << 32) | (unsigned long long)(j - r0));
        }
    }
}

__device__ __forceinline__ bool cc_won(const int32_t* nb, const uint8_t* vis, const unsigned long long* key, int64_t f,
                                       int64_t r0, int64_t j)
{
    const int32_t y = nb[j];
    return !vis[y] && key[y] == (((unsigned long long)f << 32) | (unsigned long long)(j - r0));
}

__global__ void k_cc_count(const int32_t* __restrict__ frontier, int64_t nf, const int64_t* __restrict__ off,
                           const int32_t* __restrict__ nb, const uint8_t* __restrict__ vis,
                           const unsigned long long* __restrict__ key, uint32_t* __restrict__ cnt)
{
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = frontier[f];
        const int64_t r0 = off[x];
        uint32_t c = 0;
        for (int64_t j = r0; j < off[x + 1]; ++j) c += cc_won(nb, vis, key, f, r0, j) ? 1u : 0u;
        cnt[f] = c;
    }
}

__global__ void k_cc_write(const int32_t* __restrict__ frontier, int64_t nf, const int64_t* __restrict__ off,
                           const int32_t* __restrict__ nb, const uint8_t* __restrict__ vis,
                           const unsigned long long* __restrict__ key, const uint32_t* __restrict__ base,
                           int32_t* __restrict__ next)
{
    for (int64_t f = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; f < nf; f += (int64_t)gridDim.x * blockDim.x) {
        const int32_t x = frontier[f];
        const int64_t r0 = off[x];
        uint32_t w = base[f];
        for (int64_t j = r0; j < off[x + 1]; ++j)
            if (cc_won(nb, vis, key, f, r0, j)) next[w++] = nb[j];
    }
}

// Mark the new frontier visited and give it its global discovery numbers.
__global__ void k_cc_visit(const int32_t* __restrict__ next, int64_t nn, int64_t seq0, uint8_t* __restrict__ vis,
                           int64_t* __restrict__ seq)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < nn; i += (int64_t)gridDim.x * blockDim.x) {
        vis[next[i]] = 1;
        seq[next[i]] = seq0 + i;
    }
}

__global__ void k_cc_keys(const int32_t* __restrict__ root, const int64_t* __restrict__ seq, int64_t n, int B,
                          uint64_t* __restrict__ keys)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        keys[v] = ((uint64_t)root[v] << B) | (uint64_t)seq[v];
}

__global__ void k_cc_unpack(const uint64_t* __restrict__ sorted, int64_t n, int B, const int32_t* __restrict__ by_seq,
                            int32_t* __restrict__ out, uint32_t* __restrict__ head)
{
    const uint64_t mask = (1ull << B) - 1;
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x) {
        out[j] = by_seq[sorted[j] & mask];
        head[j] = (j == 0 || (sorted[j] >> B) != (sorted[j - 1] >> B)) ? 1u : 0u;
    }
}

__global__ void k_cc_by_seq(const int64_t* __restrict__ seq, int64_t n, int32_t* __restrict__ by_seq)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        by_seq[seq[v]] = (int32_t)v;
}

__global__ void k_cc_offsets(const uint32_t* __restrict__ head, const uint32_t* __restrict__ hpos, int64_t n,
                             int64_t* __restrict__ comp_off)
{
    for (int64_t j = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; j < n; j += (int64_t)gridDim.x * blockDim.x)
        if (head[j]) comp_off[hpos[j]] = j;
}

}  // namespace

int connected_components(rtr_graph* g)
{
    if (g->stage < 1) {
        set_error("components requested before the graph was built");
        return RTR_ERR_STATE;
    }
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m = g->m;
    const int gn = grid_for(n, kBlock), gm = grid_for(m, kBlock);
    Scratch sc(g);
    int32_t* root = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    unsigned long long* key = (unsigned long long*)sc.get(sizeof(unsigned long long) * (n + 1));
    uint8_t* vis = (uint8_t*)sc.get(n + 16);
    uint32_t* is_root = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* pos = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* tmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(n + 1));
    uint32_t* d_cnt = (uint32_t*)sc.get(sizeof(uint32_t) * 2);
    int32_t* fa = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    int32_t* fb = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    uint32_t* cnt = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    uint32_t* base = (uint32_t*)sc.get(sizeof(uint32_t) * (n + 1));
    int64_t* seq = (int64_t*)sc.get(sizeof(int64_t) * (n + 1));
    if (!root || !key || !vis || !is_root || !pos || !tmp || !d_cnt || !fa || !fb || !cnt || !base || !seq) {
        set_error("device allocation failed (components)");
        return RTR_ERR_CUDA;
    }
    k_cc_init<<<gn, kBlock, 0, s>>>(root, key, vis, n);
    k_cc_hook<<<gm, kBlock, 0, s>>>(g->esrc, g->nbors, g->fwd, m, root);
    k_cc_flatten<<<gn, kBlock, 0, s>>>(root, n, is_root);
    exclusive_scan_u32(is_root, pos, n, d_cnt, tmp, s);
    k_cc_roots<<<gn, kBlock, 0, s>>>(is_root, pos, n, fa, vis, seq);
    g->launches += 7;
    uint32_t ncomp = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&ncomp, d_cnt, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    int64_t nf = ncomp, seq0 = ncomp;
    int32_t* cur = fa;
    int32_t* nxt = fb;
    while (nf > 0) {
        const int gf = grid_for(nf, kBlock);
        k_cc_offer<<<gf, kBlock, 0, s>>>(cur, nf, g->offsets, g->nbors, vis, key);
        k_cc_count<<<gf, kBlock, 0, s>>>(cur, nf, g->offsets, g->nbors, vis, key, cnt);
        exclusive_scan_u32(cnt, base, nf, d_cnt + 1, tmp, s);
        k_cc_write<<<gf, kBlock, 0, s>>>(cur, nf, g->offsets, g->nbors, vis, key, base, nxt);
        g->launches += 6;
        uint32_t nn = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&nn, d_cnt + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        if (nn > 0) {
            k_cc_visit<<<grid_for(nn, kBlock), kBlock, 0, s>>>(nxt, nn, seq0, vis, seq);
            g->launches += 1;
        }
        seq0 += nn;
        nf = nn;
        std::swap(cur, nxt);
    }
    if (seq0 != n) {
        set_error("component search reached %lld of %lld vertices", (long long)seq0, (long long)n);
        return RTR_ERR_DEVICE;
    }
    // group by component (creation order), discovery order inside
    const int B = bits_for((uint64_t)(n - 1));
    uint64_t* k1 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    uint64_t* k2 = (uint64_t*)sc.get(sizeof(uint64_t) * (n + 1));
    void* rtmp = sc.get(radix_temp_bytes(n));
    int32_t* by_seq = (int32_t*)sc.get(sizeof(int32_t) * (n + 1));
    if (!k1 || !k2 || !rtmp || !by_seq) {
        set_error("device allocation failed (components order)");
        return RTR_ERR_CUDA;
    }
    if (!g->cc_vert) {
        g->cc_vert = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
        g->cc_off = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 2));
        if (!g->cc_vert || !g->cc_off) {
            set_error("device allocation failed (components output)");
            return RTR_ERR_CUDA;
        }
    }
    k_cc_keys<<<gn, kBlock, 0, s>>>(root, seq, n, B, k1);
    k_cc_by_seq<<<gn, kBlock, 0, s>>>(seq, n, by_seq);
    uint64_t* sorted = radix_sort_u64(k1, k2, n, 2 * B, rtmp, s);
    k_cc_unpack<<<gn, kBlock, 0, s>>>(sorted, n, B, by_seq, g->cc_vert, is_root);
    exclusive_scan_u32(is_root, pos, n, nullptr, tmp, s);
    k_cc_offsets<<<gn, kBlock, 0, s>>>(is_root, pos, n, g->cc_off);
    RTR_CUDA_TRY(cudaMemcpyAsync(g->cc_off + ncomp, &n, sizeof(int64_t), cudaMemcpyHostToDevice, s));
    g->launches += 7 + 3 * ((2 * B + 7) / 8);
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    g->ncc = ncomp;
    return RTR_OK;
}

}  // namespace rtr
