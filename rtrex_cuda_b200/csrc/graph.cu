// CSR construction on the device (the reference builds it on the host:
// loadGraph_Escape stores both directions, RTRex_Sequential/GraphIO.cpp:42-63;
// makeCSR sorts the pairs and compresses sources, Graph.cpp:344-384; the CUDA
// port uploads that host CSR and binary-searches partners, gpu_graph.cu:8-92).
//
// Here: the undirected pairs are expanded to 2m packed keys (src << B | dst),
// radix-sorted on the device, checked for self-loops / duplicates, unpacked to
// int32 neighbour ids + source ids, compressed into int64 offsets, and every
// slot gets its reverse-copy index by a binary search in the neighbour's row.
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

namespace rtr {

namespace {
thread_local std::string t_last_error;
}

void set_error(const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    t_last_error = buf;
}

const char* last_error() { return t_last_error.c_str(); }

int cuda_fail(cudaError_t e, const char* what, const char* file, int line)
{
    set_error("CUDA error %s (%s) at %s:%d: %s", cudaGetErrorName(e), cudaGetErrorString(e), file, line, what);
    return RTR_ERR_CUDA;
}

void* dev_alloc(rtr_graph* g, size_t bytes)
{
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, g->stream) != cudaSuccess) return nullptr;
    g->owned.push_back(p);
    g->owned_bytes += (int64_t)bytes;
    return p;
}

void dev_free_all(rtr_graph* g)
{
    for (void* p : g->owned) cudaFreeAsync(p, g->stream);
    g->owned.clear();
    g->owned_bytes = 0;
}

void* Scratch::get(size_t bytes)
{
    void* p = nullptr;
    if (bytes == 0) bytes = 16;
    if (cudaMallocAsync(&p, bytes, g->stream) != cudaSuccess) return nullptr;
    ptrs.push_back(p);
    this->bytes += (int64_t)bytes;
    g->scratch_bytes += (int64_t)bytes;
    if (g->scratch_bytes > g->scratch_peak) g->scratch_peak = g->scratch_bytes;
    return p;
}

Scratch::~Scratch()
{
    for (void* p : ptrs) cudaFreeAsync(p, g->stream);
    g->scratch_bytes -= bytes;
}

// Free device memory.  The device pool keeps freed blocks cached (its release
// threshold is unbounded), and cudaMemGetInfo counts them as used; with trim the
// pool first returns the blocks no allocation holds, so the figure is what a
// large allocation can get.
size_t device_avail_bytes(rtr_graph* g)
{
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    cudaMemPool_t pool;
    uint64_t reserved = 0, used = 0;
    if (cudaDeviceGetDefaultMemPool(&pool, g->device) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) == cudaSuccess &&
        cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) == cudaSuccess && reserved > used)
        free_b += (size_t)(reserved - used);
    return free_b;
}

void release_owned(rtr_graph* g, void** buf, int64_t* cap)
{
    if (!*buf) return;
    for (size_t k = 0; k < g->owned.size(); ++k)
        if (g->owned[k] == *buf) {
            g->owned.erase(g->owned.begin() + (long)k);
            break;
        }
    cudaFreeAsync(*buf, g->stream);
    g->owned_bytes -= *cap;
    *buf = nullptr;
    *cap = 0;
}

void* grow_owned(rtr_graph* g, void** buf, int64_t* cap, int64_t bytes)
{
    if (*cap >= bytes && *buf) return *buf;
    release_owned(g, buf, cap);
    *buf = dev_alloc(g, (size_t)bytes);  // from the pool's cached blocks when they can serve it
    if (!*buf) {
        cudaGetLastError();          // the failed attempt's error is not the caller's
        free_device_bytes(g, true);  // return the cached blocks, then map fresh memory
        *buf = dev_alloc(g, (size_t)bytes);
    }
    if (*buf) *cap = bytes;
    return *buf;
}

size_t free_device_bytes(rtr_graph* g, bool trim)
{
    if (trim) {
        cudaStreamSynchronize(g->stream);
        if (g->side) cudaStreamSynchronize(g->side);
        cudaMemPool_t pool;
        if (cudaDeviceGetDefaultMemPool(&pool, g->device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
    }
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) return 0;
    return free_b;
}

namespace {

constexpr int kBlock = 256;

__global__ void k_make_keys(const int64_t* __restrict__ u, const int64_t* __restrict__ v, int64_t m, int64_t n,
                            int B, uint64_t* __restrict__ keys, unsigned long long* __restrict__ bad)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t a = u[i], b = v[i];
        if (a < 0 || b < 0 || a >= n || b >= n) {
            atomicAdd(bad, 1ull);
            keys[2 * i] = 0;
            keys[2 * i + 1] = 0;
            continue;
        }
        keys[2 * i] = ((uint64_t)a << B) | (uint64_t)b;
        keys[2 * i + 1] = ((uint64_t)b << B) | (uint64_t)a;
    }
}

// keep[i] = 0 for a self-loop or a repeat of the previous key.
__global__ void k_flag_keys(const uint64_t* __restrict__ keys, int64_t m2, int B, uint32_t* __restrict__ keep,
                            unsigned long long* __restrict__ nloops, unsigned long long* __restrict__ ndups)
{
    const uint64_t mask = (B == 64) ? ~0ull : ((1ull << B) - 1);
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        const bool loop = (k >> B) == (k & mask);
        const bool dup = i > 0 && keys[i - 1] == k;
        if (loop) atomicAdd(nloops, 1ull);
        else if (dup) atomicAdd(ndups, 1ull);
        keep[i] = (loop || dup) ? 0u : 1u;
    }
}

__global__ void k_compact_keys(const uint64_t* __restrict__ keys, const uint32_t* __restrict__ keep,
                               const uint32_t* __restrict__ pos, int64_t m2, uint64_t* __restrict__ out)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x)
        if (keep[i]) out[pos[i]] = keys[i];
}

__global__ void k_unpack(const uint64_t* __restrict__ keys, int64_t m2, int B, int32_t* __restrict__ nbors,
                         int32_t* __restrict__ esrc)
{
    const uint64_t mask = (1ull << B) - 1;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys[i];
        nbors[i] = (int32_t)(k & mask);
        esrc[i] = (int32_t)(k >> B);
    }
}

// offsets[w] = first slot whose source is >= w.
__global__ void k_offsets(const int32_t* __restrict__ esrc, int64_t m2, int64_t n, int64_t* __restrict__ off)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= m2; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t cur = (i < m2) ? esrc[i] : n;
        const int64_t prev = (i > 0) ? esrc[i - 1] : -1;
        for (int64_t w = prev + 1; w <= cur; ++w) off[w] = i;
    }
}

__global__ void k_degree(const int64_t* __restrict__ off, int64_t n, int32_t* __restrict__ deg)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        deg[v] = (int32_t)(off[v + 1] - off[v]);
}

// Row lookup of v2 in v1's sorted list: CGraph::getEdgeBinary (Graph.cpp:130-149).
__device__ __forceinline__ int64_t find_slot(const int64_t* __restrict__ off, const int32_t* __restrict__ nb,
                                             int64_t v1, int32_t v2)
{
    int64_t lo = off[v1], hi = off[v1 + 1] - 1;
    while (lo <= hi) {
        const int64_t mid = (lo + hi) >> 1;
        const int32_t x = nb[mid];
        if (x == v2) return mid;
        if (x > v2) hi = mid - 1;
        else lo = mid + 1;
    }
    return -1;
}

__global__ void k_partner(const int64_t* __restrict__ off, const int32_t* __restrict__ nb,
                          const int32_t* __restrict__ esrc, int64_t m2, int32_t* __restrict__ partner,
                          unsigned long long* __restrict__ missing)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t p = find_slot(off, nb, nb[i], esrc[i]);
        if (p < 0) atomicAdd(missing, 1ull);
        partner[i] = (int32_t)p;
    }
}

__global__ void k_fwd_flags(const int32_t* __restrict__ esrc, const int32_t* __restrict__ nb, int64_t m2,
                            uint32_t* __restrict__ flag)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x)
        flag[i] = esrc[i] < nb[i] ? 1u : 0u;
}

__global__ void k_fwd_list(const uint32_t* __restrict__ flag, const uint32_t* __restrict__ pos, int64_t m2,
                           int32_t* __restrict__ fwd, int32_t* __restrict__ frank)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < m2; i += (int64_t)gridDim.x * blockDim.x) {
        frank[i] = flag[i] ? (int32_t)pos[i] : -1;
        if (flag[i]) fwd[pos[i]] = (int32_t)i;
    }
}

// Host CSR path: widen-check the int64 neighbour ids, derive esrc, check order.
__global__ void k_from_host_csr(const int64_t* __restrict__ off, const int64_t* __restrict__ nb64, int64_t n,
                                int32_t* __restrict__ nb, int32_t* __restrict__ esrc,
                                unsigned long long* __restrict__ bad)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x) {
        int64_t prev = -1;
        for (int64_t i = off[v]; i < off[v + 1]; ++i) {
            const int64_t x = nb64[i];
            if (x < 0 || x >= n || x <= prev || x == v) atomicAdd(bad, 1ull);
            nb[i] = (int32_t)x;
            esrc[i] = (int32_t)v;
            prev = x;
        }
    }
}

int finish_csr(rtr_graph* g, unsigned long long* h_ctr)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n, m2 = g->m2;
    g->deg = (int32_t*)dev_alloc(g, sizeof(int32_t) * (n + 1));
    g->partner = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    g->fwd = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 / 2 + 1));
    g->frank = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    if (!g->deg || !g->partner || !g->fwd || !g->frank) {
        set_error("device allocation failed for the CSR (n=%lld, 2m=%lld)", (long long)n, (long long)m2);
        return RTR_ERR_CUDA;
    }
    k_degree<<<grid_for(n, kBlock), kBlock, 0, s>>>(g->offsets, n, g->deg);
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr + 3, 0, sizeof(unsigned long long), s));
    k_partner<<<grid_for(m2, kBlock), kBlock, 0, s>>>(g->offsets, g->nbors, g->esrc, m2, g->partner, g->ctr + 3);
    g->launches += 2;
    Scratch sc(g);
    uint32_t* flag = (uint32_t*)sc.get(sizeof(uint32_t) * (m2 + 1));
    uint32_t* pos = (uint32_t*)sc.get(sizeof(uint32_t) * (m2 + 1));
    uint32_t* tmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(m2));
    if (!flag || !pos || !tmp) {
        set_error("device allocation failed (forward list)");
        return RTR_ERR_CUDA;
    }
    k_fwd_flags<<<grid_for(m2, kBlock), kBlock, 0, s>>>(g->esrc, g->nbors, m2, flag);
    exclusive_scan_u32(flag, pos, m2, nullptr, tmp, s);
    k_fwd_list<<<grid_for(m2, kBlock), kBlock, 0, s>>>(flag, pos, m2, g->fwd, g->frank);
    g->launches += 5;
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaMemcpyAsync(h_ctr, g->ctr, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_ctr[3] != 0) {
        set_error("graph is not symmetric: %llu directed edges have no reverse copy", h_ctr[3]);
        return RTR_ERR_INPUT;
    }
    g->m = m2 / 2;
    g->stage = 1;
    return RTR_OK;
}

}  // namespace

int build_csr(rtr_graph* g, const int64_t* d_u, const int64_t* d_v, int64_t m, bool simplify)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    if (n <= 0 || n >= (int64_t)INT32_MAX || m < 0 || 2 * m >= (int64_t)INT32_MAX) {
        set_error("unsupported size: n=%lld m=%lld (need 0 < n < 2^31-1 and 2m < 2^31-1)", (long long)n,
                  (long long)m);
        return RTR_ERR_LIMIT;
    }
    const int B = bits_for((uint64_t)(n - 1));
    if (2 * B > 64) {
        set_error("vertex id width too large");
        return RTR_ERR_LIMIT;
    }
    int64_t m2 = 2 * m;
    unsigned long long h_ctr[8] = {0};
    Scratch sc(g);
    uint64_t* keys = (uint64_t*)sc.get(sizeof(uint64_t) * (m2 + 1));
    uint64_t* alt = (uint64_t*)sc.get(sizeof(uint64_t) * (m2 + 1));
    void* rtmp = sc.get(radix_temp_bytes(m2));
    if (!keys || !alt || !rtmp) {
        set_error("device allocation failed for the edge sort (2m=%lld)", (long long)m2);
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, 8 * sizeof(unsigned long long), s));
    k_make_keys<<<grid_for(m, kBlock), kBlock, 0, s>>>(d_u, d_v, m, n, B, keys, g->ctr + 4);
    uint64_t* sorted = radix_sort_u64(keys, alt, m2, 2 * B, rtmp, s);
    g->launches += 1 + 3 * ((2 * B + 7) / 8);
    uint32_t* keep = (uint32_t*)sc.get(sizeof(uint32_t) * (m2 + 1));
    if (!keep) {
        set_error("device allocation failed");
        return RTR_ERR_CUDA;
    }
    k_flag_keys<<<grid_for(m2, kBlock), kBlock, 0, s>>>(sorted, m2, B, keep, g->ctr + 5, g->ctr + 6);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaMemcpyAsync(h_ctr, g->ctr, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_ctr[4]) {
        set_error("%llu edges have an endpoint outside [0, %lld)", h_ctr[4], (long long)n);
        return RTR_ERR_INPUT;
    }
    if (h_ctr[5] || h_ctr[6]) {
        if (!simplify) {
            set_error("input is not a simple graph: %llu self-loop slots, %llu duplicate slots "
                      "(pass the simplify flag to drop them)",
                      h_ctr[5], h_ctr[6]);
            return RTR_ERR_INPUT;
        }
        uint32_t* pos = (uint32_t*)sc.get(sizeof(uint32_t) * (m2 + 1));
        uint32_t* tmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(m2));
        uint32_t* d_tot = (uint32_t*)sc.get(sizeof(uint32_t));
        uint64_t* out = (sorted == keys) ? alt : keys;
        exclusive_scan_u32(keep, pos, m2, d_tot, tmp, s);
        k_compact_keys<<<grid_for(m2, kBlock), kBlock, 0, s>>>(sorted, keep, pos, m2, out);
        g->launches += 4;
        uint32_t tot = 0;
        RTR_CUDA_TRY(cudaMemcpyAsync(&tot, d_tot, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
        RTR_CUDA_TRY(cudaStreamSynchronize(s));
        sorted = out;
        m2 = tot;
    }
    g->m2 = m2;
    g->offsets = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 1));
    g->nbors = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    g->esrc = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    if (!g->offsets || !g->nbors || !g->esrc) {
        set_error("device allocation failed for the CSR");
        return RTR_ERR_CUDA;
    }
    k_unpack<<<grid_for(m2, kBlock), kBlock, 0, s>>>(sorted, m2, B, g->nbors, g->esrc);
    k_offsets<<<grid_for(m2 + 1, kBlock), kBlock, 0, s>>>(g->esrc, m2, n, g->offsets);
    g->launches += 2;
    return finish_csr(g, h_ctr);
}

int build_csr_from_host_csr(rtr_graph* g, const int64_t* h_offsets, const int64_t* h_nbors)
{
    cudaStream_t s = g->stream;
    const int64_t n = g->n;
    const int64_t m2 = h_offsets[n];
    if (n <= 0 || n >= (int64_t)INT32_MAX || m2 < 0 || m2 >= (int64_t)INT32_MAX || (m2 & 1)) {
        set_error("unsupported CSR size: n=%lld 2m=%lld", (long long)n, (long long)m2);
        return RTR_ERR_LIMIT;
    }
    g->m2 = m2;
    unsigned long long h_ctr[8] = {0};
    g->offsets = (int64_t*)dev_alloc(g, sizeof(int64_t) * (n + 1));
    g->nbors = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    g->esrc = (int32_t*)dev_alloc(g, sizeof(int32_t) * (m2 + 1));
    Scratch sc(g);
    int64_t* nb64 = (int64_t*)sc.get(sizeof(int64_t) * (m2 + 1));
    if (!g->offsets || !g->nbors || !g->esrc || !nb64) {
        set_error("device allocation failed for the CSR");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(g->ctr, 0, 8 * sizeof(unsigned long long), s));
    RTR_CUDA_TRY(cudaMemcpyAsync(g->offsets, h_offsets, sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(nb64, h_nbors, sizeof(int64_t) * m2, cudaMemcpyHostToDevice, s));
    k_from_host_csr<<<grid_for(n, kBlock), kBlock, 0, s>>>(g->offsets, nb64, n, g->nbors, g->esrc, g->ctr + 4);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    RTR_CUDA_TRY(cudaMemcpyAsync(h_ctr, g->ctr, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    if (h_ctr[4]) {
        set_error("CSR rows must be strictly ascending, in range and free of self-loops (%llu violations)", h_ctr[4]);
        return RTR_ERR_INPUT;
    }
    return finish_csr(g, h_ctr);
}

}  // namespace rtr
