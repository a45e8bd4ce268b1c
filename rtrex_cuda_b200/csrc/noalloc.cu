// Weighted triangle counting that allocates no device memory.
//
// Who this is for: callers that cannot let a library call cudaMalloc --
// a serving process that reserves its whole HBM budget up front and hands out
// memory only through its own arena, code on a latency-critical path where
// cudaMalloc / cudaFree may synchronise the device, or hosts that forbid
// third-party allocations.  The caller passes device buffers for the CSR it
// already holds and for every output; the only working memory is a fixed
// static device array compiled into this file.
//
// It computes what rtr_count computes (perEdge, perVertex, support, total),
// with the same ordered folds, so the results are bit-identical; it just does
// it without the triangle lists, intersecting each row pair directly.
//
// The static array (kNoAllocScratchBytes, ~4.3 MB) is held by every GPU that
// loads librtr.so until the process exits.  It holds the degree table of the
// graph (so n is limited to kNoAllocMaxVertices), one partial triangle count
// per CTA of each counting kernel, and an input-error word.  Every call reuses
// it and it keeps the previous call's contents; the degree table and partial
// counts are fully overwritten before they are read and the error word is
// cleared by the first kernel of each call, so nothing leaks between calls --
// but calls that overlap on the GPU (different streams, or different host
// threads on one device) race on it: serialise them.
#include "../../include/rtr.h"
#include "intersect.cuh"
#include "rtr_common.cuh"

#include <cstdint>
#include <mutex>

namespace rtr {
void set_error(const char* fmt, ...);
}

namespace {

using rtr::fold_hits;
using rtr::intersect_rows;
using rtr::lower_bound_row;
using rtr::warp_chunks;

constexpr int64_t kNoAllocMaxVertices = 1 << 20;
constexpr int kNoAllocBlock = 256;   // light kernel: a thread per vertex
constexpr int kNoAllocWarpBlock = 128;  // heavy kernel: a warp per vertex
constexpr int kNoAllocHeavy = 32;   // degree from which a vertex gets a warp
constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kDegBytes = sizeof(int32_t) * (size_t)kNoAllocMaxVertices;
constexpr size_t kPartialOffset = (kDegBytes + 255) / 256 * 256;
constexpr size_t kErrOffset = kPartialOffset + sizeof(unsigned long long) * 2 * kNoAllocMaxBlocks;
constexpr size_t kNoAllocScratchBytes = kErrOffset + 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch per device, looked up with that device
// current (the host-side name of a __device__ array is not a device address and
// must never be handed to a kernel).  A failed lookup is retried on the next call.
constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {};

__global__ void k_na_degrees(const int64_t* __restrict__ off, int64_t n, int32_t* __restrict__ deg,
                             unsigned* __restrict__ err)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) *err = 0u;  // runs before the counting kernels read it
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        deg[v] = (int32_t)(off[v + 1] - off[v]);
}

template <int BLOCK>
__device__ __forceinline__ void block_partial(unsigned long long tri, unsigned long long* __restrict__ partial)
{
    __shared__ unsigned long long s[BLOCK / 32];
    for (int o = 16; o > 0; o >>= 1) tri += __shfl_down_sync(0xffffffffu, tri, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = tri;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int k = 0; k < BLOCK / 32; ++k) t += s[k];
        partial[blockIdx.x] = t;  // every CTA writes its slot, so no clearing is needed
    }
}

// Vertices of degree below kNoAllocHeavy, one thread each.  For every slot
// i = (u,v) of u's row the thread intersects the two sorted rows (merging, or
// binary-searching the short row in the long one); each common neighbour z
// (ascending) adds 1/double(du*dv*dz) to perEdge[i], counts towards support[i],
// and -- when z > v -- to the perVertex[u] fold, which therefore runs over v
// ascending then z > v ascending, the order commonNbr produces
// (Decomposition.h:70-115).  Neighbour ids outside [0, n) are skipped and
// raise the error word.
__global__ void __launch_bounds__(kNoAllocBlock)
    k_na_light(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ deg,
               int64_t n, double* __restrict__ pe, double* __restrict__ pv, uint32_t* __restrict__ sup,
               unsigned long long* __restrict__ partial, unsigned* __restrict__ err)
{
    unsigned long long tri = 0;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t du = deg[u];
        if (du >= kNoAllocHeavy) continue;
        const int64_t a0 = off[u], a1 = off[u + 1];
        double vacc = 0.0;
        for (int64_t i = a0; i < a1; ++i) {
            const int32_t v = nb[i];
            if (v < 0 || v >= n) {
                atomicOr(err, 1u);
                pe[i] = 0.0;
                sup[i] = 0;
                continue;
            }
            const int64_t duv = du * (int64_t)deg[v];
            double eacc = 0.0;
            uint32_t c = 0;
            intersect_rows(nb, a0, a1, off[v], off[v + 1], 16, [&](int32_t z, int64_t, int64_t) {
                if (z < 0 || z >= n) return;  // already flagged at its own slot of u's row
                const double w = 1.0 / (double)(duv * (int64_t)deg[z]);
                eacc += w;
                ++c;
                if (z > v) {
                    vacc += w;
                    if (u < v) ++tri;
                }
            });
            pe[i] = eacc;
            sup[i] = c;
        }
        pv[u] = vacc;
    }
    block_partial<kNoAllocBlock>(tri, partial);
}

// Vertices of degree kNoAllocHeavy and more, one warp each (dealt by id
// modulo the warp count): for every slot i = (u,v) the warp walks the shorter
// of the two rows 32 elements at a time, each lane binary-searching its element
// in the longer row, and folds the common neighbours of each step in lane order
// -- ascending z -- so perEdge[i] and the perVertex[u] fold get exactly the
// thread kernel's sequence of additions.
__global__ void __launch_bounds__(kNoAllocWarpBlock)
    k_na_heavy(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ deg,
               int64_t n, double* __restrict__ pe, double* __restrict__ pv, uint32_t* __restrict__ sup,
               unsigned long long* __restrict__ partial, unsigned* __restrict__ err)
{
    __shared__ double s_w[kNoAllocWarpBlock / 32][32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t nwarps = (int64_t)gridDim.x * (kNoAllocWarpBlock / 32);
    auto search = [&](int64_t lo, int64_t hi, int32_t x) { return lower_bound_row(nb, lo, hi, x); };
    unsigned long long tri = 0;  // lane 0's count
    for (int64_t u = (int64_t)blockIdx.x * (kNoAllocWarpBlock / 32) + wib; u < n; u += nwarps) {
        const int64_t du = deg[u];
        if (du < kNoAllocHeavy) continue;  // uniform across the warp
        const int64_t a0 = off[u], a1 = off[u + 1];
        double vacc = 0.0;
        for (int64_t i = a0; i < a1; ++i) {
            const int32_t v = nb[i];
            if (v < 0 || v >= n) {
                if (lane == 0) {
                    atomicOr(err, 1u);
                    pe[i] = 0.0;
                    sup[i] = 0;
                }
                continue;
            }
            const int64_t duv = du * (int64_t)deg[v];
            const int64_t b0 = off[v], b1 = off[v + 1];
            double eacc = 0.0;
            uint32_t c = 0;
            auto chunk = [&](bool hit, int32_t z) {
                hit = hit && z >= 0 && z < n;
                const double w = hit ? 1.0 / (double)(duv * (int64_t)deg[z]) : 0.0;
                const int below = __popc(__ballot_sync(0xffffffffu, hit && z < v));
                const int cnt = fold_hits(hit, w, s_w[wib], lane, &eacc, &vacc, below);
                c += (uint32_t)cnt;
                if (u < v) tri += (unsigned long long)(cnt - below);
            };
            if (a1 - a0 <= b1 - b0) warp_chunks(nb, a0, a1, b0, b1, lane, search, chunk);
            else warp_chunks(nb, b0, b1, a0, a1, lane, search, chunk);
            if (lane == 0) {
                pe[i] = eacc;
                sup[i] = c;
            }
        }
        if (lane == 0) pv[u] = vacc;
    }
    if (lane != 0) tri = 0;
    block_partial<kNoAllocWarpBlock>(tri, partial);
}

__global__ void k_na_total(const unsigned long long* __restrict__ partial, int nlight, int nheavy,
                           const unsigned* __restrict__ err, int64_t* __restrict__ total)
{
    __shared__ unsigned long long s[32];
    unsigned long long t = 0;
    for (int b = threadIdx.x; b < nlight; b += blockDim.x) t += partial[b];
    for (int b = threadIdx.x; b < nheavy; b += blockDim.x) t += partial[kNoAllocMaxBlocks + b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int k = 0; k < (int)(blockDim.x / 32); ++k) sum += s[k];
        *total = *err ? -1 : (int64_t)sum;  // -1: a neighbour id outside [0, n) was skipped
    }
}

}  // namespace

extern "C" int rtr_count_noalloc(const int64_t* d_offsets, const int32_t* d_nbors, int64_t n, double* d_perEdge,
                                 double* d_perVertex, uint32_t* d_support, int64_t* d_total, void* stream)
{
    if (!d_offsets || !d_total || n < 0 || (n > 0 && (!d_nbors || !d_perEdge || !d_perVertex || !d_support))) {
        rtr::set_error("rtr_count_noalloc: null buffer or negative n (every buffer must be non-null when n > 0)");
        return RTR_ERR_ARG;
    }
    if (n > kNoAllocMaxVertices) {
        rtr::set_error("rtr_count_noalloc: n=%lld exceeds the fixed scratch limit of %lld vertices; "
                       "use rtr_count for larger graphs",
                       (long long)n, (long long)kNoAllocMaxVertices);
        return RTR_ERR_LIMIT;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        rtr::set_error("rtr_count_noalloc: no usable current CUDA device (%s)", cudaGetErrorString(e));
        return RTR_ERR_CUDA;
    }
    void* addr = nullptr;
    {
        // First call on this device: resolve the scratch array's device address.
        std::lock_guard<std::mutex> lock(g_addr_mu);
        if (!g_addr[dev]) {
            e = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch);
            if (e != cudaSuccess) {
                g_addr[dev] = nullptr;
                rtr::set_error("rtr_count_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                               cudaGetErrorString(e));
                return RTR_ERR_CUDA;
            }
        }
        addr = g_addr[dev];
    }
    cudaStream_t s = (cudaStream_t)stream;
    if (n == 0) {
        e = cudaMemsetAsync(d_total, 0, sizeof(int64_t), s);
        if (e != cudaSuccess) {
            rtr::set_error("rtr_count_noalloc: %s", cudaGetErrorString(e));
            return RTR_ERR_CUDA;
        }
        return RTR_OK;
    }
    unsigned char* base = (unsigned char*)addr;
    int32_t* deg = (int32_t*)base;
    unsigned long long* partial = (unsigned long long*)(base + kPartialOffset);
    unsigned* err = (unsigned*)(base + kErrOffset);
    const int64_t want_light = (n + kNoAllocBlock - 1) / kNoAllocBlock;
    const int light_blocks = (int)(want_light < kNoAllocMaxBlocks ? want_light : kNoAllocMaxBlocks);
    const int64_t want_heavy = (n + kNoAllocWarpBlock / 32 - 1) / (kNoAllocWarpBlock / 32);
    const int64_t cap_heavy = 148 * 16;
    const int heavy_blocks = (int)(want_heavy < cap_heavy ? want_heavy : cap_heavy);
    k_na_degrees<<<light_blocks, kNoAllocBlock, 0, s>>>(d_offsets, n, deg, err);
    k_na_light<<<light_blocks, kNoAllocBlock, 0, s>>>(d_offsets, d_nbors, deg, n, d_perEdge, d_perVertex, d_support,
                                                     partial, err);
    k_na_heavy<<<heavy_blocks, kNoAllocWarpBlock, 0, s>>>(d_offsets, d_nbors, deg, n, d_perEdge, d_perVertex,
                                                          d_support, partial + kNoAllocMaxBlocks, err);
    k_na_total<<<1, 1024, 0, s>>>(partial, light_blocks, heavy_blocks, err, d_total);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        rtr::set_error("rtr_count_noalloc: launch failed: %s", cudaGetErrorString(e));
        return RTR_ERR_CUDA;
    }
    return RTR_OK;
}
