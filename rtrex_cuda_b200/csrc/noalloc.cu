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
// The static array (kNoAllocScratchBytes, ~4.2 MB) is held by every GPU that
// loads librtr.so until the process exits.  It holds the degree table of the
// graph (so n is limited to kNoAllocMaxVertices) and one partial triangle
// count per CTA.  Every call reuses it and it keeps the previous call's
// contents; both parts are fully overwritten before they are read, and calls
// that overlap on the GPU (different streams, or different host threads on
// one device) race on it -- serialise them.
#include "../../include/rtr.h"
#include "rtr_common.cuh"

#include <cstdint>
#include <mutex>

namespace rtr {
void set_error(const char* fmt, ...);
}

namespace {

constexpr int64_t kNoAllocMaxVertices = 1 << 20;
constexpr int kNoAllocBlock = 256;
constexpr int kNoAllocMaxBlocks = 4096;
constexpr size_t kDegBytes = sizeof(int32_t) * (size_t)kNoAllocMaxVertices;
constexpr size_t kPartialOffset = (kDegBytes + 255) / 256 * 256;
constexpr size_t kNoAllocScratchBytes = kPartialOffset + sizeof(unsigned long long) * kNoAllocMaxBlocks;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device with that
// device current (the host-side name of a __device__ array is not a device
// address and must never be handed to a kernel).
constexpr int kMaxDevices = 64;
std::once_flag g_once[kMaxDevices];
void* g_addr[kMaxDevices] = {};
cudaError_t g_setup[kMaxDevices] = {};

__global__ void k_na_degrees(const int64_t* __restrict__ off, int64_t n, int32_t* __restrict__ deg)
{
    for (int64_t v = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; v < n; v += (int64_t)gridDim.x * blockDim.x)
        deg[v] = (int32_t)(off[v + 1] - off[v]);
}

// One thread per vertex u.  For every slot i = (u,v) of u's row it merges the
// two sorted rows; each common neighbour z (ascending) adds 1/double(du*dv*dz)
// to perEdge[i], counts towards support[i], and -- when z > v -- to the
// perVertex[u] fold, which therefore runs over v ascending then z > v
// ascending, the order commonNbr produces (Decomposition.h:70-115).
__global__ void __launch_bounds__(kNoAllocBlock)
    k_na_count(const int64_t* __restrict__ off, const int32_t* __restrict__ nb, const int32_t* __restrict__ deg,
               int64_t n, double* __restrict__ pe, double* __restrict__ pv, uint32_t* __restrict__ sup,
               unsigned long long* __restrict__ partial)
{
    unsigned long long tri = 0;
    for (int64_t u = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; u < n; u += (int64_t)gridDim.x * blockDim.x) {
        const int64_t du = deg[u];
        const int64_t a0 = off[u], a1 = off[u + 1];
        double vacc = 0.0;
        for (int64_t i = a0; i < a1; ++i) {
            const int32_t v = nb[i];
            const int64_t duv = du * (int64_t)deg[v];
            const int64_t b0 = off[v], b1 = off[v + 1];
            double eacc = 0.0;
            uint32_t c = 0;
            int64_t p = a0, q = b0;
            while (p < a1 && q < b1) {
                const int32_t x = nb[p], y = nb[q];
                if (x < y) {
                    ++p;
                } else if (x > y) {
                    ++q;
                } else {
                    const double w = 1.0 / (double)(duv * (int64_t)deg[x]);
                    eacc += w;
                    ++c;
                    if (x > v) {
                        vacc += w;
                        if (u < v) ++tri;
                    }
                    ++p;
                    ++q;
                }
            }
            pe[i] = eacc;
            sup[i] = c;
        }
        pv[u] = vacc;
    }
    __shared__ unsigned long long s[kNoAllocBlock / 32];
    for (int o = 16; o > 0; o >>= 1) tri += __shfl_down_sync(0xffffffffu, tri, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = tri;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long t = 0;
        for (int k = 0; k < kNoAllocBlock / 32; ++k) t += s[k];
        partial[blockIdx.x] = t;  // every CTA writes its slot, so no clearing is needed
    }
}

__global__ void k_na_total(const unsigned long long* __restrict__ partial, int nblocks, int64_t* __restrict__ total)
{
    __shared__ unsigned long long s[32];
    unsigned long long t = 0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) t += partial[b];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_down_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long sum = 0;
        for (int k = 0; k < (int)(blockDim.x / 32); ++k) sum += s[k];
        *total = (int64_t)sum;
    }
}

}  // namespace

extern "C" int rtr_count_noalloc(const int64_t* d_offsets, const int32_t* d_nbors, int64_t n, double* d_perEdge,
                                 double* d_perVertex, uint32_t* d_support, int64_t* d_total, void* stream)
{
    if (!d_offsets || !d_perVertex || !d_total || n < 0) {
        rtr::set_error("rtr_count_noalloc: null buffer or negative n");
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
    // First call on this device: resolve the scratch array's device address.
    std::call_once(g_once[dev], [dev] { g_setup[dev] = cudaGetSymbolAddress(&g_addr[dev], g_noalloc_scratch); });
    if (g_setup[dev] != cudaSuccess || !g_addr[dev]) {
        rtr::set_error("rtr_count_noalloc: cudaGetSymbolAddress failed on device %d: %s", dev,
                       cudaGetErrorString(g_setup[dev]));
        return RTR_ERR_CUDA;
    }
    if (n == 0) {
        cudaMemsetAsync(d_total, 0, sizeof(int64_t), (cudaStream_t)stream);
        return RTR_OK;
    }
    unsigned char* base = (unsigned char*)g_addr[dev];
    int32_t* deg = (int32_t*)base;
    unsigned long long* partial = (unsigned long long*)(base + kPartialOffset);
    cudaStream_t s = (cudaStream_t)stream;
    const int blocks = (int)((n + kNoAllocBlock - 1) / kNoAllocBlock < kNoAllocMaxBlocks
                                 ? (n + kNoAllocBlock - 1) / kNoAllocBlock
                                 : kNoAllocMaxBlocks);
    k_na_degrees<<<blocks, kNoAllocBlock, 0, s>>>(d_offsets, n, deg);
    k_na_count<<<blocks, kNoAllocBlock, 0, s>>>(d_offsets, d_nbors, deg, n, d_perEdge, d_perVertex, d_support,
                                                partial);
    k_na_total<<<1, 1024, 0, s>>>(partial, blocks, d_total);
    e = cudaGetLastError();
    if (e != cudaSuccess) {
        rtr::set_error("rtr_count_noalloc: launch failed: %s", cudaGetErrorString(e));
        return RTR_ERR_CUDA;
    }
    return RTR_OK;
}
