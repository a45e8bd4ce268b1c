// Exclusive scan and stable LSD radix sort (reduce-then-scan), sm_100a.
#include "primitives.cuh"
#include "rtr_common.cuh"

#include <algorithm>

namespace rtr {

namespace {

constexpr int kBlock = 256;
constexpr int kItems = 8;
constexpr int kTile = kBlock * kItems;  // 2048 elements per CTA tile
constexpr int kRadixBits = 8;
constexpr int kBins = 1 << kRadixBits;

template <typename T>
__device__ T block_exclusive_scan(T v, T* s_warp, T* total)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int kWarps = kBlock / 32;
    T x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (warp == 0) {
        T w = lane < kWarps ? s_warp[lane] : T(0);
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            T y = __shfl_up_sync(0xffffffffu, w, off);
            if (lane >= off) w += y;
        }
        if (lane < kWarps) s_warp[lane] = w;
    }
    __syncthreads();
    const T prefix = warp > 0 ? s_warp[warp - 1] : T(0);
    if (total) *total = s_warp[kWarps - 1];
    __syncthreads();
    return prefix + x - v;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_scan_reduce(const T* __restrict__ in, int64_t n, T* __restrict__ sums)
{
    __shared__ T s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < n) acc += in[base + k];
    T tot;
    block_exclusive_scan<T>(acc, s_warp, &tot);
    if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

// One CTA scans the per-tile sums in place (exclusive) and writes the total.
template <typename T>
__global__ void __launch_bounds__(kBlock) k_scan_top(T* __restrict__ sums, int64_t nb, T* __restrict__ total)
{
    __shared__ T s_warp[32];
    T carry = 0;
    for (int64_t start = 0; start < nb; start += kTile) {
        const int64_t base = start + (int64_t)threadIdx.x * kItems;
        T loc[kItems];
        T acc = 0;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            loc[k] = (base + k < nb) ? sums[base + k] : T(0);
            acc += loc[k];
        }
        T tile_tot;
        T pre = block_exclusive_scan<T>(acc, s_warp, &tile_tot) + carry;
#pragma unroll
        for (int k = 0; k < kItems; ++k) {
            if (base + k < nb) sums[base + k] = pre;
            pre += loc[k];
        }
        carry += tile_tot;
    }
    if (threadIdx.x == 0 && total) *total = carry;
}

template <typename T>
__global__ void __launch_bounds__(kBlock) k_scan_down(const T* __restrict__ in, T* __restrict__ out, int64_t n,
                                                       const T* __restrict__ sums)
{
    __shared__ T s_warp[32];
    const int64_t base = (int64_t)blockIdx.x * kTile + (int64_t)threadIdx.x * kItems;
    T loc[kItems];
    T acc = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        loc[k] = (base + k < n) ? in[base + k] : T(0);
        acc += loc[k];
    }
    T pre = block_exclusive_scan<T>(acc, s_warp, nullptr) + sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (base + k < n) out[base + k] = pre;
        pre += loc[k];
    }
}

template <typename T>
int scan_impl(const T* d_in, T* d_out, int64_t n, T* d_total, T* temp, cudaStream_t s)
{
    if (n <= 0) {
        if (d_total) RTR_CUDA_TRY(cudaMemsetAsync(d_total, 0, sizeof(T), s));
        return RTR_OK;
    }
    const int64_t nb = (n + kTile - 1) / kTile;
    k_scan_reduce<T><<<(unsigned)nb, kBlock, 0, s>>>(d_in, n, temp);
    k_scan_top<T><<<1, kBlock, 0, s>>>(temp, nb, d_total);
    k_scan_down<T><<<(unsigned)nb, kBlock, 0, s>>>(d_in, d_out, n, temp);
    RTR_CUDA_TRY(cudaGetLastError());
    return RTR_OK;
}

// ---------------------------------------------------------------- radix sort

__global__ void __launch_bounds__(kBlock) k_radix_hist(const uint64_t* __restrict__ keys, int64_t n, int shift,
                                                        uint32_t* __restrict__ hist, int64_t ntiles)
{
    __shared__ uint32_t h[kBins];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        const int64_t idx = base + (int64_t)k * kBlock + threadIdx.x;
        if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & (kBins - 1)], 1u);
    }
    __syncthreads();
    hist[(int64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Stable scatter: the tile is consumed in kItems rounds of kBlock keys (round
// k holds keys base + k*kBlock + t, t ascending), so ranks follow input order.
__global__ void __launch_bounds__(kBlock) k_radix_scatter(const uint64_t* __restrict__ keys,
                                                           uint64_t* __restrict__ out, int64_t n, int shift,
                                                           const uint32_t* __restrict__ offs, int64_t ntiles)
{
    constexpr int kWarps = kBlock / 32;
    __shared__ uint32_t s_base[kBins];
    __shared__ uint32_t s_run[kBins];
    __shared__ uint32_t s_cnt[kWarps][kBins + 1];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    s_base[t] = offs[(int64_t)t * ntiles + blockIdx.x];
    s_run[t] = 0;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) s_cnt[w][t] = 0;
    if (t < kWarps) s_cnt[t][kBins] = 0;
    __syncthreads();
    const int64_t base = (int64_t)blockIdx.x * kTile;
    const unsigned lt = (1u << lane) - 1u;
    for (int k = 0; k < kItems; ++k) {
        const int64_t idx = base + (int64_t)k * kBlock + t;
        const bool valid = idx < n;
        const uint64_t key = valid ? keys[idx] : 0ull;
        const unsigned d = valid ? (unsigned)((key >> shift) & (kBins - 1)) : (unsigned)kBins;
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const unsigned r = __popc(peers & lt);
        if (r == 0) s_cnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            uint32_t pre = s_run[d];
            for (int w = 0; w < warp; ++w) pre += s_cnt[w][d];
            out[s_base[d] + pre + r] = key;
        }
        __syncthreads();
        uint32_t add = 0;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) {
            add += s_cnt[w][t];
            s_cnt[w][t] = 0;
        }
        s_run[t] += add;
        if (t < kWarps) s_cnt[t][kBins] = 0;
        __syncthreads();
    }
}

}  // namespace

int64_t scan_temp_elems(int64_t n)
{
    return (n + kTile - 1) / kTile + 1;
}

int exclusive_scan_u32(const uint32_t* d_in, uint32_t* d_out, int64_t n, uint32_t* d_total, uint32_t* temp,
                       cudaStream_t s)
{
    return scan_impl<uint32_t>(d_in, d_out, n, d_total, temp, s);
}

int exclusive_scan_i64(const int64_t* d_in, int64_t* d_out, int64_t n, int64_t* d_total, int64_t* temp,
                       cudaStream_t s)
{
    return scan_impl<int64_t>(d_in, d_out, n, d_total, temp, s);
}

size_t radix_temp_bytes(int64_t n)
{
    const int64_t ntiles = (n + kTile - 1) / kTile;
    const int64_t h = ntiles * kBins;
    return (size_t)(2 * h + scan_temp_elems(h)) * sizeof(uint32_t);
}

uint64_t* radix_sort_u64(uint64_t* d_keys, uint64_t* d_alt, int64_t n, int nbits, void* temp, cudaStream_t s)
{
    if (n <= 1) return d_keys;
    const int64_t ntiles = (n + kTile - 1) / kTile;
    const int64_t h = ntiles * kBins;
    uint32_t* hist = (uint32_t*)temp;
    uint32_t* offs = hist + h;
    uint32_t* stmp = offs + h;
    uint64_t* src = d_keys;
    uint64_t* dst = d_alt;
    for (int shift = 0; shift < nbits; shift += kRadixBits) {
        k_radix_hist<<<(unsigned)ntiles, kBlock, 0, s>>>(src, n, shift, hist, ntiles);
        scan_impl<uint32_t>(hist, offs, h, nullptr, stmp, s);
        k_radix_scatter<<<(unsigned)ntiles, kBlock, 0, s>>>(src, dst, n, shift, offs, ntiles);
        std::swap(src, dst);
    }
    return src;
}

int grid_for(int64_t work, int block, int blocks_per_sm)
{
    static const int sms = [] {  // initialised once, thread-safe
        int dev = 0, count = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || count <= 0)
            count = 148;
        return count;
    }();
    const int64_t need = (work + block - 1) / block;
    const int64_t cap = (int64_t)sms * blocks_per_sm;
    int64_t g = std::min<int64_t>(need, cap);
    return (int)std::max<int64_t>(1, g);
}

}  // namespace rtr
