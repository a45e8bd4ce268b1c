// Escape edge-list parsing on the device: loadGraph_Escape
// (RTRex_Sequential/GraphIO.cpp:19-74) with the line rules of escape_text.h,
// feeding the device CSR build directly (no host edge arrays).
//
// A file is streamed to HBM through two pinned staging chunks (the read of one
// chunk overlaps the copy of the previous one; small files take one pageable
// copy), then:
//   k_nl_count   one CTA per 4 KiB tile, 16 bytes per thread: '\n' per tile
//   k_nl_write   positions of every '\n' (tile offsets from a scan, CTA-local scan)
//   k_lines      one thread per line: classify and parse (esc_line)
//   scan         rank of each data line; the first data line is the header
//   k_scatter    data line of rank r (1 <= r <= m) -> edge r-1
// All HBM-bound byte work: the text is read twice (counting, writing) plus once
// per line by the parser.
#include "escape_text.h"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <algorithm>
#include <cinttypes>
#include <cstdio>
#include <mutex>
#include <vector>

namespace rtr {
namespace {

constexpr int kBlock = 256;
constexpr int64_t kTile = 16 * kBlock;  // bytes per CTA tile

__device__ inline int count_nl16(const uint4 w, int64_t base, int64_t len)
{
    const uint32_t words[4] = {w.x, w.y, w.z, w.w};
    int c = 0;
    for (int k = 0; k < 4; ++k) {
        const uint32_t x = words[k] ^ 0x0a0a0a0au;  // zero byte where the text has '\n'
        const uint32_t z = (x - 0x01010101u) & ~x & 0x80808080u;
        if (!z) continue;
        for (int b = 0; b < 4; ++b)
            if (((x >> (8 * b)) & 0xffu) == 0 && base + 4 * k + b < len) ++c;
    }
    return c;
}

__global__ void __launch_bounds__(kBlock) k_nl_count(const char* __restrict__ text, int64_t len,
                                                     int64_t* __restrict__ tile_cnt)
{
    __shared__ int warp_sum[kBlock / 32];
    const int64_t base = blockIdx.x * kTile + 16 * (int64_t)threadIdx.x;
    int c = 0;
    if (base < len) c = count_nl16(*reinterpret_cast<const uint4*>(text + base), base, len);
    for (int o = 16; o; o >>= 1) c += __shfl_down_sync(0xffffffffu, c, o);
    if ((threadIdx.x & 31) == 0) warp_sum[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int64_t t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += warp_sum[w];
        tile_cnt[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kBlock) k_nl_write(const char* __restrict__ text, int64_t len,
                                                     const int64_t* __restrict__ tile_off, int64_t* __restrict__ nlpos)
{
    __shared__ int warp_sum[kBlock / 32];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    const int64_t base = blockIdx.x * kTile + 16 * (int64_t)threadIdx.x;
    uint4 w = make_uint4(0, 0, 0, 0);
    int c = 0;
    if (base < len) {
        w = *reinterpret_cast<const uint4*>(text + base);
        c = count_nl16(w, base, len);
    }
    int incl = c;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += y;
    }
    if (lane == 31) warp_sum[wid] = incl;
    __syncthreads();
    int before = 0;
    for (int k = 0; k < wid; ++k) before += warp_sum[k];
    if (!c) return;
    int64_t out = tile_off[blockIdx.x] + before + incl - c;
    const char* bytes = reinterpret_cast<const char*>(&w);
    for (int b = 0; b < 16; ++b)
        if (bytes[b] == '\n' && base + b < len) nlpos[out++] = base + b;
}

// One thread per line: kind (0 skipped, 1 data, 2 malformed data), the two
// values, the first data line and the first malformed one.  The two minima
// are kept per thread and reduced per warp, so the shared words see one
// atomic per warp rather than one per line.
__global__ void k_lines(const char* __restrict__ text, int64_t len, const int64_t* __restrict__ nlpos, int64_t nnl,
                        int64_t L, uint32_t* __restrict__ is_data, int64_t* __restrict__ va, int64_t* __restrict__ vb,
                        unsigned long long* __restrict__ first)
{
    unsigned first_data = 0xffffffffu, first_bad = 0xffffffffu;  // line indices are below 2^31
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
        const int64_t s = i == 0 ? 0 : nlpos[i - 1] + 1;
        const int64_t e = i < nnl ? nlpos[i] : len;
        int64_t a = 0, b = 0;
        const int kind = esc_line(text + s, text + e, &a, &b);
        is_data[i] = kind != 0;
        va[i] = a;
        vb[i] = b;
        if (kind && (unsigned)i < first_data) first_data = (unsigned)i;
        if (kind == 2 && (unsigned)i < first_bad) first_bad = (unsigned)i;
    }
    first_data = __reduce_min_sync(0xffffffffu, first_data);
    first_bad = __reduce_min_sync(0xffffffffu, first_bad);
    if ((threadIdx.x & 31) == 0) {
        if (first_data != 0xffffffffu) atomicMin(&first[0], (unsigned long long)first_data);
        if (first_bad != 0xffffffffu) atomicMin(&first[1], (unsigned long long)first_bad);
    }
}

__global__ void k_scatter(const uint32_t* __restrict__ is_data, const uint32_t* __restrict__ rank,
                          const int64_t* __restrict__ va, const int64_t* __restrict__ vb, int64_t L, int64_t m,
                          int64_t* __restrict__ du, int64_t* __restrict__ dv)
{
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < L; i += (int64_t)gridDim.x * blockDim.x) {
        if (!is_data[i]) continue;
        const int64_t r = rank[i];
        if (r < 1 || r > m) continue;  // the header, or lines past the m-th edge
        du[r - 1] = va[i];
        dv[r - 1] = vb[i];
    }
}

// Two pinned staging chunks shared by every file parse of the process
// (allocated on first use, held until exit; portable across devices).  A parse
// holds the lock while it streams its file.
struct PinnedRing {
    static constexpr size_t kChunk = 32u << 20;
    std::mutex mu;
    char* p[2] = {nullptr, nullptr};
    bool ready()
    {
        for (char*& q : p)
            if (!q && cudaHostAlloc((void**)&q, kChunk, cudaHostAllocPortable) != cudaSuccess) {
                q = nullptr;
                return false;
            }
        return true;
    }
};
PinnedRing g_ring;

}  // namespace

// Parse the Escape text [h_text or file f, len bytes) into device edge arrays
// (scratch of sc).  `what` names the input in error messages.
int parse_escape_device(rtr_graph* g, Scratch& sc, const char* h_text, FILE* f, int64_t len, const char* what,
                        int64_t* n_out, int64_t* m_out, int64_t** du_out, int64_t** dv_out)
{
    cudaStream_t s = g->stream;
    char* text = (char*)sc.get((size_t)len + kTile + 16);
    if (!text) {
        set_error("device allocation failed for %lld bytes of text", (long long)len);
        return RTR_ERR_CUDA;
    }
    char last = '\n';
    std::vector<char> small;
    constexpr int64_t kDirect = 16ll << 20;  // below this, one pageable read and copy
    if (!h_text && len <= kDirect) {
        small.resize((size_t)len + 1);
        if (len && fread(small.data(), 1, (size_t)len, f) != (size_t)len) {
            set_error("short read on %s", what);
            return RTR_ERR_IO;
        }
        h_text = small.data();
    }
    if (h_text) {
        if (len) RTR_CUDA_TRY(cudaMemcpyAsync(text, h_text, (size_t)len, cudaMemcpyHostToDevice, s));
        if (len) last = h_text[len - 1];
    } else {
        // chunked read through two pinned buffers; the read of chunk k+1
        // overlaps the copy of chunk k
        const size_t chunk = PinnedRing::kChunk;
        std::lock_guard<std::mutex> lock(g_ring.mu);
        if (!g_ring.ready()) {
            set_error("pinned host allocation failed");
            return RTR_ERR_CUDA;
        }
        char* const* pin = g_ring.p;
        cudaEvent_t done[2];
        for (int k = 0; k < 2; ++k) {
            cudaEventCreateWithFlags(&done[k], cudaEventDisableTiming);
            cudaEventRecord(done[k], s);
        }
        int64_t off = 0;
        int k = 0;
        int rc = RTR_OK;
        while (off < len) {
            cudaEventSynchronize(done[k]);
            const size_t want = (size_t)std::min<int64_t>((int64_t)chunk, len - off);
            const size_t got = fread(pin[k], 1, want, f);
            if (got != want) {
                set_error("short read on %s", what);
                rc = RTR_ERR_IO;
                break;
            }
            last = pin[k][got - 1];
            if (cudaMemcpyAsync(text + off, pin[k], got, cudaMemcpyHostToDevice, s) != cudaSuccess) {
                set_error("host-to-device copy of %s failed", what);
                rc = RTR_ERR_CUDA;
                break;
            }
            cudaEventRecord(done[k], s);
            off += (int64_t)got;
            k ^= 1;
        }
        cudaStreamSynchronize(s);
        for (int j = 0; j < 2; ++j) cudaEventDestroy(done[j]);
        if (rc) return rc;
    }
    // zero the tail so vector loads of the last tile read defined bytes
    RTR_CUDA_TRY(cudaMemsetAsync(text + len, 0, kTile + 16, s));

    const int64_t tiles = std::max<int64_t>(1, (len + kTile - 1) / kTile);
    int64_t* tile_cnt = (int64_t*)sc.get(sizeof(int64_t) * (tiles + 1));
    int64_t* tile_off = (int64_t*)sc.get(sizeof(int64_t) * (tiles + 1));
    int64_t* ltmp = (int64_t*)sc.get(sizeof(int64_t) * scan_temp_elems(tiles + 1));
    if (!tile_cnt || !tile_off || !ltmp) {
        set_error("device allocation failed (parse tiles)");
        return RTR_ERR_CUDA;
    }
    k_nl_count<<<(unsigned)tiles, kBlock, 0, s>>>(text, len, tile_cnt);
    exclusive_scan_i64(tile_cnt, tile_off, tiles, tile_off + tiles, ltmp, s);
    int64_t nnl = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(&nnl, tile_off + tiles, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    const int64_t L = nnl + ((len > 0 && last != '\n') ? 1 : 0);
    if (L >= (1ll << 31)) {
        set_error("%s has %lld lines; at most 2^31-1 are supported", what, (long long)L);
        return RTR_ERR_LIMIT;
    }
    int64_t* nlpos = (int64_t*)sc.get(sizeof(int64_t) * (nnl + 1));
    uint32_t* is_data = (uint32_t*)sc.get(sizeof(uint32_t) * (L + 1));
    uint32_t* rank = (uint32_t*)sc.get(sizeof(uint32_t) * (L + 1));
    uint32_t* utmp = (uint32_t*)sc.get(sizeof(uint32_t) * scan_temp_elems(L + 1));
    int64_t* va = (int64_t*)sc.get(sizeof(int64_t) * (L + 1));
    int64_t* vb = (int64_t*)sc.get(sizeof(int64_t) * (L + 1));
    unsigned long long* first = (unsigned long long*)sc.get(sizeof(unsigned long long) * 2);
    uint32_t* ndata = (uint32_t*)sc.get(sizeof(uint32_t) * 2);
    if (!nlpos || !is_data || !rank || !utmp || !va || !vb || !first || !ndata) {
        set_error("device allocation failed (parse lines)");
        return RTR_ERR_CUDA;
    }
    RTR_CUDA_TRY(cudaMemsetAsync(first, 0xff, sizeof(unsigned long long) * 2, s));
    RTR_CUDA_TRY(cudaMemsetAsync(ndata, 0, sizeof(uint32_t) * 2, s));
    if (nnl) k_nl_write<<<(unsigned)tiles, kBlock, 0, s>>>(text, len, tile_off, nlpos);
    if (L) {
        k_lines<<<grid_for(L, kBlock), kBlock, 0, s>>>(text, len, nlpos, nnl, L, is_data, va, vb, first);
        exclusive_scan_u32(is_data, rank, L, ndata, utmp, s);
    }
    g->launches += 6;
    RTR_CUDA_TRY(cudaGetLastError());
    unsigned long long fl[2];
    uint32_t D = 0;
    RTR_CUDA_TRY(cudaMemcpyAsync(fl, first, sizeof fl, cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(&D, ndata, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    const unsigned long long none = ~0ull;
    // the host loader's order of checks: a malformed header, then a negative
    // header, then the first malformed data line, then a short edge count
    if (fl[0] == none) {
        set_error("%s: no header line", what);
        return RTR_ERR_IO;
    }
    if (fl[1] == fl[0]) {
        set_error("%s:%lld: expected two integers", what, (long long)fl[1] + 1);
        return RTR_ERR_IO;
    }
    int64_t hdr[2];
    RTR_CUDA_TRY(cudaMemcpyAsync(&hdr[0], va + fl[0], sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaMemcpyAsync(&hdr[1], vb + fl[0], sizeof(int64_t), cudaMemcpyDeviceToHost, s));
    RTR_CUDA_TRY(cudaStreamSynchronize(s));
    const int64_t n = hdr[0], m = hdr[1];
    if (n < 0 || m < 0) {
        set_error("%s: negative header values", what);
        return RTR_ERR_IO;
    }
    if (fl[1] != none) {
        set_error("%s:%lld: expected two integers", what, (long long)fl[1] + 1);
        return RTR_ERR_IO;
    }
    const int64_t got = std::min<int64_t>((int64_t)D - 1, m);
    if (got < m) {
        // the reference reports edges counted in both directions (GraphIO.cpp:67-71)
        set_error("expected %" PRId64 " edges, only got %" PRId64, 2 * m, 2 * got);
        return RTR_ERR_IO;
    }
    int64_t* du = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    int64_t* dv = (int64_t*)sc.get(sizeof(int64_t) * (m + 1));
    if (!du || !dv) {
        set_error("device allocation failed for %lld edges", (long long)m);
        return RTR_ERR_CUDA;
    }
    if (m) k_scatter<<<grid_for(L, kBlock), kBlock, 0, s>>>(is_data, rank, va, vb, L, m, du, dv);
    g->launches += 1;
    RTR_CUDA_TRY(cudaGetLastError());
    *n_out = n;
    *m_out = m;
    *du_out = du;
    *dv_out = dv;
    return RTR_OK;
}

}  // namespace rtr
