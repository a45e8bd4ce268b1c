// Seeded R-MAT graphs generated on the device: synthetic inputs of the shape
// the large-graph measurements use (R-MAT scale 24, edge factor 16,
// a,b,c,d = .57,.19,.19,.05), without a host round trip of the raw edges.
// No counterpart in the reference, which reads edge-list files.
//
// Edge k (0 <= k < edge_factor * 2^scale) takes, at level l (0 <= l < scale),
// one 64-bit draw h = mix64(seed * 0x9E3779B97F4A7C15 ^ (k << 6 | l)), where
// mix64 is the splitmix64 output function (Steele, Lea and Flood, "Fast
// splittable pseudorandom number generators", OOPSLA 2014).  Its high 32 bits
// pick the row half (bit set when hi >= floor((a+b) 2^32)), its low 32 bits the
// column half (bit set when lo >= floor(a/(a+b) 2^32) in the top row half,
// floor(c/(1-a-b) 2^32) in the bottom one); level l sets bit scale-1-l of the
// source and destination ids.  The pairs are then symmetrised, and self-loops
// and repeated pairs dropped, by the CSR build.  rtrex_cuda_b200.graphgen.rmat_hashed
// is the same definition in numpy.
#include "../../include/rtr.h"
#include "primitives.cuh"
#include "rtr_graph.cuh"

#include <cmath>

namespace rtr {
int make_graph_handle(int64_t n, int device, rtr_graph** out);
}

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

__global__ void k_rmat(int64_t M, int scale, uint64_t seed_mix, uint64_t t_ab, uint64_t t_a, uint64_t t_c,
                       int64_t* __restrict__ u, int64_t* __restrict__ v)
{
    for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < M; k += (int64_t)gridDim.x * blockDim.x) {
        uint64_t s = 0, t = 0;
        for (int l = 0; l < scale; ++l) {
            const uint64_t h = mix64(seed_mix ^ (((uint64_t)k << 6) | (uint64_t)l));
            const uint64_t hi = h >> 32, lo = h & 0xffffffffull;
            const uint64_t ii = hi >= t_ab ? 1ull : 0ull;
            const uint64_t jj = lo >= (ii ? t_c : t_a) ? 1ull : 0ull;
            s |= ii << (scale - 1 - l);
            t |= jj << (scale - 1 - l);
        }
        u[k] = (int64_t)s;
        v[k] = (int64_t)t;
    }
}

uint64_t threshold32(double p)
{
    if (!(p > 0.0)) return 0;
    if (p >= 1.0) return 1ull << 32;
    return (uint64_t)std::floor(p * 4294967296.0);
}

}  // namespace

using namespace rtr;

extern "C" int rtr_graph_create_rmat(int scale, int64_t edge_factor, double a, double b, double c, uint64_t seed,
                                     int device, rtr_graph** out)
{
    if (!out || scale < 1 || scale > 30 || edge_factor < 1 || !(a >= 0) || !(b >= 0) || !(c >= 0) ||
        !(a + b > 0) || !(a + b < 1) || !(c <= 1 - a - b)) {
        set_error("rtr_graph_create_rmat: need 1 <= scale <= 30, edge_factor >= 1, a,b,c >= 0, 0 < a+b < 1, "
                  "c <= 1-a-b");
        return RTR_ERR_ARG;
    }
    const int64_t n = 1ll << scale;
    if (edge_factor > ((1ll << 30) - 1) / n) {
        set_error("rtr_graph_create_rmat: edge_factor * 2^scale must stay below 2^30");
        return RTR_ERR_LIMIT;
    }
    const int64_t M = edge_factor * n;
    int rc = make_graph_handle(n, device, out);
    if (rc) return rc;
    rtr_graph* g = *out;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, g->stream);
    {
        Scratch sc(g);
        int64_t* du = (int64_t*)sc.get(sizeof(int64_t) * (M + 1));
        int64_t* dv = (int64_t*)sc.get(sizeof(int64_t) * (M + 1));
        if (!du || !dv) {
            set_error("device allocation failed for %lld generated edges", (long long)M);
            rc = RTR_ERR_CUDA;
        } else {
            k_rmat<<<grid_for(M, 256), 256, 0, g->stream>>>(M, scale, seed * 0x9E3779B97F4A7C15ull,
                                                             threshold32(a + b), threshold32(a / (a + b)),
                                                             threshold32(c / (1.0 - a - b)), du, dv);
            g->launches += 1;
            rc = build_csr(g, du, dv, M, true);
        }
    }
    cudaEventRecord(e1, g->stream);
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(&g->ms_build, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) {
        rtr_graph_destroy(g);
        *out = nullptr;
    }
    return rc;
}
