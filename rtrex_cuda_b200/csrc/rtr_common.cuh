// Shared definitions for the sm_100a decomposition kernels.
//
// Data layout in HBM (one graph):
//   offsets  int64 [n+1]   CSR row starts (rows sorted by neighbour id, as makeCSR
//                          + sortById leave them, RTRex_Sequential/Graph.cpp:344-384)
//   nbors    int32 [2m]    neighbour ids
//   esrc     int32 [2m]    source vertex of every directed slot
//   partner  int32 [2m]    slot of the reverse copy (getPartnerMap, Graph.cpp:320-340)
//   deg      int32 [n]
// Per-edge state is kept once per undirected edge, at the slot of its forward
// copy (src < dst): the reference's two copies of perEdge always receive the
// same operations in the same order, so they hold the same bits.
//   pe       f64   [2m]    triangle weight  (forward slots authoritative)
//   sup      u32   [2m]    live triangle count
//   st       u8    [2m]    'Y' / 'S' / 'N'
//   pv       f64   [n]     per-vertex triangle weight
//   frank    int32 [2m]    forward rank of a forward slot (position in the forward list)
// Triangle lists (per forward slot e=(a,b), a<b): one TriEntry per common
// neighbour z, ascending in z.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/rtr.h"

namespace rtr {

constexpr int kWarp = 32;

// Status bytes use the reference's characters (Decomposition.h:127).
constexpr uint8_t ST_Y = 'Y';
constexpr uint8_t ST_S = 'S';
constexpr uint8_t ST_N = 'N';

// One triangle (a, b, z) in the list of its edge (a, b), a < b.
struct alignas(16) TriEntry {
    int32_t z;    // third vertex
    int32_t eaz;  // forward slot of edge (a,z)
    int32_t ebz;  // forward slot of edge (b,z)
    int32_t dz;   // degree of z
    double wgt;   // triangle weight 1/double(da*db*dz)  (Decomposition.h:97)
    int32_t raz;  // forward rank of edge (a,z)
    int32_t rbz;  // forward rank of edge (b,z)
};
static_assert(sizeof(TriEntry) == 32, "TriEntry must be two 16-byte vectors");

// Clean-time state of one undirected edge, indexed by forward rank: everything
// a pop reads or writes for the edge in one 32-byte record.
struct alignas(16) EdgeRec {
    double pe;     // perEdge
    double thr;    // eps * 1/double(du*dv): the edge's cleaning threshold
    int64_t t0;    // triangle-list start
    uint32_t cnt;  // triangle-list length
    uint32_t ss;   // live support (low 30 bits) | status code (top 2 bits)
};
static_assert(sizeof(EdgeRec) == 32, "EdgeRec is 32 bytes");
constexpr uint32_t SS_SUP = (1u << 30) - 1u;
constexpr uint32_t SS_Y = 0u;
constexpr uint32_t SS_S = 1u << 30;
constexpr uint32_t SS_N = 2u << 30;
constexpr uint32_t SS_CODE = 3u << 30;

// Error codes returned through the C ABI are the rtr_status values of rtr.h.

// Device-side error word bits (written by kernels, read by the host).
enum DevErr : unsigned {
    DEV_ERR_STACK_OVERFLOW = 1u << 0,
    DEV_ERR_BAD_STATUS = 1u << 1,
    DEV_ERR_SCRATCH = 1u << 2,
    DEV_ERR_SORT = 1u << 3,
    DEV_ERR_WAIT = 1u << 4,  // a bounded wait on an asynchronous copy ran out
};

__host__ __device__ inline double tri_weight(int64_t a, int64_t b, int64_t c)
{
    // 1/double(du*dv*dw) with the int64 product exact (Decomposition.h:97).
    return 1.0 / (double)(a * b * c);
}

}  // namespace rtr

#define RTR_CUDA_TRY(expr)                                     \
    do {                                                       \
        cudaError_t e_ = (expr);                               \
        if (e_ != cudaSuccess) return ::rtr::cuda_fail(e_, #expr, __FILE__, __LINE__); \
    } while (0)

namespace rtr {
int cuda_fail(cudaError_t e, const char* what, const char* file, int line);
void set_error(const char* fmt, ...);
}  // namespace rtr
