// Device-wide primitives: exclusive scan and LSD radix sort of 64-bit keys.
// Hand-written (no CUB/Thrust); all launches go to the caller's stream.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace rtr {

// Exclusive scan of n elements; writes the grand total to *d_total when non-null.
// temp must hold scan_temp_elems(n) elements of T.
int64_t scan_temp_elems(int64_t n);
int exclusive_scan_u32(const uint32_t* d_in, uint32_t* d_out, int64_t n, uint32_t* d_total,
                       uint32_t* temp, cudaStream_t s);
int exclusive_scan_i64(const int64_t* d_in, int64_t* d_out, int64_t n, int64_t* d_total,
                       int64_t* temp, cudaStream_t s);

// Stable LSD radix sort of n uint64 keys over bits [0, nbits).  Uses d_alt as
// the ping-pong buffer; returns the buffer that holds the sorted keys
// (d_keys or d_alt).  temp must hold radix_temp_bytes(n) bytes.
size_t radix_temp_bytes(int64_t n);
uint64_t* radix_sort_u64(uint64_t* d_keys, uint64_t* d_alt, int64_t n, int nbits, void* temp,
                         cudaStream_t s);

// Number of bits needed to represent values in [0, x].
inline int bits_for(uint64_t x)
{
    int b = 0;
    while (b < 64 && (x >> b) != 0) ++b;
    return b == 0 ? 1 : b;
}

// Grid size for grid-stride kernels: a multiple of the SM count.
int grid_for(int64_t work, int block, int blocks_per_sm = 8);

}  // namespace rtr
