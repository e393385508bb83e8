// primitives.cuh -- device scan and stable LSD radix sort used by the octree
// build and by the Morton ordering of queries.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace mlods
{

// Exclusive scan of n uint32 values (in may equal out).  If total != nullptr
// the sum is written there (device pointer).  temp must hold
// scan_temp_bytes(n) bytes.  Sums must fit in 32 bits.
size_t scan_temp_bytes(int64_t n);
cudaError_t exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total, void* temp,
                               cudaStream_t s);

// Stable sort of (key, value) pairs by key bits [0, nbits), least significant
// digit first, 8 bits per pass.  Keys/values are ping-ponged between the two
// buffers; on return *result_in_alt tells which buffer holds the result.
// temp must hold radix_temp_bytes(n) bytes.  vals and vals_alt may both be
// nullptr to sort keys alone.
size_t radix_temp_bytes(int64_t n);
cudaError_t radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_alt, uint32_t* vals_alt, int64_t n,
                                 int nbits, bool* result_in_alt, void* temp, cudaStream_t s);

}  // namespace mlods
