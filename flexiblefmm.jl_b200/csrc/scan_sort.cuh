// Device prefix sums and radix sort (scan_sort.cu).
#pragma once
#include "common.cuh"

namespace fmmb {

// out[i] = Σ_{j<i} in[j]; in and out may alias. Synchronises the stream.
void scan_exclusive(const int* in, int* out, int64_t n, cudaStream_t s);
// the same, returning the total (reads two entries back)
int64_t scan_exclusive_total(const int* in, int* out, int64_t n, cudaStream_t s);
// stable sort of (keys, vals) by the low `bits` bits of the keys, in place
void radix_sort_pairs(uint64_t* keys, uint32_t* vals, int64_t n, int bits, cudaStream_t s);

}  // namespace fmmb
