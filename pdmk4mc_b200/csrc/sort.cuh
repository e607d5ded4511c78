// Device-wide exclusive scan and stable LSD radix sort of (uint64 key,
// int32 value) pairs: the binning primitives of the tree build.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace pdmk {

// scratch bytes needed by exclusive_scan for n elements
size_t scan_scratch_bytes(long n);
// out[i] = sum_{j<i} in[i]; in and out may alias. n <= 16M.
void exclusive_scan(const int* in, int* out, long n, void* scratch, cudaStream_t st);
// same for 64-bit element sums of int inputs
size_t radix_sort_scratch_bytes(long n);
// stable sort by key over key bits [0, 8*passes); keys/vals are sorted in
// place (an equal-sized alternate buffer lives in scratch)
void radix_sort_pairs(uint64_t* keys, int* vals, long n, int passes, void* scratch, cudaStream_t st);

}  // namespace pdmk
