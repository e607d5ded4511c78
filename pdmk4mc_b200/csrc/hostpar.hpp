// Host-side helpers for large caller arrays: a chunked parallel loop over
// [0, n) on a few std::threads, and a pinned staging buffer per device for
// host-to-device copies of inputs (a copy from pageable memory runs at a
// fraction of the link rate; the staged copy is a parallel memcpy into
// page-locked memory and one DMA).
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <thread>
#include <vector>

namespace pdmk {

// f(begin, end) over [0, n) in up to `threads` contiguous pieces; runs
// inline below `serial_below` items
template <class F>
void parallel_chunks(long n, F f, long serial_below = 1 << 18, int threads = 8) {
  const int hw = int(std::max(1u, std::thread::hardware_concurrency()));
  const int t = int(std::min<long>(std::min(threads, hw), std::max<long>(1, n / std::max<long>(1, serial_below / 4))));
  if (n < serial_below || t <= 1) {
    f(0L, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(size_t(t) - 1);
  for (int k = 1; k < t; ++k) pool.emplace_back([&, k] { f(n * k / t, n * (k + 1) / t); });
  f(0L, n / t);
  for (auto& th : pool) th.join();
}

// one host piece of a staged copy
struct HostPiece {
  const void* src;
  size_t bytes;
};

// Copies the pieces, back to back, from host memory to device memory at dst
// on stream st through the current device's pinned staging buffer; the copy
// has been handed to the DMA engine when this returns, and the staging
// buffer is reused only after that copy has completed. Small copies go
// straight from the caller's memory.
void staged_h2d(void* dst, const std::vector<HostPiece>& pieces, cudaStream_t st);

}  // namespace pdmk
