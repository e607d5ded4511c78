// Shared device helpers for the B200 DMK library: complex FP64 arithmetic on
// double2, Morton keys, exact root-of-unity tables, error handling.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>

namespace pdmk {

constexpr int KEY_BITS = 21;   // Morton bits per axis (63-bit keys)
constexpr int MAX_LEVEL = 10;  // deepest level a node may be refined to
constexpr int MAX_LEVELS = MAX_LEVEL + 1;

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};

// a device-side error word was set (a bounded wait in a kernel gave up)
struct DeviceError : std::runtime_error {
  explicit DeviceError(const std::string& s) : std::runtime_error(s) {}
};

// invalid caller data found on the device (positions outside [0, L), charges not finite)
struct BadInput : std::runtime_error {
  explicit BadInput(const std::string& s) : std::runtime_error(s) {}
};

#define PDMK_CUDA(call)                                                                               \
  do {                                                                                                \
    cudaError_t err__ = (call);                                                                       \
    if (err__ != cudaSuccess)                                                                         \
      throw ::pdmk::CudaError(std::string(#call) + ": " + cudaGetErrorString(err__) + " at " + __FILE__ + \
                              ":" + std::to_string(__LINE__));                                        \
  } while (0)

// kernels this library has launched (graph-executed ones included)
inline std::atomic<long long> g_launch_count{0};

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes`. The attribute belongs to the function in the current
// device's context, so the limit already set is remembered per (function,
// device); it only ever grows, under a lock (trees may be driven from several
// host threads and live on different devices).
inline void raise_smem_limit(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<const void*, int>, size_t> set;
  int dev = 0;
  PDMK_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> g(mu);
  size_t& limit = set[{func, dev}];
  if (bytes > limit) {
    PDMK_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes)));
    limit = bytes;
  }
}

#define PDMK_LAUNCH_CHECK()                                  \
  do {                                                       \
    PDMK_CUDA(cudaGetLastError());                           \
    ::pdmk::g_launch_count.fetch_add(1, std::memory_order_relaxed); \
  } while (0)

// ---------------------------------------------------------------------------
// complex FP64 on double2
__host__ __device__ inline double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__host__ __device__ inline double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__host__ __device__ inline double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ inline double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ inline double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }

// ---------------------------------------------------------------------------
// Morton keys: bit 3j = x_j, 3j+1 = y_j, 3j+2 = z_j; child digit = x | y<<1 | z<<2
__host__ __device__ inline uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffff;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}
__host__ __device__ inline uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ULL;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ULL;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00fULL;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffULL;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffULL;
  x = (x ^ (x >> 32)) & 0x1fffffULL;
  return static_cast<uint32_t>(x);
}
__host__ __device__ inline uint64_t morton3(uint32_t ix, uint32_t iy, uint32_t iz) {
  return spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
}
// integer grid coordinate of x in [0, L) at 2^21 cells per axis (floor of x/L*2^21)
__host__ __device__ inline uint32_t grid_coord(double x, double L) {
  double s = floor((x / L) * 2097152.0);
  if (s < 0) s = 0;
  if (s > 2097151.0) s = 2097151.0;
  return static_cast<uint32_t>(s);
}

// my_mod of the reference (include/utils.hpp:96-105): wrap into [0, L)
__host__ __device__ inline double wrap_mod(double x, double L) {
  // bounded: inputs are finite and |dx| < 64 L is enforced by the callers
  for (int it = 0; it < 130 && x < 0; ++it) x += L;
  for (int it = 0; it < 130 && x >= L; ++it) x -= L;
  return x;
}

// exact sixth roots of unity w^m = exp(i pi m / 3), m mod 6
__host__ __device__ inline double2 root6(int m) {
  m %= 6;
  if (m < 0) m += 6;
  const double h = 0.86602540378443864676;  // sqrt(3)/2
  switch (m) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.5, h);
    case 2: return make_double2(-0.5, h);
    case 3: return make_double2(-1.0, 0.0);
    case 4: return make_double2(-0.5, -h);
    default: return make_double2(0.5, -h);
  }
}

__host__ __device__ inline int ceil_div(int a, int b) { return (a + b - 1) / b; }

}  // namespace pdmk
