// Exclusive scan (one launch up to 4096 items, else reduce-then-scan in three
// launches) and stable LSD radix sort with 8-bit digits (tile histogram ->
// digit-major scan -> stable warp-multisplit scatter). Used to bin particles
// by Morton key.
#include "common.cuh"
#include "sort.cuh"

namespace pdmk {
namespace {

constexpr int SCAN_T = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_T * SCAN_ITEMS;

__device__ inline int block_exclusive_scan_1024(int v, int* smem32, int* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = v;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) smem32[warp] = x;
  __syncthreads();
  if (warp == 0) {
    int w = lane < (blockDim.x >> 5) ? smem32[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      int y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    smem32[lane] = w;  // inclusive warp prefix
  }
  __syncthreads();
  int warp_off = warp > 0 ? smem32[warp - 1] : 0;
  if (total) *total = smem32[(blockDim.x >> 5) - 1];
  return warp_off + x - v;
}

__global__ void k_block_sums(const int* in, long n, int* bsum) {
  long base = long(blockIdx.x) * SCAN_TILE;
  int s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    long i = base + long(threadIdx.x) * SCAN_ITEMS + k;
    if (i < n) s += in[i];
  }
  __shared__ int sm[32];
  int tot;
  block_exclusive_scan_1024(s, sm, &tot);
  if (threadIdx.x == 0) bsum[blockIdx.x] = tot;
}

__global__ void k_scan_single(int* a, int n) {
  __shared__ int sm[32];
  int v[SCAN_ITEMS];
  int s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int i = threadIdx.x * SCAN_ITEMS + k;
    v[k] = i < n ? a[i] : 0;
    s += v[k];
  }
  int off = block_exclusive_scan_1024(s, sm, nullptr);
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int i = threadIdx.x * SCAN_ITEMS + k;
    if (i < n) a[i] = off;
    off += v[k];
  }
}

__global__ void k_scan_apply(const int* in, int* out, long n, const int* bsum) {
  __shared__ int sm[32];
  long base = long(blockIdx.x) * SCAN_TILE;
  int v[SCAN_ITEMS];
  int s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    long i = base + long(threadIdx.x) * SCAN_ITEMS + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  __syncthreads();  // in and out may alias: all loads before any store
  int off = block_exclusive_scan_1024(s, sm, nullptr) + bsum[blockIdx.x];
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    long i = base + long(threadIdx.x) * SCAN_ITEMS + k;
    if (i < n) out[i] = off;
    off += v[k];
  }
}

// one tile (n <= SCAN_TILE): the whole scan in one block
__global__ void k_scan_one(const int* in, int* out, int n) {
  __shared__ int sm[32];
  int v[SCAN_ITEMS];
  int s = 0;
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int i = threadIdx.x * SCAN_ITEMS + k;
    v[k] = i < n ? in[i] : 0;
    s += v[k];
  }
  __syncthreads();  // in and out may alias: all loads before any store
  int off = block_exclusive_scan_1024(s, sm, nullptr);
  for (int k = 0; k < SCAN_ITEMS; ++k) {
    int i = threadIdx.x * SCAN_ITEMS + k;
    if (i < n) out[i] = off;
    off += v[k];
  }
}

// ---------------------------------------------------------------------------
constexpr int RS_T = 256;       // threads per tile
constexpr int RS_ITEMS = 8;     // items per thread
constexpr int RS_TILE = RS_T * RS_ITEMS;
constexpr int RS_WARPS = RS_T / 32;

__global__ void k_radix_hist(const uint64_t* keys, long n, int shift, int ntiles, int* hist) {
  __shared__ int h[256];
  for (int i = threadIdx.x; i < 256; i += RS_T) h[i] = 0;
  __syncthreads();
  long base = long(blockIdx.x) * RS_TILE;
  for (int k = 0; k < RS_ITEMS; ++k) {
    long i = base + k * RS_T + threadIdx.x;
    if (i < n) atomicAdd(&h[int((keys[i] >> shift) & 0xff)], 1);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += RS_T) hist[long(d) * ntiles + blockIdx.x] = h[d];
}

__global__ void k_radix_scatter(const uint64_t* kin, const int* vin, uint64_t* kout, int* vout, long n, int shift,
                                int ntiles, const int* offs) {
  __shared__ int wh[RS_WARPS][256];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < RS_WARPS * 256; i += RS_T) (&wh[0][0])[i] = 0;
  __syncthreads();
  // warp w owns tile elements [w*256, w*256+256), visited in rounds of 32
  const long wbase = long(blockIdx.x) * RS_TILE + long(warp) * 32 * RS_ITEMS;
  uint64_t key[RS_ITEMS];
  int val[RS_ITEMS], dig[RS_ITEMS], pos[RS_ITEMS];
  const unsigned lt = (1u << lane) - 1u;
  for (int k = 0; k < RS_ITEMS; ++k) {
    long i = wbase + k * 32 + lane;
    bool ok = i < n;
    key[k] = ok ? kin[i] : 0;
    val[k] = ok ? vin[i] : 0;
    int d = ok ? int((key[k] >> shift) & 0xff) : 256 + lane;  // out-of-range items form singleton groups
    dig[k] = d;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int rank = __popc(peers & lt);
    int before = ok ? wh[warp][d] : 0;
    __syncwarp();
    pos[k] = before + rank;
    int leader = __ffs(peers) - 1;
    if (ok && lane == leader) wh[warp][d] = before + __popc(peers);
    __syncwarp();
  }
  __syncthreads();
  // per digit, exclusive prefix over warps (warp order = element order)
  for (int d = threadIdx.x; d < 256; d += RS_T) {
    int s = 0;
    for (int w = 0; w < RS_WARPS; ++w) {
      int c = wh[w][d];
      wh[w][d] = s;
      s += c;
    }
  }
  __syncthreads();
  for (int k = 0; k < RS_ITEMS; ++k) {
    long i = wbase + k * 32 + lane;
    if (i < n) {
      int d = dig[k];
      long dst = long(offs[long(d) * ntiles + blockIdx.x]) + wh[warp][d] + pos[k];
      kout[dst] = key[k];
      vout[dst] = val[k];
    }
  }
}

}  // namespace

size_t scan_scratch_bytes(long n) {
  long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  return size_t(nb + 1) * sizeof(int) + 256;
}

void exclusive_scan(const int* in, int* out, long n, void* scratch, cudaStream_t st) {
  if (n <= 0) return;
  long nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  if (nb > SCAN_TILE) throw std::invalid_argument("exclusive_scan: input too long");
  if (nb == 1) {
    k_scan_one<<<1, SCAN_T, 0, st>>>(in, out, int(n));
    PDMK_LAUNCH_CHECK();
    return;
  }
  int* bsum = static_cast<int*>(scratch);
  k_block_sums<<<unsigned(nb), SCAN_T, 0, st>>>(in, n, bsum);
  PDMK_LAUNCH_CHECK();
  k_scan_single<<<1, SCAN_T, 0, st>>>(bsum, int(nb));
  PDMK_LAUNCH_CHECK();
  k_scan_apply<<<unsigned(nb), SCAN_T, 0, st>>>(in, out, n, bsum);
  PDMK_LAUNCH_CHECK();
}

size_t radix_sort_scratch_bytes(long n) {
  long ntiles = (n + RS_TILE - 1) / RS_TILE;
  long hist = 256 * ntiles;
  size_t b = size_t(n) * (sizeof(uint64_t) + sizeof(int)) + 256;
  b += size_t(hist) * sizeof(int) + 256;
  b += scan_scratch_bytes(hist);
  return b;
}

void radix_sort_pairs(uint64_t* keys, int* vals, long n, int passes, void* scratch, cudaStream_t st) {
  if (n <= 1) return;
  long ntiles = (n + RS_TILE - 1) / RS_TILE;
  char* p = static_cast<char*>(scratch);
  uint64_t* k2 = reinterpret_cast<uint64_t*>(p);
  p += ((size_t(n) * sizeof(uint64_t) + 255) / 256) * 256;
  int* v2 = reinterpret_cast<int*>(p);
  p += ((size_t(n) * sizeof(int) + 255) / 256) * 256;
  int* hist = reinterpret_cast<int*>(p);
  p += ((size_t(256 * ntiles) * sizeof(int) + 255) / 256) * 256;
  void* sscr = p;
  uint64_t *ka = keys, *kb = k2;
  int *va = vals, *vb = v2;
  for (int pass = 0; pass < passes; ++pass) {
    int shift = 8 * pass;
    k_radix_hist<<<unsigned(ntiles), RS_T, 0, st>>>(ka, n, shift, int(ntiles), hist);
    PDMK_LAUNCH_CHECK();
    exclusive_scan(hist, hist, 256 * ntiles, sscr, st);
    k_radix_scatter<<<unsigned(ntiles), RS_T, 0, st>>>(ka, va, kb, vb, n, shift, int(ntiles), hist);
    PDMK_LAUNCH_CHECK();
    std::swap(ka, kb);
    std::swap(va, vb);
  }
  if (ka != keys) {
    PDMK_CUDA(cudaMemcpyAsync(keys, ka, size_t(n) * sizeof(uint64_t), cudaMemcpyDeviceToDevice, st));
    PDMK_CUDA(cudaMemcpyAsync(vals, va, size_t(n) * sizeof(int), cudaMemcpyDeviceToDevice, st));
  }
}

}  // namespace pdmk
