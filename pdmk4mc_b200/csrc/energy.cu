// Full-energy kernels (FP64): the plane-wave upward pass, incoming
// expansions, window / difference / residual energies.
//
// Reference counterparts: outgoing_pw_root / outgoing_pw_direct and
// nudft3d1_halfplane (src/planewave.cpp:24-84, include/nudft.hpp:66-123),
// form_incoming_pw (src/planewave.cpp:99-155), eval_energy_window /
// eval_energy_diff / eval_energy_res (src/energy.cpp:21-173).
//
// The outgoing expansion of a box, rho_B(k) = sum_j q_j exp(-i k.x_j) over
// the half grid kz <= 0, is evaluated as the complex contraction
//   out[(kz,ky), kx] = sum_j (q_j ez_j[kz] ey_j[ky]) ex_j[kx]
// with box-centred coordinates: exp(-i k.x) = exp(-i k.c_B) exp(-i k.(x-c_B)),
// where k.c_B is an exact multiple of pi/3 (k = m dk_l, dk_l bs_l = 2 pi / 3),
// so the decentring factor is an exact sixth root of unity per axis. A table
// pass writes each work item's per-particle factors ex, ey, ez to HBM once;
// the contraction streams them chunk by chunk into shared memory.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "common.cuh"
#include "mixed.hpp"
#include "tree.hpp"

namespace pdmk {
namespace {

constexpr int TPB = 256;
inline unsigned grid_for(long n, int tpb = TPB) { return unsigned(std::max<long>(1, (n + tpb - 1) / tpb)); }

__device__ inline double block_sum(double v, double* sm) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __syncthreads();
  if (lane == 0) sm[warp] = v;
  __syncthreads();
  double s = 0;
  if (threadIdx.x == 0)
    for (int w = 0; w < nw; ++w) s += sm[w];
  return s;  // valid in thread 0
}

// ---------------------------------------------------------------------------
// NUDFT work item: one row tile of one box over one slot range
struct NudftWork {
  double cx, cy, cz;  // box centre
  double dk;
  int X, Y, Z;        // integer box coordinates at its level
  int M;              // decentring multiplier: 1 for levels >= 2, 3 for the root
  int s_begin, s_end;
  int row_tile;
  int pad_;
  double2* out;       // H complex outputs of this box (or of this split-K chunk)
  const double2* tab; // factor tables of this item's particle chunks (shared by its row tiles)
};

// Each thread owns one (kz, ky) row and TC <= 20 of its kx columns: 4 TC FP64
// accumulators stay in registers (wider tiles spill), and the row factor
// q ez ey costs one complex multiply per TC multiply-adds.
template <int NK>
struct NudftShape {
  static constexpr int D = 2 * NK + 1;
  static constexpr int CG = (D + 19) / 20;            // column groups per row
  static constexpr int TC = (D + CG - 1) / CG;        // columns per thread
  static constexpr int DP = TC * CG;                  // padded row stride in smem
  static constexpr int ROWS = (NK + 1) * D;
  static constexpr int WORK = ROWS * CG;              // thread tasks per box
  static constexpr int TMAX = 512;
  static constexpr int TILES = (WORK + TMAX - 1) / TMAX;
  static constexpr int THREADS = ((WORK + TILES - 1) / TILES + 31) / 32 * 32;
  // particles per shared-memory chunk: 32, or 16 when 32 would not fit
  static constexpr int KC = 2 * 32 * (2 * DP + NK + 1) * 16 > 200 * 1024 ? 16 : 32;
  static constexpr int SMEM = 2 * KC * (2 * DP + NK + 1) * int(sizeof(double2));  // double-buffered
};

// per-axis factors exp(-i m dk (x - c)) * w6^{-M (2X+1) m}, m = m0 .. m0+cnt-1.
// The six chains m = m0 + r + 6 i each keep one root of unity, so they step
// by exp(-6 i dk (x - c)) with the root applied once per chain: a dependency
// chain of about cnt / 6 complex products instead of 2 cnt.
__device__ inline void axis_factors(double xr, double dk, int M, int X, int m0, int cnt, double scale, double2* dst) {
  const double th = dk * xr;
  double s, c;
  sincos(-double(m0) * th, &s, &c);
  const double2 v0 = make_double2(c * scale, s * scale);
  sincos(-th, &s, &c);
  const double2 st = make_double2(c, s);
  const double2 st2 = cmul(st, st), st3 = cmul(st2, st), st6 = cmul(st3, st3);
  const int dec = M * (2 * X + 1);
  double2 v[6];
  v[0] = v0;
  v[1] = cmul(v0, st);
  v[2] = cmul(v0, st2);
  v[3] = cmul(v0, st3);
  v[4] = cmul(v[1], st3);
  v[5] = cmul(v[2], st3);
#pragma unroll
  for (int r = 0; r < 6; ++r) v[r] = cmul(v[r], root6(-dec * (m0 + r)));
  for (int t = 0; t < cnt; t += 6) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (t + r < cnt) {
        dst[t + r] = v[r];
        v[r] = cmul(v[r], st6);
      }
    }
  }
}

// Factor tables of one particle chunk of a work item, in shared memory:
// ex [KC][DP], ey [KC][DP], ez [KC][NK+1] (charge folded into ez), rows past
// the item's last particle and the padding columns D .. DP-1 zero. Tasks are
// (particle, axis, half) so that each recurrence chain covers half an axis.
template <int NK>
__device__ void nudft_build(const NudftWork& w, int base, double2* buf, const double* __restrict__ sx,
                            const double* __restrict__ sy, const double* __restrict__ sz,
                            const double* __restrict__ sq) {
  using S = NudftShape<NK>;
  double2* ex = buf;
  double2* ey = ex + S::KC * S::DP;
  double2* ez = ey + S::KC * S::DP;
  const int nk = min(S::KC, w.s_end - base);
  for (int t = threadIdx.x; t < S::KC * 6; t += blockDim.x) {
    int j = t / 6, a = (t / 2) % 3, half = t & 1;
    if (j >= nk) {
      double2* dst = a == 0 ? ex + j * S::DP : (a == 1 ? ey + j * S::DP : ez + j * (NK + 1));
      int len = a == 2 ? NK + 1 : S::DP;
      for (int u = half; u < len; u += 2) dst[u] = make_double2(0.0, 0.0);
      continue;
    }
    int s = base + j;
    if (a == 0) {
      int h = (S::D + 1) / 2;
      int m0 = half ? -NK + h : -NK, cnt = half ? S::D - h : h;
      axis_factors(sx[s] - w.cx, w.dk, w.M, w.X, m0, cnt, 1.0, ex + j * S::DP + (m0 + NK));
      if (half)
        for (int u = S::D; u < S::DP; ++u) ex[j * S::DP + u] = make_double2(0.0, 0.0);
    } else if (a == 1) {
      int h = (S::D + 1) / 2;
      int m0 = half ? -NK + h : -NK, cnt = half ? S::D - h : h;
      axis_factors(sy[s] - w.cy, w.dk, w.M, w.Y, m0, cnt, 1.0, ey + j * S::DP + (m0 + NK));
    } else {
      int h = (NK + 2) / 2;
      int m0 = half ? -NK + h : -NK, cnt = half ? NK + 1 - h : h;
      axis_factors(sz[s] - w.cz, w.dk, w.M, w.Z, m0, cnt, sq[s], ez + j * (NK + 1) + (m0 + NK));
    }
  }
}

// Table pass: one block per (item, particle chunk) builds the chunk's tables
// in shared memory and writes them to the item's table range in HBM with
// coalesced stores, once for all row tiles of the item.
template <int NK>
__global__ void __launch_bounds__(NudftShape<NK>::KC * 6)
    k_nudft_tables(const NudftWork* __restrict__ work, const int2* __restrict__ chunks, const double* __restrict__ sx,
                   const double* __restrict__ sy, const double* __restrict__ sz, const double* __restrict__ sq) {
  using S = NudftShape<NK>;
  constexpr int BUF = S::KC * (2 * S::DP + NK + 1);
  extern __shared__ double2 smem[];
  const int2 ch = chunks[blockIdx.x];
  const NudftWork w = work[ch.x];
  nudft_build<NK>(w, w.s_begin + ch.y * S::KC, smem, sx, sy, sz, sq);
  __syncthreads();
  double2* dst = const_cast<double2*>(w.tab) + size_t(ch.y) * BUF;
  for (int i = threadIdx.x; i < BUF; i += blockDim.x) dst[i] = smem[i];
}

__device__ inline void cp_async16(void* smem_dst, const void* gmem_src) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem_dst));
  const size_t g = __cvta_generic_to_global(gmem_src);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(g) : "memory");
}
__device__ inline void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ inline void cp_async_wait_prior() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

// Contraction pass: one (item, row tile) per block. The chunk tables stream
// from HBM into two shared-memory buffers by asynchronous copies issued a
// chunk ahead, so every thread does the same work between two barriers.
template <int NK>
__global__ void __launch_bounds__(NudftShape<NK>::THREADS) k_nudft(const NudftWork* __restrict__ work) {
  using S = NudftShape<NK>;
  constexpr int BUF = S::KC * (2 * S::DP + NK + 1);  // complex entries per table buffer
  extern __shared__ double2 smem[];
  const NudftWork w = work[blockIdx.x];
  const int g = w.row_tile * S::THREADS + threadIdx.x;
  const bool active = g < S::WORK;
  const int row = active ? g / S::CG : 0;
  const int cg = active ? g % S::CG : 0;
  const int kz = row / S::D, ky = row % S::D;
  const int c0 = cg * S::TC;
  const int nch = (w.s_end - w.s_begin + S::KC - 1) / S::KC;
  auto fetch = [&](int c) {
    const double2* src = w.tab + size_t(c) * BUF;
    double2* dst = smem + (c & 1) * BUF;
    for (int i = threadIdx.x; i < BUF; i += blockDim.x) cp_async16(dst + i, src + i);
  };
  double2 acc[S::TC];
#pragma unroll
  for (int c = 0; c < S::TC; ++c) acc[c] = make_double2(0.0, 0.0);
  if (nch > 0) fetch(0);
  cp_async_commit();
  for (int ci = 0; ci < nch; ++ci) {
    // the next chunk's copies go out before this chunk is contracted (its
    // buffer was last read before the previous iteration's closing barrier)
    if (ci + 1 < nch) fetch(ci + 1);
    cp_async_commit();
    cp_async_wait_prior();  // everything but the group just committed has landed
    __syncthreads();
    const double2* ex = smem + (ci & 1) * BUF;
    const double2* ey = ex + S::KC * S::DP;
    const double2* ez = ey + S::KC * S::DP;
    const int nk = min(S::KC, w.s_end - (w.s_begin + ci * S::KC));
    if (active) {
#pragma unroll 1
      for (int j = 0; j < nk; ++j) {
        const double2 a = cmul(ez[j * (NK + 1) + kz], ey[j * S::DP + ky]);
        const double2* xr = ex + j * S::DP + c0;
        // one shared-memory load per column feeds its four FMAs; the 2 TC
        // accumulator chains give enough independent work to hide latency
#pragma unroll
        for (int c = 0; c < S::TC; ++c) {
          const double2 b = xr[c];
          acc[c].x = fma(a.x, b.x, acc[c].x);
          acc[c].y = fma(a.x, b.y, acc[c].y);
          acc[c].x = fma(-a.y, b.y, acc[c].x);
          acc[c].y = fma(a.y, b.x, acc[c].y);
        }
      }
    }
    __syncthreads();
  }
  if (active) {
    double2* o = w.out + size_t(row) * S::D + c0;
#pragma unroll
    for (int c = 0; c < S::TC; ++c)
      if (c0 + c < S::D) o[c] = acc[c];
  }
}

template <int NK>
void launch_nudft(const NudftWork* d_work, int nwork, const int2* d_chunks, int nchunks, const DevTree& T,
                  cudaStream_t st) {
  using S = NudftShape<NK>;
  constexpr int TAB_SMEM = S::KC * (2 * S::DP + NK + 1) * int(sizeof(double2));
  if (nwork == 0) return;
  // per device and thread-safe: replica energies call this from several host threads
  raise_smem_limit(reinterpret_cast<const void*>(k_nudft<NK>), S::SMEM);
  raise_smem_limit(reinterpret_cast<const void*>(k_nudft_tables<NK>), TAB_SMEM);
  if (nchunks > 0) {
    k_nudft_tables<NK><<<unsigned(nchunks), S::KC * 6, TAB_SMEM, st>>>(d_work, d_chunks, T.sx, T.sy, T.sz, T.sq);
    PDMK_LAUNCH_CHECK();
  }
  k_nudft<NK><<<unsigned(nwork), S::THREADS, S::SMEM, st>>>(d_work);
  PDMK_LAUNCH_CHECK();
}

struct NudftInfo {
  int tiles, kc, buf;  // row tiles per item, particles per chunk, complex entries per chunk table
};

template <int NK>
NudftInfo nudft_info_of() {
  using S = NudftShape<NK>;
  return {S::TILES, S::KC, S::KC * (2 * S::DP + NK + 1)};
}

NudftInfo nudft_info(int nk) {
  switch (nk) {
    case 4: return nudft_info_of<4>();
    case 6: return nudft_info_of<6>();
    case 8: return nudft_info_of<8>();
    case 12: return nudft_info_of<12>();
    case 13: return nudft_info_of<13>();
    case 17: return nudft_info_of<17>();
    case 19: return nudft_info_of<19>();
    case 26: return nudft_info_of<26>();
    case 32: return nudft_info_of<32>();  // Ewald structure factor, level 2
    case 64: return nudft_info_of<64>();  // Ewald structure factor, level 3
    default: throw std::invalid_argument("unsupported mode count");
  }
}

int nudft_tiles(int nk) { return nudft_info(nk).tiles; }

// Lays out the factor tables of a work list whose items are runs of `tiles`
// consecutive entries (row tiles 0 .. tiles-1 of one box or chunk): each item
// gets ceil(n / KC) chunk tables, allocated here stream-ordered on `st`, and
// the list of (first entry, chunk) pairs the table pass runs over. The caller
// frees `tables` stream-ordered after the contraction.
void plan_nudft_tables(int nk, std::vector<NudftWork>& wl, double2** tables, std::vector<int2>& chunks,
                       cudaStream_t st) {
  const NudftInfo in = nudft_info(nk);
  size_t nchunk = 0;
  for (size_t e = 0; e < wl.size(); e += in.tiles) {
    if (wl[e].row_tile != 0) throw std::logic_error("NUDFT work list: items must start at row tile 0");
    nchunk += size_t((wl[e].s_end - wl[e].s_begin + in.kc - 1) / in.kc);
  }
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(tables), sizeof(double2) * size_t(in.buf) * std::max<size_t>(nchunk, 1),
                            st));
  chunks.clear();
  chunks.reserve(nchunk);
  size_t c = 0;
  for (size_t e = 0; e < wl.size(); e += in.tiles) {
    const int n = (wl[e].s_end - wl[e].s_begin + in.kc - 1) / in.kc;
    for (int t = 0; t < in.tiles && e + t < wl.size(); ++t) wl[e + t].tab = *tables + c * size_t(in.buf);
    for (int k = 0; k < n; ++k) chunks.push_back(make_int2(int(e), k));
    c += size_t(n);
  }
}

void dispatch_nudft(int nk, const NudftWork* d_work, int nwork, const int2* d_chunks, int nchunks, const DevTree& T,
                    cudaStream_t st) {
  switch (nk) {
    case 4: launch_nudft<4>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 6: launch_nudft<6>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 8: launch_nudft<8>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 12: launch_nudft<12>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 13: launch_nudft<13>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 17: launch_nudft<17>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 19: launch_nudft<19>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 26: launch_nudft<26>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 32: launch_nudft<32>(d_work, nwork, d_chunks, nchunks, T, st); break;
    case 64: launch_nudft<64>(d_work, nwork, d_chunks, nchunks, T, st); break;
    default: throw std::invalid_argument("unsupported mode count");
  }
}

// sum split-K chunk partials of box b into its output, in chunk order
__global__ void k_reduce_chunks(const double2* part, const int* chunk_first, const int* chunk_n, double2* const* outs,
                                int H) {
  int b = blockIdx.y;
  int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= H) return;
  const double2* p = part + size_t(chunk_first[b]) * H + k;
  double2 s = make_double2(0, 0);
  for (int c = 0; c < chunk_n[b]; ++c) s = cadd(s, p[size_t(c) * H]);
  outs[b][k] = s;
}

// ---------------------------------------------------------------------------
// inc_B = conj(out_B) + sum_C conj(out_C * exp(-i k.p L)) over B's 26
// colleagues C (form_incoming_pw, src/planewave.cpp:99-155), for the
// 4 x 4 x 4 boxes of level l below one box G of level l - 2 at once: their
// 27-box neighbourhoods lie in the 6 x 6 x 6 cube of level-l cells around
// them. A block stages the cube's outgoing rows for one tile of INC_KT modes
// in shared memory (image phase applied; absent and empty cells are zero),
// then each thread sums the 3 x 3 (y, z) neighbourhood of six x columns once
// and slides the 3-wide x window over them for its 4 receivers. A row tile
// crosses L2 216 / 64 = 3.4 times per receiving box (8 times with the
// 4 x 4 x 4 cube around one parent). The energy partial of a block sums its
// non-leaf receivers, which share one level.
constexpr int INC_KT = 16;    // modes per tile
constexpr int INC_T = 256;    // threads: INC_KT modes x 16 (y, z) lines of 4 receivers along x
constexpr int INC_CELLS = 216;
constexpr size_t INC_SMEM = sizeof(double2) * INC_CELLS * INC_KT + sizeof(int) * (INC_CELLS + 64) + INC_CELLS;

// rank of a refined cell within its level (Morton order)
__device__ inline int refined_rank(const DevTree& T, int level, uint64_t cell) {
  const uint32_t w = T.bm_d[level][cell >> 5];
  return T.wprefix_d[level][cell >> 5] + __popc(w & ((1u << (cell & 31)) - 1u));
}

// Grid: ncubes x slots blocks; block (slot, c) handles the tiles slot,
// slot + slots, ... of cube c, so its set-up (the cube's cell lookup) is
// paid once, and the cubes sharing a slot walk the same tiles together (the
// cells two neighbouring cubes share meet in L2).
template <int NK>
__global__ void __launch_bounds__(INC_T, 2) k_incoming_cube(DevTree T, const int* __restrict__ cubes, int ncubes,
                                                             int slots, double* part) {
  constexpr int D = 2 * NK + 1, H = (NK + 1) * D * D;
  extern __shared__ double2 w[];                             // [INC_CELLS][INC_KT]
  int* s_row = reinterpret_cast<int*>(w + INC_CELLS * INC_KT);  // outgoing row of each cell, -1: absent or empty
  int* s_recv = s_row + INC_CELLS;                           // expansion row of each receiver, -1: none
  unsigned char* s_wrap = reinterpret_cast<unsigned char*>(s_recv + 64);  // image flags, 2 bits per axis
  __shared__ double sm[32];
  const int slot = blockIdx.x / ncubes, cb = blockIdx.x % ncubes;
  const int G = cubes[cb];
  const int l = T.node_level[G] + 2;
  const int side = 1 << l;
  const uint64_t gp = T.node_prefix[G];
  const int O[3] = {4 * int(compact3(gp)), 4 * int(compact3(gp >> 1)), 4 * int(compact3(gp >> 2))};
  const int base = T.pw_base;
  if (threadIdx.x < INC_CELLS) {
    const int t = threadIdx.x;
    const int c[3] = {t % 6 - 1, (t / 6) % 6 - 1, t / 36 - 1};
    int g[3];
    unsigned wrap = 0;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      int v = O[a] + c[a];
      const int f = v < 0 ? 1 : (v >= side ? 2 : 0);  // 1: image below (-1), 2: above (+1)
      v = f == 1 ? v + side : (f == 2 ? v - side : v);
      g[a] = v;
      wrap |= unsigned(f) << (2 * a);
    }
    const uint64_t m = morton3(uint32_t(g[0]), uint32_t(g[1]), uint32_t(g[2]));
    int node = -1;
    if ((T.bm_d[l - 1][m >> 8] >> ((m >> 3) & 31)) & 1u)
      node = T.level_start_d[l] + 8 * refined_rank(T, l - 1, m >> 3) + int(m & 7);
    s_row[t] = (node >= 0 && T.node_count[node] > 0) ? node - base : -1;
    s_wrap[t] = static_cast<unsigned char>(wrap);
    if (c[0] >= 0 && c[0] < 4 && c[1] >= 0 && c[1] < 4 && c[2] >= 0 && c[2] < 4)
      s_recv[c[0] + 4 * c[1] + 16 * c[2]] = (node >= 0 && T.node_child0[node] >= 0) ? node - base : -1;
  }
  __syncthreads();
  const int two_l = (l & 1) ? 2 : 1;
  const int kk = threadIdx.x % INC_KT;
  const int line = threadIdx.x / INC_KT, ry = line & 3, rz = line >> 2;
  const double2 w3a = make_double2(-0.5, -0.86602540378443864676);  // exp(-2 pi i / 3)
  const double2 w3b = make_double2(-0.5, 0.86602540378443864676);   // exp(-4 pi i / 3)
  double e = 0;
  constexpr int ktiles = (H + INC_KT - 1) / INC_KT;
  for (int tile = slot; tile < ktiles; tile += slots) {
    const int k = tile * INC_KT + kk;
    const bool kin = k < H;
    const int ix = k % D, iy = (k / D) % D, iz = k / (D * D);
    // the image phase is exp(-2 pi i e / 3) with e = sum over axes of
    // f (i - n) 2^l mod 3 (f = -1 below, +1 above): per axis the terms of
    // an image below and above, two bits each
    unsigned below = 0, above = 0;
    {
      const int ii[3] = {ix, iy, iz};
#pragma unroll
      for (int ax = 0; ax < 3; ++ax) {
        const int b = (((ii[ax] - NK) % 3 + 3) * two_l) % 3;
        above |= unsigned(b) << (2 * ax);
        below |= unsigned((3 - b) % 3) << (2 * ax);
      }
    }
    // stage the cube: mode kk of cells line, line + 16, ...; all loads issued
    // before the first is used
    constexpr int NPT = (INC_CELLS + INC_T / INC_KT - 1) / (INC_T / INC_KT);  // cells per thread
    double2 vv[NPT];
#pragma unroll
    for (int i = 0; i < NPT; ++i) {
      const int c = line + i * (INC_T / INC_KT);
      const int row = c < INC_CELLS ? s_row[c] : -1;
      vv[i] = (row >= 0 && kin) ? T.out[size_t(row) * H + k] : make_double2(0.0, 0.0);
    }
#pragma unroll
    for (int i = 0; i < NPT; ++i) {
      const int c = line + i * (INC_T / INC_KT);
      if (c >= INC_CELLS) break;
      double2 v = vv[i];
      const unsigned wr = s_wrap[c];
      if (wr) {
        unsigned ep = 0;
#pragma unroll
        for (int ax = 0; ax < 3; ++ax) {
          const unsigned f = (wr >> (2 * ax)) & 3u;
          ep += f == 1 ? (below >> (2 * ax)) & 3u : (f == 2 ? (above >> (2 * ax)) & 3u : 0u);
        }
        ep = ep >= 3 ? ep - 3 : ep;
        ep = ep >= 3 ? ep - 3 : ep;
        if (ep) v = cmul(v, ep == 1 ? w3a : w3b);
      }
      w[c * INC_KT + kk] = v;
    }
    __syncthreads();
    // the 3 x 3 (y, z) sums of the six x columns of this thread's line
    double2 col[6];
#pragma unroll
    for (int cx = 0; cx < 6; ++cx) {
      double2 acc = make_double2(0.0, 0.0);
#pragma unroll
      for (int dz = 0; dz < 3; ++dz)
#pragma unroll
        for (int dy = 0; dy < 3; ++dy) acc = cadd(acc, w[((rz + dz) * 36 + (ry + dy) * 6 + cx) * INC_KT + kk]);
      col[cx] = acc;
    }
    if (kin) {
      const double d2 = T.D2[k];
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const int rrow = s_recv[x + 4 * ry + 16 * rz];
        if (rrow < 0) continue;
        const double2 inc = cconj(cadd(cadd(col[x], col[x + 1]), col[x + 2]));
        T.inc[size_t(rrow) * H + k] = inc;
        const double2 o = w[((rz + 1) * 36 + (ry + 1) * 6 + x + 1) * INC_KT + kk];  // the receiver's own row
        e += (o.x * inc.x - o.y * inc.y) * d2;
      }
    }
    __syncthreads();
  }
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

template <int NK>
void launch_incoming_nk(const DevTree& D, const int* cubes, int ncubes, int slots, double* part, cudaStream_t st) {
  raise_smem_limit(reinterpret_cast<const void*>(k_incoming_cube<NK>), INC_SMEM);
  k_incoming_cube<NK><<<unsigned(slots * ncubes), INC_T, INC_SMEM, st>>>(D, cubes, ncubes, slots, part);
  PDMK_LAUNCH_CHECK();
}

void launch_incoming(const DevTree& D, const int* cubes, int ncubes, int slots, double* part, cudaStream_t st) {
  switch (D.n_diff) {
    case 4: launch_incoming_nk<4>(D, cubes, ncubes, slots, part, st); break;
    case 6: launch_incoming_nk<6>(D, cubes, ncubes, slots, part, st); break;
    case 8: launch_incoming_nk<8>(D, cubes, ncubes, slots, part, st); break;
    case 12: launch_incoming_nk<12>(D, cubes, ncubes, slots, part, st); break;
    case 13: launch_incoming_nk<13>(D, cubes, ncubes, slots, part, st); break;
    case 17: launch_incoming_nk<17>(D, cubes, ncubes, slots, part, st); break;
    case 19: launch_incoming_nk<19>(D, cubes, ncubes, slots, part, st); break;
    case 26: launch_incoming_nk<26>(D, cubes, ncubes, slots, part, st); break;
    default: throw std::invalid_argument("incoming pass: unsupported mode count");
  }
}

// E_diff from the cube-tiled partials: sum over cubes C_l dscale_l
// sum_slots part, minus sum over non-leaf boxes Q_B S_l
__global__ void k_diff_finish_cube(DevTree T, const int* __restrict__ cubes, int ncubes, int slots,
                                   const double* part, const int* __restrict__ boxes, int nboxes, const double* q2,
                                   const double* Cl, const double* Sl, double* out) {
  __shared__ double sm[32];
  double e = 0;
  for (int c = threadIdx.x; c < ncubes; c += blockDim.x) {
    const int l = T.node_level[cubes[c]] + 2;
    double t = 0;
    for (int sl = 0; sl < slots; ++sl) t += part[size_t(sl) * ncubes + c];
    e += Cl[l] * level_dscale(l) * t;
  }
  for (int b = threadIdx.x; b < nboxes; b += blockDim.x) e -= q2[b] * Sl[T.node_level[boxes[b]]];
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) *out = s;
}

// Re sum out_B inc_B D_2 per (box, k tile) on the stored incoming expansions
__global__ void k_tridot(DevTree T, const int* __restrict__ boxes, int nboxes, double* part) {
  __shared__ double sm[32];
  const int tile = blockIdx.x / nboxes, b = blockIdx.x % nboxes;
  const int node = boxes[b];
  const int k = tile * blockDim.x + threadIdx.x;
  const int base = T.pw_base;
  double e = 0;
  if (k < T.H) {
    double2 o = T.out[size_t(node - base) * T.H + k];
    double2 c = T.inc[size_t(node - base) * T.H + k];
    e = (o.x * c.x - o.y * c.y) * T.D2[k];
  }
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// sum of q^2 over each box's slots
__global__ void k_box_q2(DevTree T, const int* __restrict__ boxes, double* q2) {
  __shared__ double sm[32];
  int node = boxes[blockIdx.x];
  double v = 0;
  for (int s = T.node_begin[node] + threadIdx.x; s < T.node_end[node]; s += blockDim.x) v += T.sq[s] * T.sq[s];
  double tot = block_sum(v, sm);
  if (threadIdx.x == 0) q2[blockIdx.x] = tot;
}

// E_diff = sum_box [C_l dscale_l sum_tiles part - Q_B S_l]
__global__ void k_diff_finish(DevTree T, const int* __restrict__ boxes, int nboxes, int ktiles, const double* part,
                              const double* q2, const double* Cl, const double* Sl, double* out) {
  __shared__ double sm[32];
  double e = 0;
  for (int b = threadIdx.x; b < nboxes; b += blockDim.x) {
    int node = boxes[b];
    int l = T.node_level[node];
    double t = 0;
    for (int tile = 0; tile < ktiles; ++tile) t += part[size_t(tile) * nboxes + b];
    e += Cl[l] * level_dscale(l) * t - q2[b] * Sl[l];
  }
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) *out = s;
}

// window energy; the self term sum(q^2) psi_0(0) / (2 b_2 C0) takes sum(q^2)
// from the device (q2) so that no host round trip is needed
__global__ void k_window(DevTree T, double scale, const double* q2, double psi0_0, double self_den, double* out) {
  __shared__ double sm[32];
  double e = 0;
  for (int k = threadIdx.x; k < T.Hw; k += blockDim.x) {
    double2 o = T.out_root[k];
    e += (o.x * o.x + o.y * o.y) * T.W[k];
  }
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) *out = s * scale - *q2 * psi0_0 / self_den;
}


__device__ inline int periodic_shift_d(double xi, double xj, double L, double bi, double bj) {
  if (xi < bi && xj > (L - bj)) return 1;
  if (xi > (L - bi) && xj < bj) return -1;
  return 0;
}

__device__ inline void node_center(const DevTree& T, int node, double* c) {
  uint64_t p = T.node_prefix[node];
  int l = T.node_level[node];
  double scale = ldexp(1.0, -l);
  c[0] = T.L * (double(compact3(p)) * scale + 0.5 * scale);
  c[1] = T.L * (double(compact3(p >> 1)) * scale + 0.5 * scale);
  c[2] = T.L * (double(compact3(p >> 2)) * scale + 0.5 * scale);
}

constexpr int RES_T = 128;
constexpr int RES_TCH = 64;   // targets of one work item
constexpr int RES_SCH = 256;  // sources staged in shared memory per round

// leaf near field: 1/2 sum_{i in B} q_i sum_{j in N(B), j != i} q_j res(r_ij; bs_B)
// (eval_energy_res, src/energy.cpp:82-173). One block per (leaf, chunk of
// RES_TCH targets), so a large leaf is spread over several blocks; leaves are
// listed coarse level first, so the big items start first. The up to 35
// source boxes (self, colleagues, coarse-grain) are flattened into one index
// range, staged in rounds of RES_SCH with their periodic offsets applied.
// Each thread keeps one target in registers and walks a share of the staged
// sources (a warp reads the same source: a shared-memory broadcast).
template <int NP>
__global__ void __launch_bounds__(RES_T) k_residual(DevTree T, const int* __restrict__ leaves, int ny,
                                                    double* part) {
  __shared__ double ux[RES_SCH], uy[RES_SCH], uz[RES_SCH], uq[RES_SCH];
  __shared__ int uslot[RES_SCH];
  __shared__ int m_beg[36], m_pre[37];
  __shared__ double m_off[36][3], m_w[36];
  __shared__ double sm[32];
  // per warp, the pairs inside the cut-off waiting for a polynomial: r^2 and
  // q_target q_source (at most 31 waiting plus 32 added in one step)
  __shared__ double q_r2[RES_T / 32][64], q_w[RES_T / 32][64];
  const ResidualPoly<NP> poly(T);
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int qn = 0;  // pairs waiting in this warp's queue (warp-uniform)
  const int node = leaves[blockIdx.x / ny], chunk = blockIdx.x % ny;
  const int l = T.node_level[node];
  const int cnt = T.leaf_count[node];
  double e = 0;
  double inv_b_all = 0;
  if (l >= 2 && cnt > chunk * RES_TCH) {
    const double b = level_box(T, l), inv_b = 1.0 / b;
    inv_b_all = inv_b;
    const double b2 = b * b * (1.0 + 1e-14);  // square roots only near or inside the cut-off
    const int tb = T.node_begin[node];
    if (threadIdx.x < 36) {
      const int src = threadIdx.x;
      int j = -1;
      if (src == 0) j = node;
      else if (src <= 27) j = (src - 1 == 13) ? -1 : T.col27[size_t(node) * 27 + (src - 1)];
      else j = T.coarse8[size_t(node) * 8 + (src - 28)];
      // A pair of particles in two leaves of the same level meets the same
      // cut-off from either side, so only the leaf with the smaller id sums
      // it, with weight 2. Other sources (non-leaf colleagues, coarser
      // neighbours) see a cut-off that depends on the target's level: both
      // sides sum those.
      const bool same_level_leaf = src >= 1 && src <= 27 && j >= 0 && T.node_child0[j] < 0;
      const bool skip = same_level_leaf && j < node;
      int beg = 0, n = 0;
      double off[3] = {0, 0, 0};
      if (j >= 0 && !skip && T.node_count[j] > 0) {
        double ci[3], cj[3];
        node_center(T, node, ci);
        node_center(T, j, cj);
        const double bj = level_box(T, T.node_level[j]);
        for (int dd = 0; dd < 3; ++dd) off[dd] = -periodic_shift_d(ci[dd], cj[dd], T.L, b, bj) * T.L;
        beg = T.node_begin[j];
        n = (T.node_child0[j] < 0 ? beg + T.leaf_count[j] : T.node_end[j]) - beg;
      }
      m_beg[src] = beg;
      m_pre[src] = n;
      m_w[src] = same_level_leaf ? 2.0 : 1.0;
      for (int dd = 0; dd < 3; ++dd) m_off[src][dd] = off[dd];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int s = 0;
      for (int src = 0; src < 36; ++src) {
        const int n = m_pre[src];
        m_pre[src] = s;
        s += n;
      }
      m_pre[36] = s;
    }
    __syncthreads();
    const int total = m_pre[36];
    for (int t0 = chunk * RES_TCH; t0 < cnt; t0 += ny * RES_TCH) {
      const int nt = min(RES_TCH, cnt - t0);
      const int npad = nt <= 32 ? 32 : 64;
      const int nparts = RES_T / npad;
      const int it = threadIdx.x % npad, sp = threadIdx.x / npad;
      const bool act = it < nt;
      int tslot = -2;
      double tx = 0, ty = 0, tz = 0, tq = 0;
      if (act) {
        tslot = tb + t0 + it;
        tx = T.sx[tslot];
        ty = T.sy[tslot];
        tz = T.sz[tslot];
        tq = T.sq[tslot];
      }
      for (int u0 = 0; u0 < total; u0 += RES_SCH) {
        const int ns = min(RES_SCH, total - u0);
        __syncthreads();
        for (int t = threadIdx.x; t < ns; t += blockDim.x) {
          const int ei = u0 + t;
          int lo = 0, hi = 36;  // largest src with m_pre[src] <= ei
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (m_pre[mid] <= ei) lo = mid;
            else hi = mid;
          }
          const int s = m_beg[lo] + (ei - m_pre[lo]);
          ux[t] = T.sx[s] + m_off[lo][0];
          uy[t] = T.sy[s] + m_off[lo][1];
          uz[t] = T.sz[s] + m_off[lo][2];
          uq[t] = T.sq[s] * m_w[lo];
          uslot[t] = lo == 0 ? s : -1;
        }
        __syncthreads();
        // About one pair in six lies inside the cut-off, and a warp would run
        // the Horner chain whenever any lane needs it: the lanes push their
        // in-range pairs into the warp's queue instead, and the warp
        // evaluates the polynomial 32 queued pairs at a time. The loop is
        // warp-uniform (every lane of a warp has the same source partition).
        for (int js = sp; js < ns; js += nparts) {
          const double dx = tx - ux[js], dy = ty - uy[js], dz = tz - uz[js];
          const double r2 = dx * dx + dy * dy + dz * dz;
          const bool in = act && r2 <= b2 && uslot[js] != tslot;
          const unsigned m = __ballot_sync(0xffffffffu, in);
          if (in) {
            const int pos = qn + __popc(m & ((1u << lane) - 1u));
            q_r2[wid][pos] = r2;
            q_w[wid][pos] = tq * uq[js];
          }
          qn += __popc(m);
          if (qn >= 32) {
            __syncwarp();
            e += q_w[wid][lane] * poly.from_r2(q_r2[wid][lane], inv_b);  // from_r2 is zero beyond the cut-off
            const int rem = qn - 32;
            double r2m = 0, wm = 0;
            if (lane < rem) {
              r2m = q_r2[wid][32 + lane];
              wm = q_w[wid][32 + lane];
            }
            __syncwarp();
            if (lane < rem) {
              q_r2[wid][lane] = r2m;
              q_w[wid][lane] = wm;
            }
            __syncwarp();
            qn = rem;
          }
        }
      }
    }
  }
  // the pairs still queued
  __syncwarp();
  if (lane < qn) e += q_w[wid][lane] * poly.from_r2(q_r2[wid][lane], inv_b_all);
  double s = block_sum(0.5 * e, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// ---------------------------------------------------------------------------
// FP64 Ewald comparator (the reference's Ewald summation, src/ewald.cpp:17-223):
// E = 1/2 sum_{i != j, images} q_i q_j erfc(alpha r)/r
//   + (2 pi / V) sum_{k != 0} exp(-k^2 / (4 alpha^2)) / k^2 |S(k)|^2
//   - alpha / sqrt(pi) sum_i q_i^2,  S(k) = sum_j q_j exp(i k.r_j).
// The real-space cut-off is the box size of one tree level, so the 27 boxes
// of that level around a box hold every pair; S(k) comes from the NUDFT
// kernel (the conjugate, which leaves |S|^2 unchanged).

// real space: one block per (box, chunk of RES_TCH targets), as the near field
__global__ void __launch_bounds__(RES_T) k_ewald_real(DevTree T, int level, int ny, double alpha, double rc,
                                                      double* part) {
  __shared__ double ux[RES_SCH], uy[RES_SCH], uz[RES_SCH], uq[RES_SCH];
  __shared__ int uslot[RES_SCH];
  __shared__ int m_beg[27], m_pre[28];
  __shared__ double m_off[27][3];
  __shared__ double sm[32];
  const int node = T.level_start_d[level] + int(blockIdx.x) / ny, chunk = int(blockIdx.x) % ny;
  const int tb = T.node_begin[node];
  const int cnt = T.node_end[node] - tb;  // slots, empty ones carry q = 0
  double e = 0;
  if (cnt > chunk * RES_TCH) {
    const double b = level_box(T, level);
    const double rc2 = rc * rc;
    if (threadIdx.x < 27) {
      const int dir = threadIdx.x;
      const int j = dir == 13 ? node : T.col27[size_t(node) * 27 + dir];
      int beg = 0, n = 0;
      double off[3] = {0, 0, 0};
      if (j >= 0) {
        double ci[3], cj[3];
        node_center(T, node, ci);
        node_center(T, j, cj);
        for (int dd = 0; dd < 3; ++dd) off[dd] = -periodic_shift_d(ci[dd], cj[dd], T.L, b, b) * T.L;
        beg = T.node_begin[j];
        n = T.node_end[j] - beg;
      }
      m_beg[dir] = beg;
      m_pre[dir] = n;
      for (int dd = 0; dd < 3; ++dd) m_off[dir][dd] = off[dd];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int src = 0; src < 27; ++src) {
        const int n = m_pre[src];
        m_pre[src] = acc;
        acc += n;
      }
      m_pre[27] = acc;
    }
    __syncthreads();
    const int total = m_pre[27];
    for (int t0 = chunk * RES_TCH; t0 < cnt; t0 += ny * RES_TCH) {
      const int nt = min(RES_TCH, cnt - t0);
      const int npad = nt <= 32 ? 32 : 64;
      const int nparts = RES_T / npad;
      const int it = threadIdx.x % npad, sp = threadIdx.x / npad;
      const bool act = it < nt;
      int tslot = -2;
      double tx = 0, ty = 0, tz = 0, tq = 0;
      if (act) {
        tslot = tb + t0 + it;
        tx = T.sx[tslot];
        ty = T.sy[tslot];
        tz = T.sz[tslot];
        tq = T.sq[tslot];
      }
      double et = 0;
      for (int u0 = 0; u0 < total; u0 += RES_SCH) {
        const int ns = min(RES_SCH, total - u0);
        __syncthreads();
        for (int t = threadIdx.x; t < ns; t += blockDim.x) {
          const int ei = u0 + t;
          int lo = 0, hi = 27;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (m_pre[mid] <= ei) lo = mid;
            else hi = mid;
          }
          const int sl = m_beg[lo] + (ei - m_pre[lo]);
          ux[t] = T.sx[sl] + m_off[lo][0];
          uy[t] = T.sy[sl] + m_off[lo][1];
          uz[t] = T.sz[sl] + m_off[lo][2];
          uq[t] = T.sq[sl];
          uslot[t] = sl;
        }
        __syncthreads();
        if (act && tq != 0.0)
          for (int js = sp; js < ns; js += nparts) {
            const double dx = tx - ux[js], dy = ty - uy[js], dz = tz - uz[js];
            const double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 < rc2 && uslot[js] != tslot && uq[js] != 0.0) {
              const double r = sqrt(r2);
              et += uq[js] * erfc(alpha * r) / r;
            }
          }
      }
      e += tq * et;
    }
  }
  double sum = block_sum(0.5 * e, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = sum;
}

// reciprocal space over the stored half grid kz <= 0 (kz < 0 stands for its
// mirror too)
__global__ void k_ewald_recip(const double2* __restrict__ S, int nk, double dk, double alpha, double* part) {
  __shared__ double sm[32];
  const int d = 2 * nk + 1;
  const long H = long(d) * d * (nk + 1);
  double e = 0;
  for (long k = long(blockIdx.x) * blockDim.x + threadIdx.x; k < H; k += long(gridDim.x) * blockDim.x) {
    const int ix = int(k % d), iy = int((k / d) % d), iz = int(k / (long(d) * d));
    const int mx = ix - nk, my = iy - nk, mz = iz - nk;
    if ((mx | my | mz) == 0) continue;
    const double k2 = dk * dk * double(mx * mx + my * my + mz * mz);
    const double2 v = S[k];
    e += (mz < 0 ? 2.0 : 1.0) * exp(-k2 / (4.0 * alpha * alpha)) / k2 * (v.x * v.x + v.y * v.y);
  }
  const double sum = block_sum(e, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = sum;
}

__global__ void k_sum(const double* part, int n, double* out) {
  __shared__ double sm[32];
  double e = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) e += part[i];
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) *out = s;
}

// sum of q^2 over the slots: block b sums a grid-strided share into out[b]
// (one block gives the total in out[0])
__global__ void k_sum_q2(const double* sq, int n, double* out) {
  __shared__ double sm[32];
  double e = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) e += sq[i] * sq[i];
  double s = block_sum(e, sm);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

}  // namespace

// ---------------------------------------------------------------------------
// host side

constexpr int RES_NY_MAX = 8;  // the partials buffer holds this many near-field chunks per node

// target chunks per leaf in the near-field launch: enough for a full leaf
// with its slack (larger leaves loop over their chunks), at most the tuned cap
int DmkTree::res_chunks() const {
  return std::min(std::min(RES_NY_MAX, tune_.res_ny_max),
                  std::max(1, (n_per_leaf_ + opt_.leaf_slack + RES_TCH - 1) / RES_TCH));
}

void DmkTree::set_tuning(const Tuning& t) {
  Tuning c = t;
  // the mixed pass's exact int32 sums hold 16384 particles per split-K
  // chunk: an accumulator takes at most four slice products per K entry, top
  // digits lie in [-127, 127] and lower ones in [-128, 127], so one K entry
  // adds at most 2 127 128 + 2 128^2 = 65280, and two K entries per particle
  // give 2 16384 65280 < 2^31
  const int cap = opt_.precision == 1 ? 16384 : 1 << 20;
  c.ksplit = std::min(cap, std::max(256, c.ksplit));
  c.ksplit_root = std::min(cap, std::max(256, c.ksplit_root));
  c.inc_waves = std::min(64, std::max(1, c.inc_waves));
  c.res_ny_max = std::min(RES_NY_MAX, std::max(1, c.res_ny_max));
  tune_ = c;
}

double DmkTree::time_phase(int phase, int reps) {
  std::vector<float> ms;
  cudaEvent_t a, b;
  PDMK_CUDA(cudaEventCreate(&a));
  PDMK_CUDA(cudaEventCreate(&b));
  for (int r = 0; r < reps; ++r) {
    PDMK_CUDA(cudaStreamSynchronize(st_));
    PDMK_CUDA(cudaEventRecord(a, st_));
    if (phase == 0) {
      form_outgoing_pw();
    } else if (phase == 1) {
      form_incoming_pw();
    } else {
      ensure_packed();
      launch_res_energy();
    }
    PDMK_CUDA(cudaEventRecord(b, st_));
    PDMK_CUDA(cudaEventSynchronize(b));
    float t = 0;
    PDMK_CUDA(cudaEventElapsedTime(&t, a, b));
    ms.push_back(t);
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  std::sort(ms.begin(), ms.end());
  return ms.empty() ? 0.0 : double(ms[ms.size() / 2]);
}

size_t DmkTree::partials_needed() const {
  const DevTree& D = dev_;
  size_t need = 8192;
  long n_pw = D.pw_hi >= D.pw_lo ? long(D.level_start[D.pw_hi + 1]) - D.level_start[D.pw_lo] : 0;
  long ktiles = (D.H + TPB - 1) / TPB;
  need = std::max<size_t>(need, size_t(n_pw) * ktiles + 2 * size_t(n_pw) + 64);
  // cube-tiled incoming: at most one cube per 8 expansion boxes
  need = std::max<size_t>(need, size_t((D.H + INC_KT - 1) / INC_KT) * size_t(n_pw / 8 + 1) + 2 * size_t(n_pw) + 64);
  need = std::max<size_t>(need, size_t(D.n_nodes) * RES_NY_MAX + 64);
  return need;
}

void DmkTree::ensure_packed() {
  // only accepted moves put particles into the overflow pool: a tree without
  // moves since its build or last pack needs no device round trip
  if (!moved_) return;
  int pn = 0;
  PDMK_CUDA(cudaMemcpyAsync(&pn, dev_.pool_n, 4, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  if (pn > 0) repack(opt_.leaf_slack);
  moved_ = false;
}

void DmkTree::form_outgoing_pw() {
  ensure_packed();
  DevTree& D = dev_;
  // split-K bookkeeping: chunks go to a partial buffer, then reduce
  struct Chunked {
    int first, n;
    double2* out;
  };
  // the row tiles of one box (or box chunk) over the slots [sb, se)
  auto make_work = [&](std::vector<NudftWork>& wl, int nk, int l, uint64_t p, double2* out, int sb, int se) {
    NudftWork w{};
    double scale = std::ldexp(1.0, -l);
    int X = int(compact3(p)), Y = int(compact3(p >> 1)), Z = int(compact3(p >> 2));
    w.cx = L_ * (double(X) * scale + 0.5 * scale);
    w.cy = L_ * (double(Y) * scale + 0.5 * scale);
    w.cz = L_ * (double(Z) * scale + 0.5 * scale);
    w.dk = D.delta_k[l];
    w.X = X;
    w.Y = Y;
    w.Z = Z;
    w.M = l == 0 ? 3 : 1;
    w.s_begin = sb;
    w.s_end = se;
    w.out = out;
    int tiles = nudft_tiles(nk);
    for (int t = 0; t < tiles; ++t) {
      w.row_tile = t;
      wl.push_back(w);
    }
  };
  // the mixed pass: one item per (box or box chunk, pair of 128-row M tiles)
  auto make_mix = [&](std::vector<MixItem>& wl, int nk, int l, uint64_t p, double2* out, int sb, int se) {
    MixItem w{};
    double scale = std::ldexp(1.0, -l);
    int X = int(compact3(p)), Y = int(compact3(p >> 1)), Z = int(compact3(p >> 2));
    w.cx = L_ * (double(X) * scale + 0.5 * scale);
    w.cy = L_ * (double(Y) * scale + 0.5 * scale);
    w.cz = L_ * (double(Z) * scale + 0.5 * scale);
    w.dk = D.delta_k[l];
    w.X = X;
    w.Y = Y;
    w.Z = Z;
    w.M = l == 0 ? 3 : 1;
    w.s_begin = sb;
    w.s_end = se;
    w.out = out;
    const int pairs = mixed_pairs(nk);
    for (int t = 0; t < pairs; ++t) {
      w.pair = t;
      wl.push_back(w);
    }
  };
  const bool mixed = opt_.precision == 1;
  CUtensorMap tmap_root{}, tmap_box{};
  if (mixed) {
    if (!d_mix_) {
      d_mix_ = static_cast<double*>(alloc(sizeof(double) * 2));
      PDMK_CUDA(cudaMemsetAsync(d_mix_, 0, sizeof(double) * 2, st_));
    }
    if (!qmax_ready_) {
      launch_absmax(D.sq, D.n_slots, d_mix_, st_);
      qmax_ready_ = true;
    }
    make_coord_map(&tmap_root, D.sx, slot_capacity_, mixed_chunk(D.n_window));
    make_coord_map(&tmap_box, D.sx, slot_capacity_, mixed_chunk(D.n_diff));
  }
  int* d_mix_err = mixed ? reinterpret_cast<int*>(d_mix_ + 1) : nullptr;
  auto align16 = [](size_t b) { return (b + 15) & ~size_t(15); };
  // one upload per pass: the work items, their table chunk lists, then per
  // split-K group its first chunk, chunk count and output
  auto upload = [&](const auto& wl, const std::vector<int2>& ch, const std::vector<Chunked>& sp, size_t* off_ch,
                    size_t* off_meta, size_t* off_out) {
    using Item = typename std::decay_t<decltype(wl)>::value_type;
    *off_ch = align16(sizeof(Item) * wl.size());
    *off_meta = align16(*off_ch + sizeof(int2) * ch.size());
    *off_out = align16(*off_meta + sizeof(int) * 2 * sp.size());
    const size_t bytes = align16(*off_out + sizeof(double2*) * sp.size()) + 16;
    std::vector<unsigned char> blob(bytes, 0);
    std::memcpy(blob.data(), wl.data(), sizeof(Item) * wl.size());
    std::memcpy(blob.data() + *off_ch, ch.data(), sizeof(int2) * ch.size());
    int* meta = reinterpret_cast<int*>(blob.data() + *off_meta);
    double2** outs = reinterpret_cast<double2**>(blob.data() + *off_out);
    for (size_t i = 0; i < sp.size(); ++i) {
      meta[i] = sp[i].first;
      meta[sp.size() + i] = sp[i].n;
      outs[i] = sp[i].out;
    }
    unsigned char* d_blob;
    PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_blob), bytes, st_));
    PDMK_CUDA(cudaMemcpyAsync(d_blob, blob.data(), bytes, cudaMemcpyHostToDevice, st_));
    return d_blob;
  };
  auto reduce = [&](const std::vector<Chunked>& sp, const double2* pbase, int H, const unsigned char* d_blob,
                    size_t off_meta, size_t off_out, cudaStream_t st) {
    if (sp.empty()) return;
    const int nbx = int(sp.size());
    const int* d_meta = reinterpret_cast<const int*>(d_blob + off_meta);
    double2* const* d_outs = reinterpret_cast<double2* const*>(d_blob + off_out);
    dim3 grid(grid_for(H), unsigned(nbx));
    k_reduce_chunks<<<grid, TPB, 0, st>>>(pbase, d_meta, d_meta + nbx, d_outs, H);
    PDMK_LAUNCH_CHECK();
  };
  // the mixed pass's chunk tables: one block of mixed_table_bytes per chunk
  // of each slot range, shared by the range's consecutive tile items; the
  // chunk list names each chunk's range by its first tile item
  auto plan_mix_tables = [&](int nk, std::vector<MixItem>& wl, unsigned char** tab, std::vector<int2>& ch) {
    const int kcp = mixed_chunk(nk), tiles = mixed_pairs(nk);
    const size_t tb = size_t(mixed_table_bytes(nk));
    size_t total = 0;
    for (size_t i = 0; i < wl.size(); i += tiles) total += size_t((wl[i].s_end - wl[i].s_begin + kcp - 1) / kcp);
    PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(tab), total * tb + 16, st_));
    size_t cur = 0;
    for (size_t i = 0; i < wl.size(); i += tiles) {
      const int n = (wl[i].s_end - wl[i].s_begin + kcp - 1) / kcp;
      for (int t = 0; t < tiles; ++t) wl[i + t].tab = *tab + cur * tb;
      for (int c = 0; c < n; ++c) ch.push_back(make_int2(int(i), c));
      cur += size_t(n);
    }
  };
  if (!aux_) {
    PDMK_CUDA(cudaStreamCreateWithFlags(&aux_, cudaStreamNonBlocking));
    PDMK_CUDA(cudaEventCreateWithFlags(&ev_fork_, cudaEventDisableTiming));
    PDMK_CUDA(cudaEventCreateWithFlags(&ev_join_, cudaEventDisableTiming));
  }

  // Root pass first, on the second stream: the root (node 0, all slots) needs
  // no host view of the tree, so it runs while the host lays out the boxes.
  // Its allocations are made on the tree's stream before the fork event.
  const int KSPLIT = tune_.ksplit, KSPLIT_ROOT = tune_.ksplit_root;
  const int nch_root = std::max(1, (D.n_slots + KSPLIT_ROOT - 1) / KSPLIT_ROOT);
  std::vector<Chunked> root_split{{0, nch_root, D.out_root}};
  double2* part_r = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part_r), sizeof(double2) * (size_t(nch_root) * D.Hw + 1), st_));
  std::vector<NudftWork> wroot;
  std::vector<MixItem> mroot;
  for (int c = 0; c < nch_root; ++c) {
    int sb = c * KSPLIT_ROOT, se = std::min(D.n_slots, sb + KSPLIT_ROOT);
    if (mixed) make_mix(mroot, D.n_window, 0, 0, part_r + size_t(c) * D.Hw, sb, se);
    else make_work(wroot, D.n_window, 0, 0, part_r + size_t(c) * D.Hw, sb, se);
  }
  double2* tab_root = nullptr;
  unsigned char* mtab_root = nullptr;
  std::vector<int2> ch_root;
  size_t rch, rmeta, rout;
  unsigned char* d_root = nullptr;
  if (mixed) {
    plan_mix_tables(D.n_window, mroot, &mtab_root, ch_root);
    d_root = upload(mroot, ch_root, root_split, &rch, &rmeta, &rout);
  } else {
    plan_nudft_tables(D.n_window, wroot, &tab_root, ch_root, st_);
    d_root = upload(wroot, ch_root, root_split, &rch, &rmeta, &rout);
  }
  PDMK_CUDA(cudaEventRecord(ev_fork_, st_));
  PDMK_CUDA(cudaStreamWaitEvent(aux_, ev_fork_, 0));
  if (mixed)
    dispatch_mixed(D.n_window, tmap_root, reinterpret_cast<const MixItem*>(d_root), int(mroot.size()),
                   reinterpret_cast<const int2*>(d_root + rch), int(ch_root.size()), d_mix_, d_mix_err, aux_);
  else
    dispatch_nudft(D.n_window, reinterpret_cast<const NudftWork*>(d_root), int(wroot.size()),
                   reinterpret_cast<const int2*>(d_root + rch), int(ch_root.size()), D, aux_);
  reduce(root_split, part_r, D.Hw, d_root, rmeta, rout, aux_);
  PDMK_CUDA(cudaEventRecord(ev_join_, aux_));

  // host view of node slot ranges and coordinates for the box work list
  // (and, on a new tree, of the children for the box lists: one round trip)
  const int nn = D.n_nodes;
  std::vector<int> nb(nn), ne(nn), lv(nn), c0;
  std::vector<uint64_t> pf(nn);
  PDMK_CUDA(cudaMemcpyAsync(nb.data(), D.node_begin, 4 * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(ne.data(), D.node_end, 4 * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(lv.data(), D.node_level, 4 * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(pf.data(), D.node_prefix, 8 * nn, cudaMemcpyDeviceToHost, st_));
  if (!box_lists_ready_) {
    c0.resize(nn);
    PDMK_CUDA(cudaMemcpyAsync(c0.data(), D.node_child0, 4 * nn, cudaMemcpyDeviceToHost, st_));
  }
  PDMK_CUDA(cudaStreamSynchronize(st_));
  if (!box_lists_ready_) build_box_lists(c0);
  struct Box {
    int node, sb, se, level;
    double2* out;
  };
  std::vector<Box> boxes;
  const int base = D.level_start[D.pw_lo];
  if (D.pw_hi >= D.pw_lo)
    for (int id = base; id < D.level_start[D.pw_hi + 1]; ++id)
      boxes.push_back({id, nb[id], ne[id], lv[id], D.out + size_t(id - base) * D.H});
  // boxes: largest first (longest-processing-time order), split when large
  std::vector<int> order(boxes.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = int(i);
  std::stable_sort(order.begin(), order.end(),
                   [&](int a, int b) { return boxes[a].se - boxes[a].sb > boxes[b].se - boxes[b].sb; });
  std::vector<Chunked> box_split;
  long chunk_cursor = 0;
  for (int oi : order) {
    const Box& bx = boxes[oi];
    int cntp = bx.se - bx.sb;
    if (cntp > KSPLIT) {
      int nch = (cntp + KSPLIT - 1) / KSPLIT;
      box_split.push_back({int(chunk_cursor), nch, bx.out});
      chunk_cursor += nch;
    }
  }
  double2* part_b = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part_b), sizeof(double2) * (size_t(chunk_cursor) * D.H + 1), st_));
  std::vector<NudftWork> wbox;
  std::vector<MixItem> mbox;
  {
    size_t si = 0;
    long cur = 0;
    auto add = [&](int l, uint64_t p, double2* out, int sb, int se) {
      if (mixed) make_mix(mbox, D.n_diff, l, p, out, sb, se);
      else make_work(wbox, D.n_diff, l, p, out, sb, se);
    };
    for (int oi : order) {
      const Box& bx = boxes[oi];
      int cntp = bx.se - bx.sb;
      if (cntp > KSPLIT) {
        int nch = box_split[si].n;
        for (int c = 0; c < nch; ++c) {
          int sb = bx.sb + c * KSPLIT, se = std::min(bx.se, sb + KSPLIT);
          add(bx.level, pf[bx.node], part_b + size_t(cur + c) * D.H, sb, se);
        }
        cur += nch;
        ++si;
      } else {
        add(bx.level, pf[bx.node], bx.out, bx.sb, bx.se);
      }
    }
  }
  double2* tab_box = nullptr;
  unsigned char* mtab_box = nullptr;
  std::vector<int2> ch_box;
  size_t bch, bmeta, bout;
  unsigned char* d_box = nullptr;
  if (mixed) {
    plan_mix_tables(D.n_diff, mbox, &mtab_box, ch_box);
    d_box = upload(mbox, ch_box, box_split, &bch, &bmeta, &bout);
  } else {
    plan_nudft_tables(D.n_diff, wbox, &tab_box, ch_box, st_);
    d_box = upload(wbox, ch_box, box_split, &bch, &bmeta, &bout);
  }
  time_begin(3);
  if (mixed)
    dispatch_mixed(D.n_diff, tmap_box, reinterpret_cast<const MixItem*>(d_box), int(mbox.size()),
                   reinterpret_cast<const int2*>(d_box + bch), int(ch_box.size()), d_mix_, d_mix_err, st_);
  else
    dispatch_nudft(D.n_diff, reinterpret_cast<const NudftWork*>(d_box), int(wbox.size()),
                   reinterpret_cast<const int2*>(d_box + bch), int(ch_box.size()), D, st_);
  time_end(3);
  reduce(box_split, part_b, D.H, d_box, bmeta, bout, st_);
  // the root pass's buffers are released after it joins the tree's stream
  PDMK_CUDA(cudaStreamWaitEvent(st_, ev_join_, 0));
  for (void* p : {static_cast<void*>(d_root), static_cast<void*>(tab_root), static_cast<void*>(mtab_root),
                  static_cast<void*>(part_r), static_cast<void*>(d_box), static_cast<void*>(tab_box),
                  static_cast<void*>(mtab_box), static_cast<void*>(part_b)})
    if (p) PDMK_CUDA(cudaFreeAsync(p, st_));
  diff_cached_ = false;
}

void DmkTree::prepare_box_lists() {
  if (box_lists_ready_) return;
  std::vector<int> c0(dev_.n_nodes);
  PDMK_CUDA(cudaMemcpyAsync(c0.data(), dev_.node_child0, 4 * dev_.n_nodes, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  build_box_lists(c0);
}

void DmkTree::build_box_lists(const std::vector<int>& c0) {
  DevTree& D = dev_;
  std::vector<int> nonleaf;
  if (D.pw_hi >= D.pw_lo)
    for (int id = D.level_start[D.pw_lo]; id < D.level_start[D.pw_hi + 1]; ++id)
      if (c0[id] >= 0) nonleaf.push_back(id);
  std::vector<int> leaves;
  for (int id = D.level_start[2]; id < D.n_nodes; ++id)
    if (c0[id] < 0) leaves.push_back(id);
  // boxes two levels above the expansion levels with a non-leaf grandchild:
  // each names the 4 x 4 x 4 receiving boxes of one incoming block
  std::vector<int> cubes;
  if (D.pw_hi >= D.pw_lo)
    for (int id = D.level_start[D.pw_lo - 2]; id < D.level_start[D.pw_hi - 1]; ++id) {
      if (c0[id] < 0) continue;
      bool any = false;
      for (int a = 0; a < 8 && !any; ++a) {
        const int ch = c0[id] + a;
        if (c0[ch] < 0) continue;
        for (int b = 0; b < 8; ++b) any = any || c0[c0[ch] + b] >= 0;
      }
      if (any) cubes.push_back(id);
    }
  n_cubes_ = int(cubes.size());
  d_cubes_ = static_cast<int*>(alloc(sizeof(int) * (n_cubes_ + 1)));
  PDMK_CUDA(cudaMemcpyAsync(d_cubes_, cubes.data(), sizeof(int) * n_cubes_, cudaMemcpyHostToDevice, st_));
  n_nonleaf_ = int(nonleaf.size());
  n_leaves_ = int(leaves.size());
  d_nonleaf_ = static_cast<int*>(alloc(sizeof(int) * (n_nonleaf_ + 1)));
  d_leaves_ = static_cast<int*>(alloc(sizeof(int) * (n_leaves_ + 1)));
  PDMK_CUDA(cudaMemcpyAsync(d_nonleaf_, nonleaf.data(), sizeof(int) * n_nonleaf_, cudaMemcpyHostToDevice, st_));
  PDMK_CUDA(cudaMemcpyAsync(d_leaves_, leaves.data(), sizeof(int) * n_leaves_, cudaMemcpyHostToDevice, st_));
  // per-level constants of eval_energy_diff (src/energy.cpp:50-57)
  const double pi = 3.14159265358979323846;
  std::vector<double> Cl(MAX_LEVELS + 2, 0.0), Sl(MAX_LEVELS + 2, 0.0);
  for (int l = 2; l < MAX_LEVELS + 1; ++l) {
    Cl[l] = 1 / (2 * std::pow(2 * pi, 3)) * std::pow(D.delta_k[l], 3);
    Sl[l] = ps_.psi0_0 * (1 / (2 * D.boxsize[l + 1] * ps_.C0) - 1 / (2 * D.boxsize[l] * ps_.C0));
  }
  d_Cl_ = static_cast<double*>(alloc(sizeof(double) * 2 * (MAX_LEVELS + 2)));
  d_Sl_ = d_Cl_ + (MAX_LEVELS + 2);
  PDMK_CUDA(cudaMemcpyAsync(d_Cl_, Cl.data(), sizeof(double) * (MAX_LEVELS + 2), cudaMemcpyHostToDevice, st_));
  PDMK_CUDA(cudaMemcpyAsync(d_Sl_, Sl.data(), sizeof(double) * (MAX_LEVELS + 2), cudaMemcpyHostToDevice, st_));
  d_scalars_ = static_cast<double*>(alloc(sizeof(double) * 8));
  // sum(q^2) for the window self term: 64 block partials, then a fixed-order sum
  k_sum_q2<<<64, 256, 0, st_>>>(D.sq, D.n_slots, D.partials);
  PDMK_LAUNCH_CHECK();
  k_sum<<<1, 1024, 0, st_>>>(D.partials, 64, d_scalars_ + 4);
  PDMK_LAUNCH_CHECK();
  box_lists_ready_ = true;
}

void DmkTree::run_incoming(bool write_inc) {
  ensure_packed();
  prepare_box_lists();
  DevTree& D = dev_;
  if (n_nonleaf_ == 0) {
    PDMK_CUDA(cudaMemsetAsync(d_scalars_ + 1, 0, sizeof(double), st_));
    return;
  }
  const int ktiles = (D.H + TPB - 1) / TPB;
  const size_t n_part = std::max(size_t(ktiles) * n_nonleaf_, size_t((D.H + INC_KT - 1) / INC_KT) * n_cubes_);
  double* part = D.partials;
  double* q2 = D.partials + n_part;
  k_box_q2<<<unsigned(n_nonleaf_), TPB, 0, st_>>>(D, d_nonleaf_, q2);
  PDMK_LAUNCH_CHECK();
  if (write_inc) {
    // about inc_waves resident waves of blocks (two per SM), each walking a
    // strided set of tiles
    const int kt = (D.H + INC_KT - 1) / INC_KT;
    const int nc = std::max(n_cubes_, 1);
    const int slots = std::max(1, std::min(kt, (tune_.inc_waves * 2 * 148 + nc - 1) / nc));
    if (n_cubes_ > 0) launch_incoming(D, d_cubes_, n_cubes_, slots, part, st_);
    k_diff_finish_cube<<<1, 1024, 0, st_>>>(D, d_cubes_, n_cubes_, slots, part, d_nonleaf_, n_nonleaf_, q2, d_Cl_,
                                            d_Sl_, d_scalars_ + 1);
    PDMK_LAUNCH_CHECK();
  } else {
    k_tridot<<<unsigned(ktiles * n_nonleaf_), TPB, 0, st_>>>(D, d_nonleaf_, n_nonleaf_, part);
    PDMK_LAUNCH_CHECK();
    k_diff_finish<<<1, 1024, 0, st_>>>(D, d_nonleaf_, n_nonleaf_, ktiles, part, q2, d_Cl_, d_Sl_, d_scalars_ + 1);
    PDMK_LAUNCH_CHECK();
  }
}

void DmkTree::form_incoming_pw() {
  run_incoming(true);
  diff_cached_ = true;
}

void DmkTree::launch_window_energy() {
  prepare_box_lists();
  DevTree& D = dev_;
  const double pi = 3.14159265358979323846;
  double scale = 1 / (2 * std::pow(2 * pi, 3)) * std::pow(D.delta_k[0], 3);
  k_window<<<1, 1024, 0, st_>>>(D, scale, d_scalars_ + 4, ps_.psi0_0, 2 * D.boxsize[2] * ps_.C0, d_scalars_ + 0);
  PDMK_LAUNCH_CHECK();
}

double DmkTree::eval_window_energy() {
  launch_window_energy();
  double e;
  PDMK_CUDA(cudaMemcpyAsync(&e, d_scalars_ + 0, sizeof(double), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  return e;
}

double DmkTree::eval_diff_energy() {
  ensure_packed();
  if (!diff_cached_) run_incoming(false);
  double e;
  PDMK_CUDA(cudaMemcpyAsync(&e, d_scalars_ + 1, sizeof(double), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  return e;
}

void DmkTree::launch_res_energy() {
  prepare_box_lists();
  DevTree& D = dev_;
  if (n_leaves_ > 0) {
    auto kern = D.n_poly == 7 ? k_residual<7> : D.n_poly == 13 ? k_residual<13> : D.n_poly == 19 ? k_residual<19>
                                                                                                 : k_residual<25>;
    const int ny = res_chunks();
    kern<<<unsigned(n_leaves_ * ny), RES_T, 0, st_>>>(D, d_leaves_, ny, D.partials);
    PDMK_LAUNCH_CHECK();
    k_sum<<<1, 1024, 0, st_>>>(D.partials, n_leaves_ * ny, d_scalars_ + 2);
    PDMK_LAUNCH_CHECK();
  } else {
    PDMK_CUDA(cudaMemsetAsync(d_scalars_ + 2, 0, sizeof(double), st_));
  }
}

double DmkTree::eval_res_energy() {
  ensure_packed();
  launch_res_energy();
  double e = 0;
  PDMK_CUDA(cudaMemcpyAsync(&e, d_scalars_ + 2, sizeof(double), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  return e;
}

int DmkTree::check_mixed_error() {
  if (!d_mix_) return 0;
  int e = 0;
  PDMK_CUDA(cudaMemcpyAsync(&e, d_mix_ + 1, sizeof(int), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  return e;
}

EnergyParts DmkTree::eval_energy() {
  // per-box charge sums and the near field read particles from the slot
  // ranges: fold any overflow-pool arrivals back into them first. The three
  // parts are enqueued back to back and read with one synchronisation.
  ensure_packed();
  launch_window_energy();
  if (!diff_cached_) run_incoming(false);
  launch_res_energy();
  double e[3];
  int mix_err = 0;
  PDMK_CUDA(cudaMemcpyAsync(e, d_scalars_, sizeof(e), cudaMemcpyDeviceToHost, st_));
  if (d_mix_) PDMK_CUDA(cudaMemcpyAsync(&mix_err, d_mix_ + 1, sizeof(int), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  if (mix_err) throw DeviceError("mixed-precision outgoing pass: a pipeline wait gave up");
  EnergyParts p;
  p.window = e[0];
  p.diff = e[1];
  p.res = e[2];
  return p;
}

// FP64 Ewald energy of the current particles (comparator; s = 5: erfc(5) and
// exp(-25) put the truncation near 1e-12 relative). The real-space cut-off is
// the box size of level 2, or of level 3 when that level is complete and the
// system is large; the k cube then needs 32 or 64 modes per axis half.
double DmkTree::ewald_energy(double* parts) {
  ensure_packed();
  DevTree& D = dev_;
  const double s = 5.0, pi = 3.14159265358979323846;
  const bool l3 = D.max_depth > 4 && D.level_start[4] - D.level_start[3] == 512 && D.n_slots > 300000;
  const int le = l3 ? 3 : 2;
  const int nk = l3 ? 64 : 32;
  const double rc = std::ldexp(L_, -le), alpha = s / rc, dk = 2 * pi / L_;
  const int nbox = D.level_start[le + 1] - D.level_start[le];
  // chunks of targets per box: enough for the fullest box of the level
  std::vector<int> nb(nbox), ne(nbox);
  PDMK_CUDA(cudaMemcpyAsync(nb.data(), D.node_begin + D.level_start[le], 4 * nbox, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(ne.data(), D.node_end + D.level_start[le], 4 * nbox, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  int maxc = 1;
  for (int b = 0; b < nbox; ++b) maxc = std::max(maxc, ne[b] - nb[b]);
  const int ny = (maxc + RES_TCH - 1) / RES_TCH;
  // structure factor by the NUDFT over all slots, split in chunks
  const int Hs = (2 * nk + 1) * (2 * nk + 1) * (nk + 1);
  const int kspl = std::max(4096, (D.n_slots + 295) / 296);
  const int nch = std::max(1, (D.n_slots + kspl - 1) / kspl);
  const int tiles = nudft_tiles(nk);
  std::vector<NudftWork> wl;
  for (int c = 0; c < nch; ++c) {
    NudftWork w{};
    w.cx = w.cy = w.cz = 0.5 * L_;
    w.dk = dk;
    w.M = 3;  // exp(-i k L/2) = (-1)^m: the root's decentring
    w.s_begin = c * kspl;
    w.s_end = std::min(D.n_slots, (c + 1) * kspl);
    for (int t = 0; t < tiles; ++t) {
      w.row_tile = t;
      wl.push_back(w);
    }
  }
  double2* part = nullptr;
  double2* S = nullptr;
  NudftWork* d_work = nullptr;
  const int nblk_real = nbox * ny, nblk_rec = 1024;
  double* sums = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&part), sizeof(double2) * size_t(Hs) * nch, st_));
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&S), sizeof(double2) * size_t(Hs), st_));
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&sums), sizeof(double) * (nblk_real + nblk_rec + 8), st_));
  for (size_t i = 0; i < wl.size(); ++i) wl[i].out = part + size_t(i / tiles) * Hs;
  double2* tab = nullptr;
  std::vector<int2> chunks;
  plan_nudft_tables(nk, wl, &tab, chunks, st_);
  const size_t off_ch = (sizeof(NudftWork) * wl.size() + 15) & ~size_t(15);
  std::vector<unsigned char> blob(off_ch + sizeof(int2) * chunks.size() + 16, 0);
  std::memcpy(blob.data(), wl.data(), sizeof(NudftWork) * wl.size());
  std::memcpy(blob.data() + off_ch, chunks.data(), sizeof(int2) * chunks.size());
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_work), blob.size(), st_));
  PDMK_CUDA(cudaMemcpyAsync(d_work, blob.data(), blob.size(), cudaMemcpyHostToDevice, st_));
  dispatch_nudft(nk, d_work, int(wl.size()),
                 reinterpret_cast<const int2*>(reinterpret_cast<unsigned char*>(d_work) + off_ch), int(chunks.size()),
                 D, st_);
  PDMK_CUDA(cudaFreeAsync(tab, st_));
  {
    int* d_meta;
    double2** d_outs;
    const int meta[2] = {0, nch};
    PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_meta), sizeof(int) * 2, st_));
    PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_outs), sizeof(double2*), st_));
    PDMK_CUDA(cudaMemcpyAsync(d_meta, meta, sizeof(meta), cudaMemcpyHostToDevice, st_));
    PDMK_CUDA(cudaMemcpyAsync(d_outs, &S, sizeof(double2*), cudaMemcpyHostToDevice, st_));
    k_reduce_chunks<<<dim3(grid_for(Hs), 1u), TPB, 0, st_>>>(part, d_meta, d_meta + 1, d_outs, Hs);
    PDMK_LAUNCH_CHECK();
    PDMK_CUDA(cudaFreeAsync(d_meta, st_));
    PDMK_CUDA(cudaFreeAsync(d_outs, st_));
  }
  k_ewald_recip<<<unsigned(nblk_rec), TPB, 0, st_>>>(S, nk, dk, alpha, sums + nblk_real);
  PDMK_LAUNCH_CHECK();
  k_ewald_real<<<unsigned(nblk_real), RES_T, 0, st_>>>(D, le, ny, alpha, rc, sums);
  PDMK_LAUNCH_CHECK();
  k_sum<<<1, 1024, 0, st_>>>(sums, nblk_real, sums + nblk_real + nblk_rec);
  PDMK_LAUNCH_CHECK();
  k_sum<<<1, 1024, 0, st_>>>(sums + nblk_real, nblk_rec, sums + nblk_real + nblk_rec + 1);
  PDMK_LAUNCH_CHECK();
  k_sum_q2<<<1, 1024, 0, st_>>>(D.sq, D.n_slots, sums + nblk_real + nblk_rec + 2);
  PDMK_LAUNCH_CHECK();
  double r3[3];
  PDMK_CUDA(cudaMemcpyAsync(r3, sums + nblk_real + nblk_rec, sizeof(r3), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaFreeAsync(part, st_));
  PDMK_CUDA(cudaFreeAsync(S, st_));
  PDMK_CUDA(cudaFreeAsync(d_work, st_));
  PDMK_CUDA(cudaFreeAsync(sums, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  const double e_real = r3[0];
  const double e_rec = 2 * pi / (L_ * L_ * L_) * r3[1];
  const double e_self = -alpha / std::sqrt(pi) * r3[2];
  if (parts) {
    parts[0] = e_real;
    parts[1] = e_rec;
    parts[2] = e_self;
  }
  return e_real + e_rec + e_self;
}

}  // namespace pdmk
