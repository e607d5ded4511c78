// Mixed-precision outgoing plane-wave expansions on the 5th-generation tensor
// cores (tcgen05), for HPDMK_PRECISION_MIXED.
//
// Reference counterparts: the per-box direct NUDFT of the upward pass,
// nudft3d1_halfplane (include/nudft.hpp:95-121) as called by
// outgoing_pw_direct (src/planewave.cpp:48-84), and the root pass
// outgoing_pw_root (src/planewave.cpp:24-46, finufft in the reference).
//
// The outgoing expansion of a box over its particles j,
//   out[(kz,ky), kx] = sum_j A_j[(kz,ky)] B_j[kx],
//   A_j = q_j ez_j[kz] ey_j[ky],  B_j = ex_j[kx],  e*_j[m] = exp(-i m dk (x_j - c)),
// is one real matrix product over K = 2 x (particles):
//   [Re | Im](rows x 2d) = [Ar Ai](rows x 2K) . [[Br, Bi], [-Bi, Br]](2K x 2d).
// Both operands lie in [-1, 1] after the scaling below, so each is written in
// fixed point, t = 127 v, as three signed 8-bit slices in base 254,
// t = a1 + a2 / 254 + a3 / 254^2 (|a_s| <= 127; truncation 0.5 / 254^2 of t,
// 6e-8 of the operand's range, about the FP32 rounding of the operand
// itself). The six slice products with s + t <= 4 run as tcgen05.mma
// kind::i8 (int8 x int8 into exact int32 accumulators in TMEM):
// acc0 = a1 b1, acc1 = a1 b2 + a2 b1, acc2 = a1 b3 + a2 b2 + a3 b1. Integer
// accumulation is exact, so the sum over a box's particles adds no rounding
// at all; the three accumulators are combined in FP64 at the end,
// out = qmax / 127^2 (acc0 + acc1 / 254 + acc2 / 254^2). This is the slice
// splitting of Ozaki, Ogita and Oishi (error-free splitting of floating-point
// products) in the fixed-point form of Ootomo, Ozaki and Yokota (DGEMM on
// integer matrix multiplication units, 2024), applied to operands bounded by
// one.
//
// One CTA computes up to two 128-row M tiles of one box (or split-K chunk of
// a box) and streams the box's particles through shared memory 32 at a time:
//   - producer warps: TMA (cp.async.bulk.tensor) brings the next chunk's
//     coordinates and charges into shared memory; the chunk's phase factors
//     are formed in FP64 (box-centred phases, exact sixth roots of unity for
//     the decentring), rounded to FP32, and the B operand is sliced;
//   - consumer warps: one output row (kz, ky) per thread forms A = ez ey in
//     FP32 and slices it;
//   - one consumer thread issues the MMAs and commits them to an mbarrier;
//     the shared-memory stages are double-buffered, so the tensor core works
//     on chunk c while the warps build chunk c + 1;
//   - epilogue: tcgen05.ld of the accumulators, FP64 combination, staging
//     in shared memory and one bulk copy (cp.async.bulk) per M tile into the
//     box's expansion row range, which is contiguous in HBM.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>

#include "common.cuh"
#include "mixed.hpp"
#include "tc.cuh"

namespace pdmk {
namespace {

constexpr int KCP = 32;        // particles per pipeline chunk
constexpr int KB = 2 * KCP;    // K bytes per chunk (real and imaginary part per particle)
constexpr int PTHREADS = 128;  // producer threads (4 warps)
constexpr int COORD_BOX = KCP + 2;  // TMA box along the slots: even start, one spare element each side
constexpr int COORD_BYTES = 4 * COORD_BOX * 8;
constexpr int COORD_STRIDE = (COORD_BYTES + 127) / 128 * 128;

template <int NK>
struct MixShape {
  static constexpr int D = 2 * NK + 1;
  static constexpr int ROWS = (NK + 1) * D;
  static constexpr int NPAD = (2 * D + 15) / 16 * 16;  // MMA N: Re columns [0, D), Im columns [HALF, HALF + D)
  static constexpr int HALF = NPAD / 2;
  static constexpr int MTC = 3 * NPAD <= 256 ? 2 : 1;  // 128-row M tiles per CTA (TMEM: 3 NPAD columns each)
  static constexpr int RPC = 128 * MTC;                // rows per CTA, one consumer thread each
  static constexpr int PAIRS = (ROWS + RPC - 1) / RPC;  // CTAs per box
  static constexpr int THREADS = RPC + PTHREADS;
  static constexpr int TCOLS_USED = MTC * 3 * NPAD;
  static constexpr int TCOLS = TCOLS_USED <= 32 ? 32 : TCOLS_USED <= 64 ? 64 : TCOLS_USED <= 128 ? 128
                               : TCOLS_USED <= 256 ? 256 : 512;
  // shared memory (bytes)
  static constexpr int A_SLICE = RPC * KB;
  static constexpr int B_SLICE = NPAD * KB;
  static constexpr int A_STAGE = 3 * A_SLICE;
  static constexpr int B_STAGE = 3 * B_SLICE;
  static constexpr int F_STAGE = KCP * (2 * D + NK + 1) * 8;  // ex, ey, ez as float2
  static constexpr int OFF_A = 0;
  static constexpr int OFF_B = OFF_A + 2 * A_STAGE;
  static constexpr int OFF_F = OFF_B + 2 * B_STAGE;
  static constexpr int OFF_P = (OFF_F + 2 * F_STAGE + 127) / 128 * 128;
  static constexpr int PIPE_BYTES = OFF_P + 2 * COORD_STRIDE;
  static constexpr int STAGE_OUT = MTC * 128 * D * 16;  // epilogue staging, reuses the pipeline buffers
  static constexpr int SMEM = (PIPE_BYTES > STAGE_OUT ? PIPE_BYTES : STAGE_OUT) + 1024;  // + alignment slack
  static_assert(TCOLS_USED <= 512, "accumulators exceed TMEM");
  static_assert(HALF >= D, "imaginary columns overlap the real ones");
  static_assert(SMEM <= 227 * 1024, "shared memory");
};

// named barrier ids
constexpr int BAR_FULL0 = 1, BAR_EMPTY0 = 3, BAR_CONS = 5, BAR_PROD = 6;

constexpr float SL_BASE = 254.0f;  // slice base; operands are scaled to |t| <= 127
constexpr double SL_SCALE = 127.0;

// t in [-127, 127] -> three float words whose low bytes are the signed 8-bit
// slices a1, a2, a3 with t = a1 + a2 / 254 + a3 / 254^2 + e, |e| <= 0.5 / 254^2,
// for a pair of values (the real and imaginary part of one complex operand)
// with the paired FP32 instructions of sm_100 (one issue slot for both lanes,
// each lane rounded as its scalar instruction). Adding MAG = 1.5 * 2^23
// rounds to an integer that lands in the low mantissa bits; -round(t) =
// MAG - (t + MAG) is exact, t - a1 is exact, and each FMA forms r * 254 - a
// exactly before its one rounding.
__device__ __forceinline__ void slice3x2(float2 t, uint32_t (&re)[3], uint32_t (&im)[3]) {
  const float2 MAG2 = make_float2(12582912.0f, 12582912.0f);
  const float2 NEG1 = make_float2(-1.0f, -1.0f);
  const float2 B2 = make_float2(SL_BASE, SL_BASE);
  const float2 f1 = __fadd2_rn(t, MAG2);
  const float2 r1 = __fadd2_rn(t, __ffma2_rn(f1, NEG1, MAG2));
  const float2 f2 = __ffma2_rn(r1, B2, MAG2);
  const float2 r2 = __ffma2_rn(r1, B2, __ffma2_rn(f2, NEG1, MAG2));
  const float2 f3 = __ffma2_rn(r2, B2, MAG2);
  re[0] = __float_as_uint(f1.x);
  re[1] = __float_as_uint(f2.x);
  re[2] = __float_as_uint(f3.x);
  im[0] = __float_as_uint(f1.y);
  im[1] = __float_as_uint(f2.y);
  im[2] = __float_as_uint(f3.y);
}

// z y for complex FP32 operands with two paired instructions
__device__ __forceinline__ float2 cmul_x2(float2 z, float2 y) {
  const float2 p = __fmul2_rn(make_float2(z.x, z.x), y);               // (zr yr, zr yi)
  return __ffma2_rn(make_float2(-z.y, z.y), make_float2(y.y, y.x), p);  // (zr yr - zi yi, zr yi + zi yr)
}

// low bytes of four words -> one word [x0.b0, x1.b0, x2.b0, x3.b0]
__device__ __forceinline__ uint32_t pack4(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3) {
  const uint32_t lo = __byte_perm(x0, x1, 0x0040);
  const uint32_t hi = __byte_perm(x2, x3, 0x4000);
  return __byte_perm(lo, hi, 0x7610);
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// exact sixth roots of unity exp(i pi m / 3)
__device__ __forceinline__ double2 root6_d(int m) {
  m %= 6;
  if (m < 0) m += 6;
  const double h = 0.86602540378443864676;
  switch (m) {
    case 0: return make_double2(1.0, 0.0);
    case 1: return make_double2(0.5, h);
    case 2: return make_double2(-0.5, h);
    case 3: return make_double2(-1.0, 0.0);
    case 4: return make_double2(-0.5, -h);
    default: return make_double2(0.5, -h);
  }
}

// FP64 phase factors exp(-i m dk (x - c)) w6^{-M (2X+1) m} for m = -NK .. -NK + cnt - 1,
// scaled and rounded to FP32 (six interleaved recurrence chains, each with
// its own exact root of unity, as in the FP64 path)
__device__ void axis_factors_f32(double xr, double dk, int M, int X, int NK, int cnt, double scale, float2* dst) {
  const double th = dk * xr;
  double s, c;
  sincos(double(NK) * th, &s, &c);  // m0 = -NK: exp(-i m0 th) = exp(i NK th)
  const double2 v0 = make_double2(c * scale, s * scale);
  sincos(-th, &s, &c);
  const double2 st = make_double2(c, s);
  const double2 st2 = cmul_d(st, st), st3 = cmul_d(st2, st), st6 = cmul_d(st3, st3);
  const int dec = M * (2 * X + 1);
  const int m0 = -NK;
  double2 v[6];
  v[0] = v0;
  v[1] = cmul_d(v0, st);
  v[2] = cmul_d(v0, st2);
  v[3] = cmul_d(v0, st3);
  v[4] = cmul_d(v[1], st3);
  v[5] = cmul_d(v[2], st3);
#pragma unroll
  for (int r = 0; r < 6; ++r) v[r] = cmul_d(v[r], root6_d(-dec * (m0 + r)));
  for (int t = 0; t < cnt; t += 6) {
#pragma unroll
    for (int r = 0; r < 6; ++r) {
      if (t + r < cnt) {
        dst[t + r] = make_float2(float(v[r].x), float(v[r].y));
        v[r] = cmul_d(v[r], st6);
      }
    }
  }
}

template <int NK>
__global__ void __launch_bounds__(MixShape<NK>::THREADS, 1)
    k_pw_mixed(const __grid_constant__ CUtensorMap coords, const MixItem* __restrict__ items,
               const double* __restrict__ qmax_p, int* __restrict__ err) {
  using S = MixShape<NK>;
  constexpr int D = S::D, NPAD = S::NPAD, HALF = S::HALF, RPC = S::RPC, MTC = S::MTC;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* sm = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  __shared__ __align__(8) uint64_t mma_bar[2];
  __shared__ __align__(8) uint64_t tma_bar[2];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const bool producer = tid >= RPC;
  const int ptid = tid - RPC;
  const MixItem it = items[blockIdx.x];
  const int row0 = it.pair * RPC;
  const int nrows = min(RPC, S::ROWS - row0);  // valid rows of this CTA
  const int ntot = it.s_end - it.s_begin;
  const int nch = (ntot + KCP - 1) / KCP;
  const double qmax = *qmax_p;
  const double inv_qmax = qmax > 0.0 ? 1.0 / qmax : 0.0;

  if (tid == 0) {
    tc::mbar_init(&mma_bar[0], 1);
    tc::mbar_init(&mma_bar[1], 1);
    tc::mbar_init(&tma_bar[0], 1);
    tc::mbar_init(&tma_bar[1], 1);
    tc::mbar_fence_init();
    s_abort = 0;
  }
  if (warp == 0) tc::tmem_alloc(&s_tmem, S::TCOLS);
  tc::tc_fence_before();
  __syncthreads();
  tc::tc_fence_after();
  const uint32_t tmem = s_tmem;

  auto wait_bar = [&](uint64_t* bar, uint32_t parity) {
    if (*(volatile int*)&s_abort) return;
    if (!tc::mbar_wait(bar, parity)) {
      atomicOr(err, 4);
      s_abort = 1;
    }
  };

  if (producer) {
    // ------------------------------------------------------------ producers
    if (ptid == 0 && nch > 0) {
      tc::tma_prefetch_desc(&coords);
      const int x0 = it.s_begin & ~1;
      tc::mbar_arrive_expect_tx(&tma_bar[0], COORD_BYTES);
      tc::tma_load_2d(sm + S::OFF_P, &coords, x0, 0, &tma_bar[0]);
    }
    for (int c = 0; c < nch; ++c) {
      const int s = c & 1;
      const uint32_t u = uint32_t(c >> 1);
      if (c >= 2) tc::bar_sync(BAR_EMPTY0 + s, S::THREADS);
      wait_bar(&tma_bar[s], u & 1);
      const int sb = it.s_begin + c * KCP;
      const int nk = min(KCP, it.s_end - sb);
      const int off = sb - (sb & ~1);
      const double* P = reinterpret_cast<const double*>(sm + S::OFF_P + s * COORD_STRIDE);
      float2* ex = reinterpret_cast<float2*>(sm + S::OFF_F + s * S::F_STAGE);
      float2* ey = ex + KCP * D;
      float2* ez = ey + KCP * D;
      // phase factors: one task per (particle, axis)
      if (ptid < 3 * KCP) {
        const int j = ptid / 3, a = ptid % 3;
        const int len = a == 2 ? NK + 1 : D;
        float2* dst = a == 0 ? ex + j * D : (a == 1 ? ey + j * D : ez + j * (NK + 1));
        if (j < nk) {
          const double xa = P[a * COORD_BOX + off + j];
          const double ca = a == 0 ? it.cx : (a == 1 ? it.cy : it.cz);
          const int Xa = a == 0 ? it.X : (a == 1 ? it.Y : it.Z);
          const double scale = a == 0 ? SL_SCALE : (a == 1 ? 1.0 : SL_SCALE * P[3 * COORD_BOX + off + j] * inv_qmax);
          axis_factors_f32(xa - ca, it.dk, it.M, Xa, NK, len, scale, dst);
        } else {
          for (int m = 0; m < len; ++m) dst[m] = make_float2(0.f, 0.f);
        }
      }
      tc::bar_sync(BAR_PROD, PTHREADS);
      // the next chunk's coordinates: its buffer was last read before the
      // previous producer barrier
      if (ptid == 0 && c + 1 < nch && !s_abort) {
        const int x0 = (it.s_begin + (c + 1) * KCP) & ~1;
        tc::mbar_arrive_expect_tx(&tma_bar[s ^ 1], COORD_BYTES);
        tc::tma_load_2d(sm + S::OFF_P + (s ^ 1) * COORD_STRIDE, &coords, x0, 0, &tma_bar[s ^ 1]);
      }
      // B operand: the MMAs of chunk c - 2 must have finished reading it
      if (c >= 2) wait_bar(&mma_bar[s], (u - 1) & 1);
      const uint32_t bbase = tc::smem_u32(sm + S::OFF_B + s * S::B_STAGE);
      for (int task = ptid; task < NPAD * (KB / 16); task += PTHREADS) {
        const int n = task % NPAD, kc = task / NPAD;
        uint32_t w[3][4];
        const bool re = n < D, im = n >= HALF && n < HALF + D;
        const int kx = re ? n : n - HALF;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const int j0 = kc * 8 + 2 * p;
          float2 v0 = make_float2(0.f, 0.f), v1 = make_float2(0.f, 0.f);
          if (re || im) {
            const float2 e0 = ex[j0 * D + kx], e1 = ex[(j0 + 1) * D + kx];
            // K rows (2j, 2j+1) of a real output column: (Br, -Bi); of an imaginary one: (Bi, Br)
            v0 = re ? make_float2(e0.x, -e0.y) : make_float2(e0.y, e0.x);
            v1 = re ? make_float2(e1.x, -e1.y) : make_float2(e1.y, e1.x);
          }
          uint32_t a0[3], b0[3], a1[3], b1[3];
          slice3x2(v0, a0, b0);
          slice3x2(v1, a1, b1);
#pragma unroll
          for (int sl = 0; sl < 3; ++sl) w[sl][p] = pack4(a0[sl], b0[sl], a1[sl], b1[sl]);
        }
#pragma unroll
        for (int sl = 0; sl < 3; ++sl)
          st_shared_v4(bbase + sl * S::B_SLICE + kc * (NPAD * 16) + n * 16, w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
      }
      tc::fence_async_smem();
      tc::bar_arrive(BAR_FULL0 + s, S::THREADS);
    }
  } else {
    // ------------------------------------------------------------ consumers
    const int lr = tid;  // local row
    const int r = row0 + lr;
    const bool active = lr < nrows;
    const int kz = active ? r / D : 0, ky = active ? r % D : 0;
    const uint32_t id = tc::idesc_i8(128, NPAD);
    for (int c = 0; c < nch; ++c) {
      const int s = c & 1;
      const uint32_t u = uint32_t(c >> 1);
      tc::bar_sync(BAR_FULL0 + s, S::THREADS);
      if (c >= 2) wait_bar(&mma_bar[s], (u - 1) & 1);
      const uint32_t abase = tc::smem_u32(sm + S::OFF_A + s * S::A_STAGE);
      if (active) {
        const float2* ey = reinterpret_cast<const float2*>(sm + S::OFF_F + s * S::F_STAGE) + KCP * D;
        const float2* ez = ey + KCP * D;
#pragma unroll 1
        for (int kc = 0; kc < KB / 16; ++kc) {
          uint32_t w[3][4];
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const int j0 = kc * 8 + 2 * p;
            const float2 v0 = cmul_x2(ez[j0 * (NK + 1) + kz], ey[j0 * D + ky]);
            const float2 v1 = cmul_x2(ez[(j0 + 1) * (NK + 1) + kz], ey[(j0 + 1) * D + ky]);
            uint32_t a0r[3], a0i[3], a1r[3], a1i[3];
            slice3x2(v0, a0r, a0i);
            slice3x2(v1, a1r, a1i);
#pragma unroll
            for (int sl = 0; sl < 3; ++sl) w[sl][p] = pack4(a0r[sl], a0i[sl], a1r[sl], a1i[sl]);
          }
#pragma unroll
          for (int sl = 0; sl < 3; ++sl)
            st_shared_v4(abase + sl * S::A_SLICE + kc * (RPC * 16) + lr * 16, w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
        }
      }
      tc::fence_async_smem();
      if (c + 2 < nch) tc::bar_arrive(BAR_EMPTY0 + s, S::THREADS);
      tc::bar_sync(BAR_CONS, RPC);
      if (tid == 0 && !s_abort) {
        tc::tc_fence_after();
        const uint32_t bbase = tc::smem_u32(sm + S::OFF_B + s * S::B_STAGE);
        constexpr uint32_t LBO_A = RPC * 16, LBO_B = NPAD * 16;
        for (int t = 0; t < MTC; ++t) {
          if (t * 128 >= nrows) break;
#pragma unroll
          for (int ks = 0; ks < KB / 32; ++ks) {
            const uint32_t ka = abase + t * (16 * 128) + ks * 2 * LBO_A;
            const uint32_t kb = bbase + ks * 2 * LBO_B;
            const uint32_t first = (c == 0 && ks == 0) ? 0u : 1u;
            // (a slice, b slice) -> accumulator a + b
            const uint32_t d0 = tmem + uint32_t((t * 3 + 0) * NPAD);
            const uint32_t d1 = tmem + uint32_t((t * 3 + 1) * NPAD);
            const uint32_t d2 = tmem + uint32_t((t * 3 + 2) * NPAD);
            const uint64_t A0 = tc::smem_desc(ka, LBO_A, 128), A1 = tc::smem_desc(ka + S::A_SLICE, LBO_A, 128),
                           A2 = tc::smem_desc(ka + 2 * S::A_SLICE, LBO_A, 128);
            const uint64_t B0 = tc::smem_desc(kb, LBO_B, 128), B1 = tc::smem_desc(kb + S::B_SLICE, LBO_B, 128),
                           B2 = tc::smem_desc(kb + 2 * S::B_SLICE, LBO_B, 128);
            tc::mma_i8(d0, A0, B0, id, first);
            tc::mma_i8(d1, A0, B1, id, first);
            tc::mma_i8(d1, A1, B0, id, 1u);
            tc::mma_i8(d2, A0, B2, id, first);
            tc::mma_i8(d2, A1, B1, id, 1u);
            tc::mma_i8(d2, A2, B0, id, 1u);
          }
        }
        tc::mma_commit(&mma_bar[s]);
      }
    }
    // ------------------------------------------------------------ epilogue
    if (nch > 0) {
      const int cl = nch - 1;
      wait_bar(&mma_bar[cl & 1], uint32_t(cl >> 1) & 1);
    }
    tc::tc_fence_after();
    tc::bar_sync(BAR_CONS, RPC);  // every consumer is past its last shared-memory read of the pipeline
    const int t = warp >> 2;      // M tile of this warp
    const int q = warp & 3;       // TMEM lane quarter
    const int lt = lr & 127;      // row within the tile
    double2* stage = reinterpret_cast<double2*>(sm) + size_t(t * 128 + lt) * D;
    const double scale = qmax / (SL_SCALE * SL_SCALE);
    if (t * 128 < nrows) {
      if (nch > 0 && !s_abort) {
#pragma unroll 1
        for (int cb = 0; cb < NPAD / 16; ++cb) {
          uint32_t r0[16], r1[16], r2[16];
          const uint32_t ta = tmem + (uint32_t(32 * q) << 16) + uint32_t(t * 3 * NPAD + cb * 16);
          tc::tmem_ld16(ta, r0);
          tc::tmem_ld16(ta + NPAD, r1);
          tc::tmem_ld16(ta + 2 * NPAD, r2);
          tc::tmem_ld_wait();
#pragma unroll
          for (int k = 0; k < 16; ++k) {
            const int n = cb * 16 + k;
            const double v = scale * fma(double(int(r2[k])), 1.0 / (254.0 * 254.0),
                                         fma(double(int(r1[k])), 1.0 / 254.0, double(int(r0[k]))));
            if (n < D) stage[n].x = v;
            else if (n >= HALF && n < HALF + D) reinterpret_cast<double*>(stage + (n - HALF))[1] = v;
          }
        }
      } else {
        for (int n = 0; n < D; ++n) stage[n] = make_double2(0.0, 0.0);
      }
    }
    tc::fence_async_smem();
    tc::bar_sync(BAR_CONS, RPC);
    if (tid == 0) {
      for (int tt = 0; tt < MTC; ++tt) {
        const int rows = min(128, nrows - tt * 128);
        if (rows <= 0) break;
        tc::bulk_store(it.out + size_t(row0 + tt * 128) * D, reinterpret_cast<const double2*>(sm) + size_t(tt * 128) * D,
                       uint32_t(rows) * D * 16u);
      }
      tc::bulk_commit();
      tc::bulk_wait_all();
    }
  }
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TCOLS);
}

// max |q| over the slots, one block, fixed order (the fixed-point scale of A)
__global__ void k_absmax(const double* __restrict__ q, int n, double* out) {
  __shared__ double sm[32];
  double m = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs(q[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmax(t, sm[w]);
    *out = t;
  }
}

template <int NK>
void launch_mixed(const CUtensorMap& tmap, const MixItem* d_items, int nitems, const double* d_qmax, int* d_err,
                  cudaStream_t st) {
  using S = MixShape<NK>;
  if (nitems == 0) return;
  raise_smem_limit(reinterpret_cast<const void*>(k_pw_mixed<NK>), S::SMEM);
  k_pw_mixed<NK><<<unsigned(nitems), S::THREADS, S::SMEM, st>>>(tmap, d_items, d_qmax, d_err);
  PDMK_LAUNCH_CHECK();
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    PDMK_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q));
    if (!p || q != cudaDriverEntryPointSuccess) throw CudaError("cuTensorMapEncodeTiled is not available");
    return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }();
  return fn;
}

}  // namespace

int mixed_pairs(int nk) {
  switch (nk) {
    case 4: return MixShape<4>::PAIRS;
    case 6: return MixShape<6>::PAIRS;
    case 8: return MixShape<8>::PAIRS;
    case 12: return MixShape<12>::PAIRS;
    case 13: return MixShape<13>::PAIRS;
    case 17: return MixShape<17>::PAIRS;
    case 19: return MixShape<19>::PAIRS;
    case 26: return MixShape<26>::PAIRS;
    default: throw std::invalid_argument("mixed precision: unsupported mode count");
  }
}

void make_coord_map(CUtensorMap* map, const double* sx, int slot_capacity) {
  if (slot_capacity % 2 != 0) throw std::logic_error("slot capacity must be even for the coordinate tensor map");
  // the four slot arrays x, y, z, q lie back to back with stride slot_capacity
  const cuuint64_t dims[2] = {cuuint64_t(slot_capacity), 4};
  const cuuint64_t strides[1] = {cuuint64_t(slot_capacity) * sizeof(double)};
  const cuuint32_t box[2] = {cuuint32_t(COORD_BOX), 4};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(sx), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
}

void launch_absmax(const double* sq, int n, double* out, cudaStream_t st) {
  k_absmax<<<1, 1024, 0, st>>>(sq, n, out);
  PDMK_LAUNCH_CHECK();
}

void dispatch_mixed(int nk, const CUtensorMap& tmap, const MixItem* d_items, int nitems, const double* d_qmax,
                    int* d_err, cudaStream_t st) {
  switch (nk) {
    case 4: launch_mixed<4>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 6: launch_mixed<6>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 8: launch_mixed<8>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 12: launch_mixed<12>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 13: launch_mixed<13>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 17: launch_mixed<17>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 19: launch_mixed<19>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    case 26: launch_mixed<26>(tmap, d_items, nitems, d_qmax, d_err, st); break;
    default: throw std::invalid_argument("mixed precision: unsupported mode count");
  }
}

}  // namespace pdmk
