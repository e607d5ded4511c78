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
// Both operands lie in [-1, 1] after the scaling below. Each value v is formed
// in FP64 and written in 32-bit fixed point, X = round(127 v 2^24), with one
// FMA (adding 1.5 * 2^52 rounds to an integer that lands in the low word),
// as four signed base-256 digits, X = a1 2^24 + a2 2^16 + a3 2^8 + a4 with
// every a_s in [-128, 127]: the bytes of Y = X + 0x808080 (folded into the
// FMA's constant) with the top bit of the three lower bytes flipped. Signed
// digits have zero mean, so the products left out below do not add up
// coherently over a box's particles. The ten slice products with s + t <= 5
// run as tcgen05.mma kind::i8 (signed 8-bit operands into exact 32-bit
// integer accumulators in TMEM), summed by order:
// acc_k = sum_{s+t=k} a_s b_t for k = 2..5. Integer accumulation is
// exact, so the sum over a box's particles adds no rounding at all; the
// accumulators are combined in FP64 at the end,
//   out = qmax / 127^2 (acc_2 + acc_3 / 2^8 + acc_4 / 2^16 + acc_5 / 2^24).
// The operand error is the rounding of X (2.3e-10 of the operand's range) and
// the dropped products (s + t > 5, below 1e-9 of the range). This is the slice
// splitting of Ozaki, Ogita and Oishi (error-free splitting of
// floating-point products) in the fixed-point form of Ootomo, Ozaki and
// Yokota (DGEMM on integer matrix multiplication units, 2024), applied to
// operands bounded by one.
//
// One CTA computes one 128-row M tile of one box (or split-K chunk of a box)
// and streams the box's particles through shared memory KCP at a time:
//   - producer warps: TMA (cp.async.bulk.tensor) brings the next chunk's
//     coordinates and charges into shared memory; the chunk's phase factors
//     are formed in FP64 (box-centred phases, exact sixth roots of unity for
//     the decentring; one task per particle, axis and half of the mode
//     range), and the B operand is sliced;
//   - consumer warps: one output row (kz, ky) per thread forms A = ez ey in
//     FP64 and slices it;
//   - one consumer thread issues the MMAs and commits them to an mbarrier;
//     the shared-memory stages are double-buffered, so the tensor core works
//     on chunk c while the warps build chunk c + 1;
//   - epilogue: tcgen05.ld of the accumulators, FP64 combination, staging
//     in shared memory and one bulk copy (cp.async.bulk) into the box's
//     expansion row range, which is contiguous in HBM.
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

constexpr int RPC = 128;  // rows (one M tile) per CTA, one consumer thread each
constexpr int NACC = 4;   // accumulators: slice-product orders s + t = 2 .. 5

// smem footprint of the pipeline for a chunk of kcp particles
__host__ __device__ constexpr int mix_pipe_bytes(int nk, int kcp) {
  return 2 * 4 * RPC * 2 * kcp                          // A stages: 4 slices x rows x K bytes
         + 2 * 4 * ((2 * (2 * nk + 1) + 15) / 16 * 16) * 2 * kcp  // B stages
         + 2 * kcp * (2 * (2 * nk + 1) + nk + 1) * 16    // FP64 factor stages (ex, ey, ez)
         + 2 * (((4 * (kcp + 2) * 8) + 127) / 128 * 128) // coordinate stages
         + 1024;                                         // alignment slack
}

template <int NK>
struct MixShape {
  static constexpr int D = 2 * NK + 1;
  static constexpr int ROWS = (NK + 1) * D;
  static constexpr int NPAD = (2 * D + 15) / 16 * 16;  // MMA N: Re columns [0, D), Im columns [HALF, HALF + D)
  static constexpr int HALF = NPAD / 2;
  static constexpr int TILES = (ROWS + RPC - 1) / RPC;  // CTAs per box
  // particles per chunk: 32 when the stages fit, else 16
  static constexpr int KCP = mix_pipe_bytes(NK, 32) <= 227 * 1024 ? 32 : 16;
  static constexpr int KB = 2 * KCP;                    // K bytes per chunk (real and imaginary part per particle)
  static constexpr int KSTEPS = KB / 32;                // MMA K steps (32 bytes each) per chunk
  static constexpr int PTHREADS = 6 * KCP;              // producers: one task per (particle, axis, half)
  static constexpr int THREADS = RPC + PTHREADS;
  static constexpr int COORD_BOX = KCP + 2;             // TMA box along the slots: even start, one spare each side
  static constexpr int COORD_BYTES = 4 * COORD_BOX * 8;
  static constexpr int COORD_STRIDE = (COORD_BYTES + 127) / 128 * 128;
  static constexpr int TCOLS_USED = NACC * NPAD;
  static constexpr int TCOLS = TCOLS_USED <= 32 ? 32 : TCOLS_USED <= 64 ? 64 : TCOLS_USED <= 128 ? 128
                               : TCOLS_USED <= 256 ? 256 : 512;
  // shared memory (bytes)
  static constexpr int A_SLICE = RPC * KB;
  static constexpr int B_SLICE = NPAD * KB;
  static constexpr int A_STAGE = 4 * A_SLICE;
  static constexpr int B_STAGE = 4 * B_SLICE;
  static constexpr int F_STAGE = KCP * (2 * D + NK + 1) * 16;  // ex, ey, ez as double2
  static constexpr int OFF_A = 0;
  static constexpr int OFF_B = OFF_A + 2 * A_STAGE;
  static constexpr int OFF_F = OFF_B + 2 * B_STAGE;
  static constexpr int OFF_P = (OFF_F + 2 * F_STAGE + 127) / 128 * 128;
  static constexpr int PIPE_BYTES = OFF_P + 2 * COORD_STRIDE;
  static constexpr int STAGE_OUT = RPC * D * 16;  // epilogue staging, reuses the pipeline buffers
  static constexpr int SMEM = (PIPE_BYTES > STAGE_OUT ? PIPE_BYTES : STAGE_OUT) + 1024;  // + alignment slack
  static_assert(TCOLS_USED <= 512, "accumulators exceed TMEM");
  static_assert(HALF >= D, "imaginary columns overlap the real ones");
  static_assert(SMEM <= 227 * 1024, "shared memory");
  static_assert(KB % 32 == 0, "chunks are whole MMA K steps");
  static_assert(PTHREADS % 32 == 0, "producer warps");
};

// named barrier ids
constexpr int BAR_FULL0 = 1, BAR_EMPTY0 = 3, BAR_CONS = 5, BAR_PROD = 6;

constexpr double SL_SCALE = 127.0;  // operands are scaled to |t| <= 127

// The signed base-256 digits of X = round(t 2^24), t in [-127, 127], as the
// four bytes of one word (top byte = highest digit): the low word of
// t 2^24 + 1.5 2^52 + 0x808080 is Y = X + 0x808080 (one FMA, exact to the
// rounding of t 2^24); with y_i the bytes of Y, X = y_3 2^24 + sum_{i<3}
// (y_i - 128) 256^i, and y_i - 128 is byte y_i with its top bit flipped.
__device__ __forceinline__ uint32_t fix24(double t) {
  return uint32_t(__double2loint(fma(t, 16777216.0, 6755399449477248.0))) ^ 0x808080u;
}

// bytes of four words transposed: out[b] = [w0.byte b, w1.byte b, w2.byte b, w3.byte b]
__device__ __forceinline__ void transpose4(uint32_t w0, uint32_t w1, uint32_t w2, uint32_t w3, uint32_t (&out)[4]) {
  const uint32_t l01 = __byte_perm(w0, w1, 0x5140), h01 = __byte_perm(w0, w1, 0x7362);
  const uint32_t l23 = __byte_perm(w2, w3, 0x5140), h23 = __byte_perm(w2, w3, 0x7362);
  out[0] = __byte_perm(l01, l23, 0x5410);
  out[1] = __byte_perm(l01, l23, 0x7632);
  out[2] = __byte_perm(h01, h23, 0x5410);
  out[3] = __byte_perm(h01, h23, 0x7632);
}

// exact int32 -> double without the conversion pipe: x + 2^31 as the low word
// of 1.5 2^52, less 1.5 2^52 + 2^31
__device__ __forceinline__ double i2d(uint32_t x) {
  return __hiloint2double(0x43380000, int(x ^ 0x80000000u)) - 6755401588539392.0;
}

__device__ __forceinline__ void st_shared_v4(uint32_t addr, uint32_t a, uint32_t b, uint32_t c, uint32_t d) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};\n" ::"r"(addr), "r"(a), "r"(b), "r"(c), "r"(d) : "memory");
}

__device__ __forceinline__ double2 cmul_d(double2 a, double2 b) {
  return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
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

// FP64 phase factors exp(-i m dk (x - c)) w6^{-M (2X+1) m} for m = m0 .. m0 + cnt - 1,
// times `scale`, into dst[0 .. cnt) (six interleaved recurrence chains, each
// with its own exact root of unity, as in the FP64 path)
__device__ void axis_factors_d(double xr, double dk, int M, int X, int m0, int cnt, double scale, double2* dst) {
  const double th = dk * xr;
  double s, c;
  sincos(-double(m0) * th, &s, &c);
  const double2 v0 = make_double2(c * scale, s * scale);
  sincos(-th, &s, &c);
  const double2 st = make_double2(c, s);
  const double2 st2 = cmul_d(st, st), st3 = cmul_d(st2, st), st6 = cmul_d(st3, st3);
  const int dec = M * (2 * X + 1);
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
        dst[t + r] = v[r];
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
  constexpr int D = S::D, NPAD = S::NPAD, HALF = S::HALF, KCP = S::KCP, KB = S::KB;
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
  int last_tma = -1;     // the last chunk whose coordinates were requested (producer thread 0)
  int last_commit = -1;  // the last chunk whose MMAs were committed (consumer thread 0)

  if (producer) {
    // ------------------------------------------------------------ producers
    if (ptid == 0 && nch > 0) {
      tc::tma_prefetch_desc(&coords);
      tc::mbar_arrive_expect_tx(&tma_bar[0], S::COORD_BYTES);
      tc::tma_load_2d(sm + S::OFF_P, &coords, it.s_begin & ~1, 0, &tma_bar[0]);
      last_tma = 0;
    }
    for (int c = 0; c < nch; ++c) {
      const int s = c & 1;
      const uint32_t u = uint32_t(c >> 1);
      if (c >= 2) tc::bar_sync(BAR_EMPTY0 + s, S::THREADS);
      wait_bar(&tma_bar[s], u & 1);
      const int sb = it.s_begin + c * KCP;
      const int nk = min(KCP, it.s_end - sb);
      const int off = sb - (sb & ~1);
      const double* P = reinterpret_cast<const double*>(sm + S::OFF_P + s * S::COORD_STRIDE);
      double2* ex = reinterpret_cast<double2*>(sm + S::OFF_F + s * S::F_STAGE);
      double2* ey = ex + KCP * D;
      double2* ez = ey + KCP * D;
      {
        // phase factors: one task per (particle, axis, half of the mode range)
        const int j = ptid / 6, a = (ptid >> 1) % 3, half = ptid & 1;
        const int len = a == 2 ? NK + 1 : D;
        const int h0 = (len + 1) / 2;
        const int m0 = half ? -NK + h0 : -NK, cnt = half ? len - h0 : h0;
        double2* dst = (a == 0 ? ex + j * D : (a == 1 ? ey + j * D : ez + j * (NK + 1))) + (m0 + NK);
        if (j < nk) {
          const double xa = P[a * S::COORD_BOX + off + j];
          const double ca = a == 0 ? it.cx : (a == 1 ? it.cy : it.cz);
          const int Xa = a == 0 ? it.X : (a == 1 ? it.Y : it.Z);
          const double scale =
              a == 0 ? SL_SCALE : (a == 1 ? 1.0 : SL_SCALE * P[3 * S::COORD_BOX + off + j] * inv_qmax);
          axis_factors_d(xa - ca, it.dk, it.M, Xa, m0, cnt, scale, dst);
        } else {
          for (int m = 0; m < cnt; ++m) dst[m] = make_double2(0.0, 0.0);
        }
      }
      tc::bar_sync(BAR_PROD, S::PTHREADS);
      // the next chunk's coordinates: its buffer was last read before the
      // previous producer barrier
      if (ptid == 0 && c + 1 < nch && !s_abort) {
        tc::mbar_arrive_expect_tx(&tma_bar[s ^ 1], S::COORD_BYTES);
        tc::tma_load_2d(sm + S::OFF_P + (s ^ 1) * S::COORD_STRIDE, &coords, (it.s_begin + (c + 1) * KCP) & ~1, 0,
                        &tma_bar[s ^ 1]);
        last_tma = c + 1;
      }
      // B operand: the MMAs of chunk c - 2 must have finished reading it
      if (c >= 2) wait_bar(&mma_bar[s], (u - 1) & 1);
      const uint32_t bbase = tc::smem_u32(sm + S::OFF_B + s * S::B_STAGE);
      for (int task = ptid; task < NPAD * (KB / 16); task += S::PTHREADS) {
        const int n = task % NPAD, kc = task / NPAD;
        uint32_t w[4][4];
        const bool re = n < D, im = n >= HALF && n < HALF + D;
        const int kx = re ? n : n - HALF;
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const int j0 = kc * 8 + 2 * p;
          double2 v0 = make_double2(0.0, 0.0), v1 = make_double2(0.0, 0.0);
          if (re || im) {
            const double2 e0 = ex[j0 * D + kx], e1 = ex[(j0 + 1) * D + kx];
            // K rows (2j, 2j+1) of a real output column: (Br, -Bi); of an imaginary one: (Bi, Br)
            v0 = re ? make_double2(e0.x, -e0.y) : make_double2(e0.y, e0.x);
            v1 = re ? make_double2(e1.x, -e1.y) : make_double2(e1.y, e1.x);
          }
          uint32_t by[4];
          transpose4(fix24(v0.x), fix24(v0.y), fix24(v1.x), fix24(v1.y), by);
#pragma unroll
          for (int sl = 0; sl < 4; ++sl) w[sl][p] = by[3 - sl];  // slice 0 = the top byte
        }
#pragma unroll
        for (int sl = 0; sl < 4; ++sl)
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
    for (int c = 0; c < nch; ++c) {
      const int s = c & 1;
      const uint32_t u = uint32_t(c >> 1);
      tc::bar_sync(BAR_FULL0 + s, S::THREADS);
      if (c >= 2) wait_bar(&mma_bar[s], (u - 1) & 1);
      const uint32_t abase = tc::smem_u32(sm + S::OFF_A + s * S::A_STAGE);
      if (active) {
        const double2* ey = reinterpret_cast<const double2*>(sm + S::OFF_F + s * S::F_STAGE) + KCP * D;
        const double2* ez = ey + KCP * D;
#pragma unroll 1
        for (int kc = 0; kc < KB / 16; ++kc) {
          uint32_t w[4][4];
#pragma unroll
          for (int p = 0; p < 4; ++p) {
            const int j0 = kc * 8 + 2 * p;
            const double2 v0 = cmul_d(ez[j0 * (NK + 1) + kz], ey[j0 * D + ky]);
            const double2 v1 = cmul_d(ez[(j0 + 1) * (NK + 1) + kz], ey[(j0 + 1) * D + ky]);
            uint32_t by[4];
            transpose4(fix24(v0.x), fix24(v0.y), fix24(v1.x), fix24(v1.y), by);
#pragma unroll
            for (int sl = 0; sl < 4; ++sl) w[sl][p] = by[3 - sl];
          }
#pragma unroll
          for (int sl = 0; sl < 4; ++sl)
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
#pragma unroll
        for (int ks = 0; ks < S::KSTEPS; ++ks) {
          const uint32_t ka = abase + ks * 2 * LBO_A;
          const uint32_t kb = bbase + ks * 2 * LBO_B;
          // slice products (a slice sa, b slice sb) of order sa + sb <= 3, into accumulator sa + sb
#pragma unroll
          for (int sa = 0; sa < 4; ++sa) {
#pragma unroll
            for (int sb2 = 0; sb2 + sa < 4; ++sb2) {
              const int k = sa + sb2;
              const uint32_t first = (c == 0 && ks == 0 && sa == 0) ? 0u : 1u;
              tc::mma_i8(tmem + uint32_t(k * NPAD), tc::smem_desc(ka + sa * S::A_SLICE, LBO_A, 128),
                         tc::smem_desc(kb + sb2 * S::B_SLICE, LBO_B, 128), tc::idesc_i8(RPC, NPAD), first);
            }
          }
        }
        tc::mma_commit(&mma_bar[s]);
        last_commit = c;
      }
    }
    // ------------------------------------------------------------ epilogue
    if (nch > 0) {
      const int cl = nch - 1;
      wait_bar(&mma_bar[cl & 1], uint32_t(cl >> 1) & 1);
    }
    tc::tc_fence_after();
    tc::bar_sync(BAR_CONS, RPC);  // every consumer is past its last shared-memory read of the pipeline
    const int q = warp & 3;       // TMEM lane quarter
    double2* stage = reinterpret_cast<double2*>(sm) + size_t(lr) * D;
    const double scale = qmax / (SL_SCALE * SL_SCALE);
    if (nch > 0 && !s_abort) {
#pragma unroll 1
      for (int cb = 0; cb < NPAD / 16; ++cb) {
        uint32_t a0[16], a1[16], a2[16], a3[16];
        const uint32_t ta = tmem + (uint32_t(32 * q) << 16) + uint32_t(cb * 16);
        tc::tmem_ld16(ta, a0);
        tc::tmem_ld16(ta + NPAD, a1);
        tc::tmem_ld16(ta + 2 * NPAD, a2);
        tc::tmem_ld16(ta + 3 * NPAD, a3);
        tc::tmem_ld_wait();
#pragma unroll
        for (int k = 0; k < 16; ++k) {
          const int n = cb * 16 + k;
          const double v = scale * fma(i2d(a3[k]), 1.0 / 16777216.0,
                                       fma(i2d(a2[k]), 1.0 / 65536.0, fma(i2d(a1[k]), 1.0 / 256.0, i2d(a0[k]))));
          if (n < D) stage[n].x = v;
          else if (n >= HALF && n < HALF + D) reinterpret_cast<double*>(stage + (n - HALF))[1] = v;
        }
      }
    } else {
      for (int n = 0; n < D; ++n) stage[n] = make_double2(0.0, 0.0);
    }
    tc::fence_async_smem();
    tc::bar_sync(BAR_CONS, RPC);
    if (tid == 0) {
      tc::bulk_store(it.out + size_t(row0) * D, sm, uint32_t(nrows) * D * 16u);
      tc::bulk_commit();
      tc::bulk_wait_all();
    }
  }
  // copies and MMAs this CTA started have ended (bounded waits; they only
  // matter when a pipeline wait gave up) before its TMEM is released
  if (ptid == 0 && last_tma >= 0) tc::mbar_wait(&tma_bar[last_tma & 1], uint32_t(last_tma >> 1) & 1);
  if (tid == 0 && last_commit >= 0) tc::mbar_wait(&mma_bar[last_commit & 1], uint32_t(last_commit >> 1) & 1);
  tc::tc_fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tmem, S::TCOLS);
}

// max |q| over the slots (the fixed-point scale of A): a grid-strided block
// maximum, then an atomic maximum on the bit patterns, whose integer order
// is the numeric order for non-negative doubles (*out must start at zero;
// the maximum does not depend on the order of the arrivals)
__global__ void k_absmax(const double* __restrict__ q, int n, double* out) {
  __shared__ double sm[32];
  double m = 0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, fabs(q[i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) t = fmax(t, sm[w]);
    atomicMax(reinterpret_cast<unsigned long long*>(out), static_cast<unsigned long long>(__double_as_longlong(t)));
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

int mixed_chunk(int nk) {
  switch (nk) {
    case 4: return MixShape<4>::KCP;
    case 6: return MixShape<6>::KCP;
    case 8: return MixShape<8>::KCP;
    case 12: return MixShape<12>::KCP;
    case 13: return MixShape<13>::KCP;
    case 17: return MixShape<17>::KCP;
    case 19: return MixShape<19>::KCP;
    case 26: return MixShape<26>::KCP;
    default: throw std::invalid_argument("mixed precision: unsupported mode count");
  }
}

int mixed_pairs(int nk) {
  switch (nk) {
    case 4: return MixShape<4>::TILES;
    case 6: return MixShape<6>::TILES;
    case 8: return MixShape<8>::TILES;
    case 12: return MixShape<12>::TILES;
    case 13: return MixShape<13>::TILES;
    case 17: return MixShape<17>::TILES;
    case 19: return MixShape<19>::TILES;
    case 26: return MixShape<26>::TILES;
    default: throw std::invalid_argument("mixed precision: unsupported mode count");
  }
}

void make_coord_map(CUtensorMap* map, const double* sx, int slot_capacity, int kcp) {
  if (slot_capacity % 2 != 0) throw std::logic_error("slot capacity must be even for the coordinate tensor map");
  // the four slot arrays x, y, z, q lie back to back with stride slot_capacity
  const cuuint64_t dims[2] = {cuuint64_t(slot_capacity), 4};
  const cuuint64_t strides[1] = {cuuint64_t(slot_capacity) * sizeof(double)};
  const cuuint32_t box[2] = {cuuint32_t(kcp + 2), 4};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = encode_fn()(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double*>(sx), dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed: " + std::to_string(int(r)));
}

void launch_absmax(const double* sq, int n, double* out, cudaStream_t st) {
  PDMK_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
  const int blocks = std::max(1, std::min(592, (n + 255) / 256));
  k_absmax<<<unsigned(blocks), 256, 0, st>>>(sq, n, out);
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
