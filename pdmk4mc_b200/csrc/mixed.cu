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
// in FP64 and written in 32-bit fixed point, X = round(127 v 2^24) (adding
// 1.5 * 2^52 rounds to an integer that lands in the low word): one FMA for
// B; for A the product's two terms are added into that constant by two
// FMAs, each rounding to an integer (ez carries the factor 2^24), so X is
// within one unit instead of half a unit. X is written
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
// The operand error is the rounding of X (2.3e-10 of the operand's range for
// B, twice that at most for A) and
// the dropped products (s + t > 5, below 1e-9 of the range). This is the slice
// splitting of Ozaki, Ogita and Oishi (error-free splitting of
// floating-point products) in the fixed-point form of Ootomo, Ozaki and
// Yokota (DGEMM on integer matrix multiplication units, 2024), applied to
// operands bounded by one.
//
// Two kernels per pass:
//   - k_pw_tables, one CTA per 32-particle chunk of a box: TMA
//     (cp.async.bulk.tensor) brings the chunk's coordinates and charges into
//     shared memory; the phase factors are formed in FP64 (box-centred
//     phases, exact sixth roots of unity for the decentring; one thread per
//     particle, axis and half of the mode range), the B operand is sliced
//     into the tensor core's shared-memory layout, and the block (B slices,
//     ey and ez factors) goes to HBM with one bulk copy. Every M tile of the
//     box reads these once-formed tables.
//   - k_pw_mixed, one CTA per 128-row M tile of a box (or split-K chunk): a
//     control warp brings each chunk's table block into shared memory with a
//     bulk copy (three or four chunks in flight) and issues the MMAs, A from
//     tensor memory and B from shared memory; the consumer warps form
//     A = ez ey in FP64, one thread per output row (kz, ky) and group of 8
//     particles, slice it and store the slices into tensor memory
//     (tcgen05.st), which keeps A's traffic off shared memory; the A stages
//     are double-buffered, so the tensor core works on chunk c while the
//     consumers build chunk c + 1; the
//     epilogue reads the accumulators (tcgen05.ld), combines them in FP64,
//     stages the rows in shared memory and writes them with one bulk copy
//     into the box's expansion row range, which is contiguous in HBM.
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

constexpr int RPC = 128;           // rows (one M tile) per CTA
constexpr int NACC = 4;            // accumulators: slice-product orders s + t = 2 .. 5
constexpr int SMEM_MAX = 227 * 1024;

__host__ __device__ constexpr int npad_of(int nk) { return (2 * (2 * nk + 1) + 15) / 16 * 16; }
__host__ __device__ constexpr int ezs_of(int nk) { return (nk + 1) | 1; }
// bytes of one chunk's table block: B slices, then the ey and ez factors
__host__ __device__ constexpr int table_bytes(int nk, int kcp) {
  return 4 * npad_of(nk) * 2 * kcp + kcp * ((2 * nk + 1) + ezs_of(nk)) * 16;
}
__host__ __device__ constexpr int table_stride(int nk, int kcp) { return (table_bytes(nk, kcp) + 127) / 128 * 128; }
// TMEM columns: the four accumulators, then two A stages of 2 kcp columns
// (four slices of 2 kcp bytes per row, four bytes to a column)
__host__ __device__ constexpr int tmem_cols(int nk, int kcp) { return NACC * npad_of(nk) + 2 * 2 * kcp; }
// chunks of 32 particles when three table stages and the TMEM columns fit
__host__ __device__ constexpr bool chunk32_fits(int nk) {
  return 3 * table_stride(nk, 32) + 1024 <= SMEM_MAX && tmem_cols(nk, 32) <= 512;
}

template <int NK>
struct MixShape {
  static constexpr int D = 2 * NK + 1;
  static constexpr int ROWS = (NK + 1) * D;  // row r = kz D + ky, as the expansion's layout
  // rows computed: the kz < 0 planes whole, the kz = 0 plane for ky >= 0
  // only; its ky < 0 rows follow by conjugate symmetry (real charges:
  // out(-k) = conj(out(k))). Computed row rho maps to r = rho below NK D and
  // to r = rho + NK above.
  static constexpr int ROWS_C = NK * D + NK + 1;
  static_assert(ROWS_C <= ROWS, "computed rows");
  static constexpr int NPAD = npad_of(NK);  // MMA N: Re columns [0, D), Im columns [HALF, HALF + D)
  static constexpr int HALF = NPAD / 2;
  static constexpr int EZS = ezs_of(NK);    // odd row strides keep 16-byte stores on distinct bank groups
  static constexpr int TILES = (ROWS_C + RPC - 1) / RPC;  // CTAs per box
  static constexpr int KCP = chunk32_fits(NK) ? 32 : 16;  // particles per chunk
  static constexpr int KB = 2 * KCP;        // K bytes per chunk (real and imaginary part per particle)
  static constexpr int KSTEPS = KB / 32;    // MMA K steps (32 bytes each) per chunk
  static constexpr int CPR = KB / 16;            // consumer threads per row: one per 16-byte K group (8 particles)
  static constexpr int CTHREADS = RPC * CPR;
  static constexpr int THREADS = CTHREADS + 32;  // consumers + the control warp
  static constexpr int TTHREADS = 6 * KCP;       // table kernel: one thread per (particle, axis, half)
  static constexpr int COORD_BOX = KCP + 2;      // TMA box along the slots: even start, one spare each side
  static constexpr int COORD_BYTES = 4 * COORD_BOX * 8;
  // TMEM: accumulators at columns [0, NACC NPAD), A stage s slice t at
  // columns A_COL0 + s KB + t KB / 4 (lane = row)
  static constexpr int A_COL0 = NACC * NPAD;
  static constexpr int TCOLS_USED = tmem_cols(NK, KCP);
  static constexpr int TCOLS = TCOLS_USED <= 32 ? 32 : TCOLS_USED <= 64 ? 64 : TCOLS_USED <= 128 ? 128
                               : TCOLS_USED <= 256 ? 256 : 512;
  // one chunk's table block
  // B: the four slices side by side along N ([16-byte K group][slice][column]
  // [16 bytes]), so that one MMA can take up to BGROUP consecutive slices
  static constexpr int B_KGROUP = 4 * NPAD * 16;  // bytes per 16-byte K group
  static constexpr int B_BYTES = (KB / 16) * B_KGROUP;
  static constexpr int BGROUP = 3 * NPAD <= 256 ? 3 : 2;  // slices per MMA (N <= 256)
  // then the FP64 factors (double2): ey [particle][ky], ez [particle][kz]
  static constexpr int EY_OFF = B_BYTES;
  static constexpr int EZ_OFF = EY_OFF + KCP * D * 16;
  static constexpr int T_BYTES = EZ_OFF + KCP * EZS * 16;
  static constexpr int T_STRIDE = table_stride(NK, KCP);
  // contraction kernel shared memory: the table stages (four when they fit)
  static constexpr int TSTAGES = 4 * T_STRIDE + 1024 <= SMEM_MAX ? 4 : 3;
  static constexpr int PIPE_BYTES = TSTAGES * T_STRIDE;
  static constexpr int STAGE_OUT = RPC * D * 16;  // epilogue staging, reuses the table stages
  static constexpr int SMEM = (PIPE_BYTES > STAGE_OUT ? PIPE_BYTES : STAGE_OUT) + 1024;  // + alignment slack
  // table kernel shared memory: coordinates, ex scratch, the block
  static constexpr int TK_COORD_STRIDE = (COORD_BYTES + 127) / 128 * 128;  // two coordinate buffers
  static constexpr int TK_OFF_EX = 2 * TK_COORD_STRIDE;
  static constexpr int TK_OFF_T = (TK_OFF_EX + KCP * D * 16 + 127) / 128 * 128;
  static constexpr int TK_SMEM = TK_OFF_T + T_STRIDE + 1024;
  static_assert(TCOLS_USED <= 512, "accumulators and A stages exceed TMEM");
  static_assert(HALF >= D, "imaginary columns overlap the real ones");
  static_assert(SMEM <= SMEM_MAX && TK_SMEM <= SMEM_MAX, "shared memory");
  static_assert(KB % 32 == 0, "chunks are whole MMA K steps");
  static_assert(T_BYTES % 16 == 0, "bulk copies move multiples of 16 bytes");
};

// named barrier ids: A stage s ready (consumers -> control), consumers only
constexpr int BAR_AREADY0 = 1, BAR_CONS = 5;

constexpr double SL_SCALE = 127.0;  // operands are scaled to |t| <= 127

// The signed base-256 digits of X = round(t 2^24), t in [-127, 127], as the
// four bytes of one word (top byte = highest digit): the low word of
// t 2^24 + 1.5 2^52 + 0x808080 is Y = X + 0x808080 (one FMA, exact to the
// rounding of t 2^24); with y_i the bytes of Y, X = y_3 2^24 + sum_{i<3}
// (y_i - 128) 256^i, and y_i - 128 is byte y_i with its top bit flipped.
__device__ __forceinline__ uint32_t fix24(double t) {
  return uint32_t(__double2loint(fma(t, 16777216.0, 6755399449477248.0))) ^ 0x808080u;
}

// The digits word of X = round(a b + round(c d)) for |a b + c d| 2^-24 <= 127
// with a, b, c, d already carrying the factor 2^24: two FMAs into the
// rounding constant of fix24 (each rounds to an integer, so X is within one
// unit of (a b + c d) instead of half a unit)
__device__ __forceinline__ uint32_t fix24_dot(double a, double b, double c, double d) {
  return uint32_t(__double2loint(fma(a, b, fma(c, d, 6755399449477248.0)))) ^ 0x808080u;
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

// sin and cos of th, |th| <= pi (slots hold particles inside their box, or
// the leaf centre when empty, so th = dk (x - c) stays in range: |th| <= pi / 3
// at the difference levels, <= pi at the root): the Taylor series of sin and
// cos at h = th / 2 (|h| <= pi / 2; the first omitted terms are below 1e-19)
// as two Horner chains in h^2, then the double-angle formulas
__device__ __forceinline__ void sincos_taylor(double th, double& s, double& c) {
  const double h = 0.5 * th, h2 = h * h;
  double ps = 6.446950284384474e-26, pc = 1.6117375710961184e-24;
  ps = fma(ps, h2, -3.868170170630684e-23);
  pc = fma(pc, h2, -8.896791392450574e-22);
  ps = fma(ps, h2, 1.9572941063391263e-20);
  pc = fma(pc, h2, 4.110317623312165e-19);
  ps = fma(ps, h2, -8.22063524662433e-18);
  pc = fma(pc, h2, -1.5619206968586225e-16);
  ps = fma(ps, h2, 2.8114572543455206e-15);
  pc = fma(pc, h2, 4.779477332387385e-14);
  ps = fma(ps, h2, -7.647163731819816e-13);
  pc = fma(pc, h2, -1.1470745597729725e-11);
  ps = fma(ps, h2, 1.6059043836821613e-10);
  pc = fma(pc, h2, 2.08767569878681e-09);
  ps = fma(ps, h2, -2.505210838544172e-08);
  pc = fma(pc, h2, -2.755731922398589e-07);
  ps = fma(ps, h2, 2.7557319223985893e-06);
  pc = fma(pc, h2, 2.48015873015873e-05);
  ps = fma(ps, h2, -0.0001984126984126984);
  pc = fma(pc, h2, -0.001388888888888889);
  ps = fma(ps, h2, 0.008333333333333333);
  pc = fma(pc, h2, 0.041666666666666664);
  ps = fma(ps, h2, -0.16666666666666666);
  pc = fma(pc, h2, -0.5);
  ps = fma(ps, h2, 1.0);
  pc = fma(pc, h2, 1.0);
  const double sh = ps * h;  // sin(h)
  s = 2.0 * sh * pc;         // sin(2h) = 2 sin(h) cos(h)
  c = fma(-2.0 * sh, sh, 1.0);  // cos(2h) = 1 - 2 sin(h)^2
}

// FP64 phase factors exp(-i m dk (x - c)) w6^{-M (2X+1) m} for m = m0 .. m0 + cnt - 1,
// times `scale`, into dst[0 .. cnt): the step exp(-i th), the start
// exp(-i m0 th) by binary powering of the step (|m0| <= 26: at most five
// squarings), then six interleaved recurrence chains, each with its own
// exact root of unity, as in the FP64 path
__device__ void axis_factors_d(double xr, double dk, int M, int X, int m0, int cnt, double scale, double2* dst) {
  const double th = dk * xr;
  double s, c;
  sincos_taylor(-th, s, c);
  const double2 st = make_double2(c, s);
  double2 v0 = make_double2(scale, 0.0);
  {
    double2 w = m0 < 0 ? make_double2(c, -s) : st;  // exp(+i th) for negative powers
    for (int e = m0 < 0 ? -m0 : m0; e; e >>= 1) {
      if (e & 1) v0 = cmul_d(v0, w);
      w = cmul_d(w, w);
    }
  }
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



// Table pass: the FP64 phase factors of a chunk of a box, the sliced B
// operand in the tensor core's K-major layout and the ey, ez factors,
// written to the chunk's table block. Persistent: a CTA walks the chunks
// blockIdx.x, blockIdx.x + gridDim.x, ...; the next chunk's coordinates come
// in by TMA into the second coordinate buffer while the current chunk is
// formed, and a block's bulk store to HBM runs on while the next chunk's
// factors are formed (only its read of the block is awaited before the
// block is reused). One thread per (particle, axis, half of the mode range),
// consecutive lanes on consecutive particles.
template <int NK>
__global__ void __launch_bounds__(MixShape<NK>::TTHREADS)
    k_pw_tables(const __grid_constant__ CUtensorMap coords, const MixItem* __restrict__ items,
                const int2* __restrict__ chunks, int nchunks, const double* __restrict__ qmax_p,
                int* __restrict__ err) {
  using S = MixShape<NK>;
  constexpr int D = S::D, NPAD = S::NPAD, HALF = S::HALF, KCP = S::KCP, KB = S::KB;
  extern __shared__ unsigned char smem_raw[];
  // the 1024-aligned base as an offset from the shared array, so that the
  // compiler keeps shared-memory (not generic) loads and stores
  unsigned char* sm = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
  __shared__ __align__(8) uint64_t bar[2];
  const int tid = threadIdx.x;
  const double qmax = *qmax_p;
  const double inv_qmax = qmax > 0.0 ? 1.0 / qmax : 0.0;
  double2* ex = reinterpret_cast<double2*>(sm + S::TK_OFF_EX);
  unsigned char* blk = sm + S::TK_OFF_T;
  double2* ey = reinterpret_cast<double2*>(blk + S::EY_OFF);
  double2* ez = reinterpret_cast<double2*>(blk + S::EZ_OFF);
  auto chunk_start = [&](int q) {
    const int2 c = chunks[q];
    return items[c.x].s_begin + c.y * KCP;
  };
  auto load_coords = [&](int q, int b) {  // thread 0: chunk q's coordinates into buffer b
    tc::mbar_arrive_expect_tx(&bar[b], S::COORD_BYTES);
    tc::tma_load_2d(sm + b * S::TK_COORD_STRIDE, &coords, chunk_start(q) & ~1, 0, &bar[b]);
  };
  if (tid == 0) {
    tc::mbar_init(&bar[0], 1);
    tc::mbar_init(&bar[1], 1);
    tc::mbar_fence_init();
  }
  __syncthreads();
  if (tid == 0 && int(blockIdx.x) < nchunks) load_coords(blockIdx.x, 0);
  int i = 0;
  for (int q = blockIdx.x; q < nchunks; q += gridDim.x, ++i) {
    const int b = i & 1;
    const int2 ch = chunks[q];
    const MixItem it = items[ch.x];
    const int sb = it.s_begin + ch.y * KCP;
    const int nk = min(KCP, it.s_end - sb);
    const int off = sb - (sb & ~1);
    const double* P = reinterpret_cast<const double*>(sm + b * S::TK_COORD_STRIDE);
    if (tid == 0) {
      // the other buffer's last reader finished before the previous
      // iteration's last barrier
      if (q + int(gridDim.x) < nchunks) load_coords(q + gridDim.x, b ^ 1);
      // the previous chunk's store has read the block
      tc::bulk_wait_read_all();
    }
    // bounded; the zero-filled buffer is then still read safely
    if (!tc::mbar_wait(&bar[b], uint32_t(i >> 1) & 1)) atomicOr(err, 4);
    __syncthreads();
    {
      const int j = tid % KCP, ah = tid / KCP, a = ah >> 1, half = ah & 1;
      const int len = a == 2 ? NK + 1 : D;
      const int h0 = (len + 1) / 2;
      const int m0 = half ? -NK + h0 : -NK, cnt = half ? len - h0 : h0;
      double2* dst = (a == 0 ? ex + j * D : (a == 1 ? ey + j * D : ez + j * S::EZS)) + (m0 + NK);
      if (j < nk) {
        const double xa = P[a * S::COORD_BOX + off + j];
        const double ca = a == 0 ? it.cx : (a == 1 ? it.cy : it.cz);
        const int Xa = a == 0 ? it.X : (a == 1 ? it.Y : it.Z);
        // ex: 127 (B); ey: 1; ez: 127 q / max|q| times 2^24, so that A's
        // fixed point is formed by fix24_dot without a further scaling
        const double scale =
            a == 0 ? SL_SCALE : (a == 1 ? 1.0 : SL_SCALE * 16777216.0 * P[3 * S::COORD_BOX + off + j] * inv_qmax);
        axis_factors_d(xa - ca, it.dk, it.M, Xa, m0, cnt, scale, dst);
      } else {
        for (int m = 0; m < cnt; ++m) dst[m] = make_double2(0.0, 0.0);
      }
    }
    __syncthreads();
    // B operand from ex: column n < D of each slice is the real part of mode
    // kx = n, column HALF + kx its imaginary part; K rows (2j, 2j+1) carry
    // (Br, -Bi) for a real column and (Bi, Br) for an imaginary one
    const uint32_t bbase = tc::smem_u32(blk);
    for (int task = tid; task < NPAD * (KB / 16); task += S::TTHREADS) {
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
        st_shared_v4(bbase + kc * S::B_KGROUP + (sl * NPAD + n) * 16, w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
    }
    tc::fence_async_smem();
    __syncthreads();
    if (tid == 0) {
      tc::bulk_store(const_cast<unsigned char*>(it.tab) + size_t(ch.y) * S::T_BYTES, blk, S::T_BYTES);
      tc::bulk_commit();
    }
  }
  // the stores complete before the CTA ends
  if (tid == 0) tc::bulk_wait_all();
}

// Contraction: one 128-row M tile of one box (or split-K chunk) over its
// chunks' table blocks.
template <int NK>
__global__ void __launch_bounds__(MixShape<NK>::THREADS, 1)
    k_pw_mixed(const MixItem* __restrict__ items, const double* __restrict__ qmax_p, int* __restrict__ err) {
  using S = MixShape<NK>;
  constexpr int D = S::D, NPAD = S::NPAD, HALF = S::HALF, KCP = S::KCP, KB = S::KB;
  extern __shared__ unsigned char smem_raw[];
  // the 1024-aligned base as an offset from the shared array, so that the
  // compiler keeps shared-memory (not generic) loads and stores
  unsigned char* sm = smem_raw + ((1024u - (tc::smem_u32(smem_raw) & 1023u)) & 1023u);
  __shared__ __align__(8) uint64_t mma_bar[2];
  __shared__ __align__(8) uint64_t tma_bar[4];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;

  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const bool control = tid >= S::CTHREADS;
  const MixItem it = items[blockIdx.x];
  const int row0 = it.pair * RPC;                 // first computed row of this CTA
  const int nrows = min(RPC, S::ROWS_C - row0);  // valid rows of this CTA
  const int nch = (it.s_end - it.s_begin + KCP - 1) / KCP;
  const double qmax = *qmax_p;

  if (tid == 0) {
    tc::mbar_init(&mma_bar[0], 1);
    tc::mbar_init(&mma_bar[1], 1);
    for (int i = 0; i < S::TSTAGES; ++i) tc::mbar_init(&tma_bar[i], 1);
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
  auto fetch = [&](int c) {  // chunk c's table block into table stage c % TSTAGES
    const int t = c % S::TSTAGES;
    tc::mbar_arrive_expect_tx(&tma_bar[t], S::T_BYTES);
    tc::bulk_load(sm + t * S::T_STRIDE, it.tab + size_t(c) * S::T_BYTES, S::T_BYTES, &tma_bar[t]);
  };
  int last_fetch = -1;   // the last chunk requested (control lane 0)
  int last_commit = -1;  // the last chunk whose MMAs were committed (control lane 0)

  if (control) {
    // ------------------------------------------------------------ control warp
    const bool lead = (tid & 31) == 0;
    if (lead)
      for (int c = 0; c < min(S::TSTAGES, nch); ++c) {
        fetch(c);
        last_fetch = c;
      }
    for (int c = 0; c < nch; ++c) {
      const int s2 = c & 1, t = c % S::TSTAGES;
      tc::bar_sync(BAR_AREADY0 + s2, S::THREADS);  // A of chunk c is in TMEM (and its tables landed)
      if (lead && !s_abort) {
        tc::tc_fence_after();
        const uint32_t abase = tmem + uint32_t(S::A_COL0 + s2 * KB);
        // descriptor of the stage's B; the others differ by constant address offsets
        const uint64_t bdesc = tc::smem_desc(tc::smem_u32(sm + t * S::T_STRIDE), S::B_KGROUP, 128);
        const uint32_t acc0 = c > 0 ? 1u : 0u;
#pragma unroll
        for (int ks = 0; ks < S::KSTEPS; ++ks) {
          // slice products (a slice sa, b slices sb) of order sa + sb <= 3 into
          // accumulators sa + sb: one MMA per run of up to BGROUP b slices,
          // whose accumulators are adjacent in TMEM as the slices are in B
#pragma unroll
          for (int sa = 0; sa < 4; ++sa) {
#pragma unroll
            for (int sb = 0; sb < 4 - sa; sb += S::BGROUP) {
              const int nb = min(S::BGROUP, 4 - sa - sb);
              const uint32_t acc = (ks == 0 && sa == 0) ? acc0 : 1u;
              const uint64_t bd = bdesc + uint64_t((ks * 2 * S::B_KGROUP + sb * NPAD * 16) >> 4);
              tc::mma_i8_ts(tmem + uint32_t((sa + sb) * NPAD), abase + uint32_t(sa * (KB / 4) + ks * 8), bd,
                            tc::idesc_i8(RPC, nb * NPAD), acc);
            }
          }
        }
        tc::mma_commit(&mma_bar[s2]);
        last_commit = c;
        // the table stage of chunk c is free once these MMAs have read its B
        // (the consumers are past its factors: they signalled above)
        if (c + S::TSTAGES < nch) {
          wait_bar(&mma_bar[s2], uint32_t(c >> 1) & 1);
          if (!s_abort) {
            fetch(c + S::TSTAGES);
            last_fetch = c + S::TSTAGES;
          }
        }
      }
      __syncwarp();
    }
  } else {
    // ------------------------------------------------------------ consumers
    const int lr = tid & (RPC - 1);  // local row = TMEM lane
    const int kh = tid / RPC;        // this thread's 16-byte K group (8 particles) of each chunk
    const int rho = row0 + lr;
    const bool active = lr < nrows;
    const int r = rho < NK * D ? rho : rho + NK;  // the expansion row
    const int kz = active ? r / D : 0, ky = active ? r % D : 0;
    // this thread's four A columns of slice 0 of stage 0 (its warp's lane quarter)
    const uint32_t arow = tmem + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(S::A_COL0 + kh * 4);
    for (int c = 0; c < nch; ++c) {
      const int s2 = c & 1, t = c % S::TSTAGES;
      wait_bar(&tma_bar[t], uint32_t(c / S::TSTAGES) & 1);    // this chunk's tables have landed
      if (c >= 2) {
        wait_bar(&mma_bar[s2], uint32_t((c >> 1) - 1) & 1);  // A stage s2 is free
        tc::tc_fence_after();
      }
      uint32_t w[4][4] = {};
      if (active) {
        const unsigned char* tb = sm + t * S::T_STRIDE;
        const double2* ey = reinterpret_cast<const double2*>(tb + S::EY_OFF);
        const double2* ez = reinterpret_cast<const double2*>(tb + S::EZ_OFF);
#pragma unroll
        for (int p = 0; p < 4; ++p) {
          const int j0 = kh * 8 + 2 * p;
          // A = ez ey with ez carrying 2^24: each component in fixed point
          // from two FMAs
          const double2 z0 = ez[j0 * S::EZS + kz], y0 = ey[j0 * D + ky];
          const double2 z1 = ez[(j0 + 1) * S::EZS + kz], y1 = ey[(j0 + 1) * D + ky];
          uint32_t by[4];
          transpose4(fix24_dot(z0.x, y0.x, -z0.y, y0.y), fix24_dot(z0.x, y0.y, z0.y, y0.x),
                     fix24_dot(z1.x, y1.x, -z1.y, y1.y), fix24_dot(z1.x, y1.y, z1.y, y1.x), by);
#pragma unroll
          for (int sl = 0; sl < 4; ++sl) w[sl][p] = by[3 - sl];
        }
      }
      // every lane stores (rows past the tile's end store zeros, never read back)
#pragma unroll
      for (int sl = 0; sl < 4; ++sl)
        tc::tmem_st4(arow + uint32_t(s2 * KB + sl * (KB / 4)), w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
      tc::tmem_st_wait();
      tc::tc_fence_before();
      tc::bar_arrive(BAR_AREADY0 + s2, S::THREADS);
    }
    // ------------------------------------------------------------ epilogue
    if (nch > 0) {
      const int cl = nch - 1;
      wait_bar(&mma_bar[cl & 1], uint32_t(cl >> 1) & 1);
    }
    tc::tc_fence_after();
    tc::bar_sync(BAR_CONS, S::CTHREADS);  // every consumer is past its last read of the pipeline buffers
    const int q = warp & 3;            // TMEM lane quarter (warps 4k .. 4k + 3 read lanes 0 .. 127)
    double2* stage = reinterpret_cast<double2*>(sm) + size_t(lr) * D;
    const double scale = qmax / (SL_SCALE * SL_SCALE);
    if (nch > 0 && !s_abort) {
#pragma unroll 1
      for (int cb = kh; cb < NPAD / 16; cb += S::CPR) {
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
      for (int n = kh; n < D; n += S::CPR) stage[n] = make_double2(0.0, 0.0);
    }
    tc::fence_async_smem();
    tc::bar_sync(BAR_CONS, S::CTHREADS);
    // computed rows below NK D are the expansion rows themselves; those above
    // lie NK rows further on (the kz = 0, ky >= 0 rows)
    const int n_lo = max(0, min(nrows, NK * D - row0));
    if (tid == 0) {
      if (n_lo > 0) tc::bulk_store(it.out + size_t(row0) * D, sm, uint32_t(n_lo) * D * 16u);
      if (nrows > n_lo)
        tc::bulk_store(it.out + size_t(row0 + n_lo + NK) * D, sm + size_t(n_lo) * D * 16, uint32_t(nrows - n_lo) * D * 16u);
      tc::bulk_commit();
    }
    // the kz = 0, ky < 0 rows: out[NK][ky][kx] = conj(out[NK][2 NK - ky][2 NK - kx])
    // from the staged rows ky = 2 NK - ky > NK of this CTA
    {
      const double2* st0 = reinterpret_cast<const double2*>(sm);
      const int m_lo = max(row0, NK * D + 1), m_hi = row0 + nrows;  // computed rows with ky > NK
      for (int idx = tid; idx < (m_hi - m_lo) * D; idx += S::CTHREADS) {
        const int src = m_lo + idx / D, kx = idx % D;
        const int ky = NK + (src - NK * D);          // > NK
        const double2 v = st0[size_t(src - row0) * D + (2 * NK - kx)];
        it.out[size_t(NK * D + 2 * NK - ky) * D + kx] = make_double2(v.x, -v.y);
      }
    }
    if (tid == 0) tc::bulk_wait_all();
  }
  // copies and MMAs this CTA started have ended (bounded waits; they only
  // matter when a pipeline wait gave up) before its TMEM is released
  if (control && (tid & 31) == 0) {
    if (last_fetch >= 0) tc::mbar_wait(&tma_bar[last_fetch % S::TSTAGES], uint32_t(last_fetch / S::TSTAGES) & 1);
    if (last_commit >= 0) tc::mbar_wait(&mma_bar[last_commit & 1], uint32_t(last_commit >> 1) & 1);
  }
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
void launch_mixed(const CUtensorMap& tmap, const MixItem* d_items, int nitems, const int2* d_chunks, int nchunks,
                  const double* d_qmax, int* d_err, cudaStream_t st) {
  using S = MixShape<NK>;
  if (nitems == 0) return;
  if (nchunks > 0) {
    raise_smem_limit(reinterpret_cast<const void*>(k_pw_tables<NK>), S::TK_SMEM);
    // persistent: as many CTAs as are resident at once, each walking a
    // strided share of the chunks
    int dev = 0, sms = 0, per_sm = 0;
    PDMK_CUDA(cudaGetDevice(&dev));
    PDMK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PDMK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_pw_tables<NK>, S::TTHREADS, S::TK_SMEM));
    const int grid = std::max(1, std::min(nchunks, std::max(1, per_sm) * sms));
    k_pw_tables<NK><<<unsigned(grid), S::TTHREADS, S::TK_SMEM, st>>>(tmap, d_items, d_chunks, nchunks, d_qmax,
                                                                       d_err);
    PDMK_LAUNCH_CHECK();
  }
  raise_smem_limit(reinterpret_cast<const void*>(k_pw_mixed<NK>), S::SMEM);
  k_pw_mixed<NK><<<unsigned(nitems), S::THREADS, S::SMEM, st>>>(d_items, d_qmax, d_err);
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

int mixed_table_bytes(int nk) {
  switch (nk) {
    case 4: return MixShape<4>::T_BYTES;
    case 6: return MixShape<6>::T_BYTES;
    case 8: return MixShape<8>::T_BYTES;
    case 12: return MixShape<12>::T_BYTES;
    case 13: return MixShape<13>::T_BYTES;
    case 17: return MixShape<17>::T_BYTES;
    case 19: return MixShape<19>::T_BYTES;
    case 26: return MixShape<26>::T_BYTES;
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

void dispatch_mixed(int nk, const CUtensorMap& tmap, const MixItem* d_items, int nitems, const int2* d_chunks,
                    int nchunks, const double* d_qmax, int* d_err, cudaStream_t st) {
#define PDMK_MIX_CASE(n) \
  case n: launch_mixed<n>(tmap, d_items, nitems, d_chunks, nchunks, d_qmax, d_err, st); break;
  switch (nk) {
    PDMK_MIX_CASE(4)
    PDMK_MIX_CASE(6)
    PDMK_MIX_CASE(8)
    PDMK_MIX_CASE(12)
    PDMK_MIX_CASE(13)
    PDMK_MIX_CASE(17)
    PDMK_MIX_CASE(19)
    PDMK_MIX_CASE(26)
    default: throw std::invalid_argument("mixed precision: unsupported mode count");
  }
#undef PDMK_MIX_CASE
}

}  // namespace pdmk
