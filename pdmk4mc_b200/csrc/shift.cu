// Single-particle energy shift, accept-and-update, and the device-side
// Metropolis loop (FP64).
//
// Reference counterparts: eval_shift_energy and its window / difference /
// residual parts (src/energy_shift.cpp:18-302), locate_particle
// (src/tree.cpp:204-236), form_outgoing_pw_single (src/planewave.cpp:157-181)
// and update_shift (src/tree.cpp:447-597).
//
// One trial move runs as: k_shift (grid-wide partial sums; the last block
// finishes dE and the Metropolis test, lists the expansion vectors an
// accepted move changes and writes the Proposal record), then k_update (one
// read-modify-write per touched vector, target and origin contributions
// merged; block 0 also commits the particle membership). Both kernels read
// the Proposal record, so the sequence is stream-ordered and can be captured
// in a CUDA graph. Per-move latency is what bounds Monte Carlo throughput,
// so the kernels avoid dependent global loads: box coordinates along both
// paths come from the particle's grid key, the 27 minimum-image candidates
// and the two paths are resolved by the lanes of one warp in parallel.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "tree.hpp"

namespace pdmk {
namespace {

constexpr int SH_T = 256;
constexpr int MAXLV = MAX_LEVELS;

__device__ inline bool bm_get(const uint32_t* bm, uint64_t cell) { return (bm[cell >> 5] >> (cell & 31)) & 1u; }

__device__ inline int bm_rank(const DevTree& T, int level, uint64_t cell) {
  uint32_t w = T.bm_d[level][cell >> 5];
  return T.wprefix_d[level][cell >> 5] + __popc(w & ((1u << (cell & 31)) - 1u));
}

__device__ inline double center_of(double L, int l, int X) {
  double scale = ldexp(1.0, -l);
  return L * (double(X) * scale + 0.5 * scale);
}

__device__ inline int periodic_shift_d(double xi, double xj, double L, double bi, double bj) {
  if (xi < bi && xj > (L - bj)) return 1;
  if (xi > (L - bi) && xj < bj) return -1;
  return 0;
}


// Phase tables exp(-i m dk_l x) per axis for one point on its path. Layout:
// root axes (3 x dw), then levels 2, 3, ... (3 x dd each). The accessors
// compute addresses, so no pointer array is indexed at run time.
struct Tables {
  struct Axes {
    double2* b;
    int stride;
    __device__ double2* operator[](int ax) const { return b + ax * stride; }
  };
  struct Levels {
    double2* b;
    int dw, dd;
    __device__ Axes operator[](int l) const { return Axes{b + 3 * dw + (l - 2) * 3 * dd, dd}; }
  };
  Axes root;
  Levels lev;
};

__device__ inline void alloc_tables(double2* sm, const DevTree& T, Tables& tb) {
  tb.root = Tables::Axes{sm, 2 * T.n_window + 1};
  tb.lev = Tables::Levels{sm, 2 * T.n_window + 1, 2 * T.n_diff + 1};
}

struct Header {
  int i_orig, slot;
  double q;
  double xo[3], xt[3];
  double dr;
  int depth_o, depth_t;
  int path_o[MAXLV], path_t[MAXLV];
  int Xo[MAXLV][3], Xt[MAXLV][3];  // integer box coordinates along each path
};

// Tables of one point on its path for levels 2..lmax, one entry per thread
// (threads t0, t0 + nthr, ...): e^{-i m dk_l (x - c_l)} with the box-centred
// phase and the exact decentring root of unity, times q on the z axis. Every
// entry is its own sincos, so the table costs one sincos latency instead of
// a chain of recurrence steps.
__device__ void build_tables(const DevTree& T, const double* x, double q, const int (*X)[3], int lmax,
                             const Tables& tb, int t0, int nthr) {
  const int nw = T.n_window, nd = T.n_diff;
  const int root_n = 2 * (2 * nw + 1) + (nw + 1);
  const int lev_n = 2 * (2 * nd + 1) + (nd + 1);
  const int nlev = lmax >= 2 ? lmax - 1 : 0;
  const int total = root_n + nlev * lev_n;
  for (int e = t0; e < total; e += nthr) {
    int slot, rem;
    if (e < root_n) {
      slot = 0;
      rem = e;
    } else {
      slot = 1 + (e - root_n) / lev_n;
      rem = (e - root_n) % lev_n;
    }
    const int n = slot == 0 ? nw : nd;
    const int w = 2 * n + 1;
    const int axis = rem < w ? 0 : (rem < 2 * w ? 1 : 2);
    const int t = rem - axis * w;
    const int m = t - n;
    double xr, dk;
    int dec;
    double2* dst;
    if (slot == 0) {
      xr = x[axis] - 0.5 * T.L;
      dk = T.delta_k[0];
      dec = 3;
      dst = tb.root[axis];
    } else {
      const int l = slot + 1, Xa = X[l][axis];
      xr = x[axis] - center_of(T.L, l, Xa);
      dk = level_dk(T, l);
      dec = 2 * Xa + 1;
      dst = tb.lev[l][axis];
    }
    const double th = dk * xr;
    double sn, cs;
    sincos(-double(m) * th, &sn, &cs);
    const double sc = axis == 2 ? q : 1.0;
    dst[t] = cmul(make_double2(cs * sc, sn * sc), root6(-dec * m));
  }
}

template <class A>
__device__ inline double2 phase_at(const A& ax, int k, int d) {
  int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
  return cmul(ax[2][iz], cmul(ax[1][iy], ax[0][ix]));
}

// Resolve a proposal with the first warp: particle and positions (every lane
// loads the same words), my_mod wrap, the minimum-image old-new distance
// (one image per lane, src/energy_shift.cpp:30-41) and both leaf paths
// (lanes 0-15 the target, 16-31 the origin, one level per lane, from the
// refinement bitmaps: the reference's locate_particle, src/tree.cpp:204-236).
// Loads of data that other blocks of a persistent kernel write (CG = true)
// bypass L1, which is not coherent across SMs.
template <bool CG, class V>
__device__ inline V ldm(const V* p) {
  if constexpr (CG) return __ldcg(p);
  else return *p;
}

// A particle's slot, position and charge loaded ahead of its resolve (s < 0:
// nothing loaded).
struct Preload {
  int s;
  double x, y, z, q;
};

template <bool CG = false>
__device__ void resolve(const DevTree& T, int i, const double* disp, Header& h, const Preload* pre = nullptr) {
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    const bool have = pre && pre->s >= 0;
    const int s = have ? pre->s : ldm<CG>(T.orig_slot + i);
    double xo[3], q;
    if (have) {
      xo[0] = pre->x;
      xo[1] = pre->y;
      xo[2] = pre->z;
      q = pre->q;
    } else if (s < T.n_slots) {
      xo[0] = ldm<CG>(T.sx + s);
      xo[1] = ldm<CG>(T.sy + s);
      xo[2] = ldm<CG>(T.sz + s);
      q = ldm<CG>(T.sq + s);
    } else {
      const int p = s - T.n_slots;
      xo[0] = ldm<CG>(T.px + p);
      xo[1] = ldm<CG>(T.py + p);
      xo[2] = ldm<CG>(T.pz + p);
      q = ldm<CG>(T.pq + p);
    }
    const double L = T.L;
    const double d0 = disp[0], d1 = disp[1], d2 = disp[2];
    const double xt[3] = {wrap_mod(xo[0] + d0, L), wrap_mod(xo[1] + d1, L), wrap_mod(xo[2] + d2, L)};
    double dr = sqrt(d0 * d0 + d1 * d1 + d2 * d2);
    if (lane < 27) {
      const int mx = lane % 3 - 1, my = (lane / 3) % 3 - 1, mz = lane / 9 - 1;
      const double ax = xt[0] - (xo[0] + mx * L), ay = xt[1] - (xo[1] + my * L), az = xt[2] - (xo[2] + mz * L);
      dr = fmin(dr, sqrt(ax * ax + ay * ay + az * az));
    }
    for (int o = 16; o > 0; o >>= 1) dr = fmin(dr, __shfl_xor_sync(0xffffffffu, dr, o));
    const int half = lane >> 4, l = lane & 15;
    const double* p = half == 0 ? xt : xo;
    const uint32_t g[3] = {grid_coord(p[0], L), grid_coord(p[1], L), grid_coord(p[2], L)};
    const uint64_t key = morton3(g[0], g[1], g[2]);
    bool is_leaf = false;
    int node = -1;
    if (l < T.max_depth) {
      const uint64_t cell = l == 0 ? 0 : key >> (3 * (KEY_BITS - l));
      const bool exists = l <= 1 || bm_get(T.bm_d[l - 1], cell >> 3);
      if (exists) {
        node = l == 0 ? 0
                      : (l == 1 ? 1 + int(cell) : T.level_start_d[l] + 8 * bm_rank(T, l - 1, cell >> 3) + int(cell & 7));
        is_leaf = !(l <= T.maxref && bm_get(T.bm_d[l], cell));
      }
    }
    const unsigned leaves = (__ballot_sync(0xffffffffu, is_leaf) >> (16 * half)) & 0xffffu;
    const int leaf_level = __ffs(leaves) - 1;
    if (l <= leaf_level) {
      int* path = half == 0 ? h.path_t : h.path_o;
      int(*X)[3] = half == 0 ? h.Xt : h.Xo;
      path[l] = node;
      for (int a = 0; a < 3; ++a) X[l][a] = int(g[a] >> (KEY_BITS - l));
    }
    if (lane == 0) {
      h.i_orig = i;
      h.slot = s;
      h.q = q;
      for (int a = 0; a < 3; ++a) {
        h.xo[a] = xo[a];
        h.xt[a] = xt[a];
      }
      h.dr = dr;
      h.depth_t = leaf_level + 1;
    }
    if (lane == 16) h.depth_o = leaf_level + 1;
  }
  __syncthreads();
}

// q * sum_{j in N(leaf)} q_j res(|x - x_j|; bs_leaf), masked r^2 in (eps, b^2)
// (eval_shift_energy_res_vec + direct_eval, src/energy_shift.cpp:233-302).
// Source metadata is fetched in parallel, then all threads share the pairs.
template <int NP>
__device__ double residual_sum(const DevTree& T, const ResidualPoly<NP>& poly, int leaf, int l, const int* Xl,
                               const double* x) {
  const double b = level_box(T, l);
  const double b2 = b * b;
  const double eps = 2.220446049250313e-16;
  __shared__ int m_beg[36], m_cnt[36], m_pre[37], m_lvl[36];
  __shared__ unsigned long long m_pfx[36];
  __shared__ double m_off[36][3];
  if (threadIdx.x < 36) {
    const int src = threadIdx.x;
    int j = -1;
    if (src == 0) j = leaf;
    else if (src <= 27) j = (src - 1 == 13) ? -1 : T.col27[size_t(leaf) * 27 + (src - 1)];
    else j = T.coarse8[size_t(leaf) * 8 + (src - 28)];
    int beg = 0, cnt = 0, lj = 0;
    unsigned long long pj = 0;
    double off[3] = {0, 0, 0};
    if (j >= 0) {
      lj = T.node_level[j];
      pj = T.node_prefix[j];
      const int ch = T.node_child0[j];
      beg = T.node_begin[j];
      const int end = ch < 0 ? beg + T.leaf_count[j] : T.node_end[j];
      cnt = end - beg;
      const double bj = level_box(T, lj);
      const int Xj[3] = {int(compact3(pj)), int(compact3(pj >> 1)), int(compact3(pj >> 2))};
      for (int d = 0; d < 3; ++d)
        off[d] = -periodic_shift_d(center_of(T.L, l, Xl[d]), center_of(T.L, lj, Xj[d]), T.L, b, bj) * T.L;
    }
    m_beg[src] = beg;
    m_cnt[src] = j >= 0 ? cnt : -1;
    m_lvl[src] = lj;
    m_pfx[src] = pj;
    for (int d = 0; d < 3; ++d) m_off[src][d] = off[d];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int src = 0; src < 36; ++src) {
      m_pre[src] = s;
      s += max(m_cnt[src], 0);
    }
    m_pre[36] = s;
  }
  __syncthreads();
  const int total = m_pre[36];
  double acc = 0;
  int src = 0;
  for (int e = threadIdx.x; e < total; e += blockDim.x) {
    while (e >= m_pre[src + 1]) ++src;
    const int s = m_beg[src] + (e - m_pre[src]);
    const double dx = x[0] - (T.sx[s] + m_off[src][0]), dy = x[1] - (T.sy[s] + m_off[src][1]),
                 dz = x[2] - (T.sz[s] + m_off[src][2]);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > eps && r2 < b2) acc += T.sq[s] * poly(sqrt(r2), b);
  }
  // arrivals parked in the overflow pool that belong to a source's subtree
  const int pn = *T.pool_n;
  for (int e = threadIdx.x; e < 36 * pn; e += blockDim.x) {
    const int sj = e / pn, p = e % pn;
    if (m_cnt[sj] < 0 || T.p_orig[p] < 0) continue;
    const int pl = T.p_leaf[p];
    const int ll = T.node_level[pl], lj = m_lvl[sj];
    if (ll < lj || (T.node_prefix[pl] >> (3 * (ll - lj))) != m_pfx[sj]) continue;
    const double dx = x[0] - (T.px[p] + m_off[sj][0]), dy = x[1] - (T.py[p] + m_off[sj][1]),
                 dz = x[2] - (T.pz[p] + m_off[sj][2]);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 > eps && r2 < b2) acc += T.pq[p] * poly(sqrt(r2), b);
  }
  return acc;
}

// sums of four values over the block, valid in thread 0
__device__ inline void block_sum4(double* v, double (*sm)[32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int c = 0; c < 4; ++c)
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  __syncthreads();
  if (lane == 0)
    for (int c = 0; c < 4; ++c) sm[c][warp] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int c = 0; c < 4; ++c) {
      double s = 0;
      for (int w = 0; w < nw; ++w) s += sm[c][w];
      v[c] = s;
    }
  __syncthreads();
}

// as block_sum4, the sums in thread 0 only and no barrier after them (the
// caller's next barrier orders its use)
__device__ inline void block_sum4_t0(double* v, double (*sm)[32]) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int c = 0; c < 4; ++c)
    for (int o = 16; o > 0; o >>= 1) v[c] += __shfl_down_sync(0xffffffffu, v[c], o);
  __syncthreads();
  if (lane == 0)
    for (int c = 0; c < 4; ++c) sm[c][warp] = v[c];
  __syncthreads();
  if (threadIdx.x == 0)
    for (int c = 0; c < 4; ++c) {
      double s = 0;
      for (int w = 0; w < nw; ++w) s += sm[c][w];
      v[c] = s;
    }
}

// slot s of a path level: 0 own outgoing, 1 own incoming, 2.. the colleague
// in direction dir (dir != 13, dx fastest)
__device__ inline int slot_of_dir(int dir) { return 2 + (dir < 13 ? dir : dir - 1); }
__device__ inline int dir_of_slot(int s) { return (s - 2) + ((s - 2) >= 13 ? 1 : 0); }

// Receivers of an accepted move (update_shift, src/tree.cpp:484-579): per
// path level own out, own inc and non-leaf colleagues' inc. A vector that
// both paths touch becomes one receiver carrying both contributions, so the
// update needs a single launch without write races. Receivers are matched by
// box coordinates (known from the header), the records go to T.recv and the
// count is returned to every thread. Block-cooperative.
__device__ int build_receivers(const DevTree& T, const Header& h, Receiver* out) {
  constexpr int PER = 28 * MAXLV;
  __shared__ int ckey[2 * PER];  // receiving node (-1 none)
  __shared__ signed char cfl[2 * PER][3];
  __shared__ short cmatch[2 * PER];
  __shared__ int wsum[32];
  const int levels = max(T.pw_hi - 1, 0);
  const int per = 28 * levels;
  const int ncand = 2 * per;
  const int ut = min(h.depth_t - 1, T.pw_hi), uo = min(h.depth_o - 1, T.pw_hi);
  for (int c = threadIdx.x; c < ncand; c += blockDim.x) {
    const int p = c / per, r = c % per;
    const int l = 2 + r / 28, s = r % 28;
    int recv = -1;
    signed char f[3] = {0, 0, 0};
    if (l <= (p == 0 ? ut : uo)) {
      const int node = p == 0 ? h.path_t[l] : h.path_o[l];
      recv = node;
      if (s >= 2) {
        const int dir = dir_of_slot(s);
        recv = T.col27[size_t(node) * 27 + dir];
        if (recv >= 0 && T.node_child0[recv] < 0) recv = -1;
        if (recv >= 0) {
          // source-centric image flag: periodic_shift(c_source, c_receiver)
          const int* X = p == 0 ? h.Xt[l] : h.Xo[l];
          const int dv[3] = {dir % 3 - 1, (dir / 3) % 3 - 1, dir / 9 - 1};
          for (int q = 0; q < 3; ++q) {
            const int v = X[q] + dv[q];
            f[q] = v < 0 ? 1 : (v >= (1 << l) ? -1 : 0);
          }
        }
      }
    }
    ckey[c] = recv;
    cfl[c][0] = f[0];
    cfl[c][1] = f[1];
    cfl[c][2] = f[2];
    cmatch[c] = -1;
  }
  __syncthreads();
  // an origin receiver equals a target receiver when it is the same vector;
  // its slot among the target's follows from the box coordinates
  for (int c = per + threadIdx.x; c < ncand; c += blockDim.x) {
    const int recv = ckey[c];
    if (recv < 0) continue;
    const int r = c - per, l = 2 + r / 28, s = r % 28;
    if (l > ut) continue;
    const int e = 1 << l;
    int ts;
    if (s == 0) {
      ts = h.path_t[l] == recv ? 0 : -1;
    } else {
      // receiver coordinates relative to the target's box at this level
      const int dir_o = s == 1 ? 13 : dir_of_slot(s);
      const int dvo[3] = {dir_o % 3 - 1, (dir_o / 3) % 3 - 1, dir_o / 9 - 1};
      int dir = 0, mul = 1;
      bool ok = true;
      for (int q = 0; q < 3; ++q) {
        int dq = ((h.Xo[l][q] + dvo[q] + e) & (e - 1)) - h.Xt[l][q];
        if (dq == e - 1) dq = -1;
        if (dq == 1 - e) dq = 1;
        ok = ok && dq >= -1 && dq <= 1;
        dir += (dq + 1) * mul;
        mul *= 3;
      }
      ts = !ok ? -1 : (dir == 13 ? 1 : slot_of_dir(dir));
    }
    if (ts >= 0) {
      const int t = (l - 2) * 28 + ts;
      if (ckey[t] == recv) {
        cmatch[c] = short(t);
        cmatch[t] = short(c);
      }
    }
  }
  __syncthreads();
  // compact: target receivers in slot order, then unmatched origin receivers
  const int per_thread = (ncand + blockDim.x - 1) / blockDim.x;
  const int c0 = threadIdx.x * per_thread;
  int cnt = 0;
  for (int c = c0; c < min(c0 + per_thread, ncand); ++c) cnt += ckey[c] >= 0 && (c < per || cmatch[c] < 0);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  int x = cnt;
  for (int o = 1; o < 32; o <<= 1) {
    int y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  if (threadIdx.x == 0) {
    int s = 0;
    for (int w = 0; w < int(blockDim.x >> 5); ++w) {
      int v = wsum[w];
      wsum[w] = s;
      s += v;
    }
    wsum[31] = s;
  }
  __syncthreads();
  int pos = wsum[warp] + x - cnt;
  const int base = T.pw_base;
  for (int c = c0; c < min(c0 + per_thread, ncand); ++c) {
    if (!(ckey[c] >= 0 && (c < per || cmatch[c] < 0))) continue;
    const int r = c % per;
    Receiver R;
    R.off = ckey[c] - base;
    R.is_out = (r % 28) == 0;
    R.level = static_cast<signed char>(2 + r / 28);
    const bool is_t = c < per;
    const int m = cmatch[c];
    R.has_t = is_t;
    R.has_o = !is_t || m >= 0;
    for (int q = 0; q < 3; ++q) {
      R.ft[q] = is_t ? cfl[c][q] : 0;
      R.fo[q] = is_t ? (m >= 0 ? cfl[m][q] : 0) : cfl[c][q];
    }
    R.pad[0] = R.pad[1] = 0;
    out[pos++] = R;
  }
  const int total = wsum[31];
  __syncthreads();
  return total;
}

struct ShiftArgs {
  const int* idx;
  const double* disp;
  const double* u;
  double beta;
  int move;
  int mode;  // 0: evaluate only, 1: Metropolis
  double* dE_out;
  int* acc_out;
  double c_window;  // dk_0^3 / (2 pi)^3
  double* partials;
  unsigned int* counter;
  Proposal* prop;
  double2* ptab;          // phase tables published for k_update
  long ptab_per;          // complex entries per path
  const MoveCursor* cur;  // non-null: proposals come from the cursor (captured graphs)
};

// Grid: blocks [0, G-2) do the plane-wave sums; block G-2 the target
// residual, block G-1 the origin residual. The last block to finish reduces.
template <int NP>
__global__ void __launch_bounds__(SH_T) k_shift(DevTree T, ShiftArgs a) {
  extern __shared__ double2 sm2[];
  __shared__ Header h;
  __shared__ double red[4][32];
  __shared__ double c_level[MAXLV + 2];  // dk_l^3 / (2 pi)^3 * dscale_l
  __shared__ bool is_last;
  const ResidualPoly<NP> poly(T);
  if (threadIdx.x >= 2 && threadIdx.x < MAXLV + 2) {
    const double dk = level_dk(T, threadIdx.x);
    c_level[threadIdx.x] = dk * dk * dk / (8.0 * 3.14159265358979323846 * 3.14159265358979323846 *
                                           3.14159265358979323846) * level_dscale(threadIdx.x);
  }
  if (a.cur) {
    const MoveCursor c = *a.cur;
    a.idx = c.idx;
    a.disp = c.disp;
    a.u = c.u;
    a.dE_out = c.dE;
    a.acc_out = c.acc;
    a.mode = c.mode;
    a.beta = c.beta;
    a.move += c.off;
  }
  const int move = a.move;
  resolve(T, a.idx[move], a.disp + 3 * move, h);
  const int G = gridDim.x;
  const int Gpw = G - 2;
  double acc[4] = {0, 0, 0, 0};  // window, difference, residual target, residual origin
  if (blockIdx.x < Gpw) {
    // dE needs the non-leaf path levels 2 .. depth-2; an accept-and-update
    // needs 2 .. min(depth-1, pw_hi): build the superset
    const int lo_max = h.depth_o - 2, lt_max = h.depth_t - 2;
    const int uo = min(h.depth_o - 1, T.pw_hi), ut = min(h.depth_t - 1, T.pw_hi);
    const int per = 3 * (2 * T.n_window + 1) + max(max(uo, ut) - 1, 0) * 3 * (2 * T.n_diff + 1);
    Tables to, oo;
    alloc_tables(sm2, T, oo);
    alloc_tables(sm2 + per, T, to);
    build_tables(T, h.xo, h.q, h.Xo, uo, oo, threadIdx.x, blockDim.x);
    build_tables(T, h.xt, h.q, h.Xt, ut, to, threadIdx.x, blockDim.x);
    __syncthreads();
    if (blockIdx.x == 0) {
      // publish the tables for k_update
      for (int p = 0; p < 2; ++p) {
        Tables g;
        alloc_tables(a.ptab + size_t(p) * a.ptab_per, T, g);
        const Tables& s = p == 0 ? oo : to;
        const int up = p == 0 ? uo : ut;
        for (int ax = 0; ax < 3; ++ax)
          for (int e = threadIdx.x; e < T.dw; e += blockDim.x) g.root[ax][e] = s.root[ax][e];
        for (int l = 2; l <= up; ++l)
          for (int ax = 0; ax < 3; ++ax)
            for (int e = threadIdx.x; e < T.dd; e += blockDim.x) g.lev[l][ax][e] = s.lev[l][ax][e];
      }
    }
    const int stride = Gpw * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    // window (src/energy_shift.cpp:72-90)
    for (int k = t0; k < T.Hw; k += stride) {
      double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
      double2 g = T.out_root[k];
      double ar = t.x - o.x, ai = t.y - o.y, br = g.x - o.x, bi = g.y - o.y;
      acc[0] += (ar * br + ai * bi) * T.W[k];
    }
    // difference (src/energy_shift.cpp:92-140), all path levels per mode
    const int base = T.pw_base;
    const int d = T.dd;
    for (int k = t0; k < T.H; k += stride) {
      const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
      double s = 0;
      for (int l = 2; l <= lo_max; ++l) {
        double2 o = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
        double2 c = T.inc[size_t(h.path_o[l] - base) * T.H + k];
        s -= (o.x * c.x - o.y * c.y - (o.x * o.x + o.y * o.y)) * c_level[l];
      }
      for (int l = 2; l <= lt_max; ++l) {
        double2 t = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
        double2 c = T.inc[size_t(h.path_t[l] - base) * T.H + k];
        s += (t.x * c.x - t.y * c.y) * c_level[l];
      }
      acc[1] += s * T.D2[k];
    }
  } else if (blockIdx.x == Gpw) {
    const int lt = h.depth_t - 1;
    acc[2] = residual_sum(T, poly, h.path_t[lt], lt, h.Xt[lt], h.xt) * h.q;
  } else {
    const int lo = h.depth_o - 1;
    acc[3] = residual_sum(T, poly, h.path_o[lo], lo, h.Xo[lo], h.xo) * h.q;
  }
  block_sum4(acc, red);
  if (threadIdx.x == 0) {
    double* pp = a.partials + 4 * size_t(blockIdx.x);
    for (int c = 0; c < 4; ++c) pp[c] = acc[c];
    __threadfence();
    unsigned prev = atomicAdd(a.counter, 1u);
    is_last = (prev == unsigned(G - 1));
  }
  __syncthreads();
  if (!is_last) return;
  __threadfence();
  // fixed-order reduction of the block partials (deterministic)
  double tot[4] = {0, 0, 0, 0};
  for (int b = threadIdx.x; b < G; b += blockDim.x)
    for (int c = 0; c < 4; ++c) tot[c] += __ldcg(a.partials + 4 * size_t(b) + c);
  block_sum4(tot, red);
  const int nrecv = build_receivers(T, h, T.recv);
  if (threadIdx.x == 0) {
    const double dEw = tot[0] * a.c_window;  // 2 * sum * dk0^3 / (2 (2 pi)^3)
    const double d = tot[1], rt = tot[2], ro = tot[3];
    double self = 0;
    if (h.dr != 0) self = poly(h.dr, level_box(T, 2)) * h.q * h.q;
    const double dE = dEw + d + rt - ro - self;
    Proposal* P = a.prop;
    P->i_orig = h.i_orig;
    P->slot = h.slot;
    P->q = h.q;
    for (int c = 0; c < 3; ++c) {
      P->xo[c] = h.xo[c];
      P->xt[c] = h.xt[c];
    }
    P->depth_o = h.depth_o;
    P->depth_t = h.depth_t;
    for (int l = 0; l < MAXLV; ++l) {
      P->path_o[l] = l < h.depth_o ? h.path_o[l] : -1;
      P->path_t[l] = l < h.depth_t ? h.path_t[l] : -1;
    }
    P->dE = dE;
    P->parts[0] = dEw;
    P->parts[1] = d;
    P->parts[2] = rt;
    P->parts[3] = ro;
    P->parts[4] = self;
    int accd = 0;
    if (a.mode == 1) {
      const double u = a.u[move];
      accd = u < exp(-a.beta * dE) ? 1 : 0;
      if (a.acc_out) a.acc_out[move] = accd;
    }
    if (a.dE_out) a.dE_out[move] = dE;
    P->accepted = accd;
    P->valid = 1;
    P->n_recv = nrecv;
    *a.counter = 0u;
  }
}

// ---------------------------------------------------------------------------
// update_shift (src/tree.cpp:447-597) in one launch. Each thread owns one
// mode k (grid x) and walks a range of receivers (grid y): out += t - o, or
// inc += conj(t s_t) - conj(o s_o) with the periodic image phases s; the
// y == 0 blocks also update the root expansion (out += t; out -= o) and
// block (0, 0) commits the particle membership.
constexpr int UPD_T = 128;
constexpr int UPD_UNROLL = 8;

__device__ void commit_move(const DevTree& T, const Proposal& P);

__global__ void __launch_bounds__(UPD_T) k_update(DevTree T, const double2* __restrict__ ptab, long ptab_per) {
  __shared__ Receiver rs[MAX_RECV];
  __shared__ int s_acc, s_nr;
  if (threadIdx.x == 0) {
    s_acc = T.prop->accepted;
    s_nr = T.prop->n_recv;
  }
  __syncthreads();
  if (!s_acc) return;
  const int nr = s_nr;
  const int r0 = int((long(blockIdx.y) * nr) / gridDim.y), r1 = int((long(blockIdx.y + 1) * nr) / gridDim.y);
  for (int r = r0 + threadIdx.x; r < r1; r += blockDim.x) rs[r - r0] = T.recv[r];
  if (blockIdx.x == 0 && blockIdx.y == 0 && threadIdx.x == 0) {
    atomicAdd(&T.work[0], 1ull);
    atomicAdd(&T.work[1], 32ull * ((unsigned long long)T.Hw + (unsigned long long)nr * T.H));
    commit_move(T, *T.prop);
  }
  __syncthreads();
  Tables tt, to;
  alloc_tables(const_cast<double2*>(ptab) + ptab_per, T, tt);
  alloc_tables(const_cast<double2*>(ptab), T, to);
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (blockIdx.y == 0 && k < T.Hw) {
    double2 t = phase_at(tt.root, k, T.dw), o = phase_at(to.root, k, T.dw);
    double2 g = T.out_root[k];
    g = cadd(g, t);
    g = csub(g, o);
    T.out_root[k] = g;
  }
  if (k >= T.H) return;
  const int n = T.n_diff, d = T.dd;
  const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
  const int a0 = ((ix - n) % 3 + 3) % 3, a1 = ((iy - n) % 3 + 3) % 3, a2 = ((iz - n) % 3 + 3) % 3;
  int r = 0;
  const int nloc = r1 - r0;
  while (r < nloc) {
    // a run of receivers on one level shares the two single-particle phases
    const int l = rs[r].level;
    int re = r + 1;
    while (re < nloc && rs[re].level == l) ++re;
    const double2 pt0 = cmul(tt.lev[l][2][iz], cmul(tt.lev[l][1][iy], tt.lev[l][0][ix]));
    const double2 po0 = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
    const double2 pt1 = cmul(pt0, root6(-2)), pt2 = cmul(pt0, root6(-4));
    const double2 po1 = cmul(po0, root6(-2)), po2 = cmul(po0, root6(-4));
    const int two_l = (l & 1) ? 2 : 1;
    for (; r < re; r += UPD_UNROLL) {
      double2 v[UPD_UNROLL];
      size_t off[UPD_UNROLL];
#pragma unroll
      for (int u = 0; u < UPD_UNROLL; ++u) {
        if (r + u < re) {
          const Receiver& R = rs[r + u];
          off[u] = size_t(R.off) * T.H + k;
          v[u] = R.is_out ? T.out[off[u]] : T.inc[off[u]];
        }
      }
#pragma unroll
      for (int u = 0; u < UPD_UNROLL; ++u) {
        if (r + u < re) {
          const Receiver& R = rs[r + u];
          // image phase: a cube root of unity, w^-e with e in [-12, 12] mod 3
          const int et = ((a0 * R.ft[0] + a1 * R.ft[1] + a2 * R.ft[2]) * two_l + 12) % 3;
          const int eo = ((a0 * R.fo[0] + a1 * R.fo[1] + a2 * R.fo[2]) * two_l + 12) % 3;
          double2 del = make_double2(0.0, 0.0);
          if (R.has_t) del = et == 0 ? pt0 : (et == 1 ? pt1 : pt2);
          if (R.has_o) del = csub(del, eo == 0 ? po0 : (eo == 1 ? po1 : po2));
          if (R.is_out) T.out[off[u]] = cadd(v[u], del);
          else T.inc[off[u]] = make_double2(v[u].x + del.x, v[u].y - del.y);
        }
      }
    }
    r = re;
  }
}

// particle membership and position (exact on every level); one thread. The
// independent loads are issued together and the per-level counts change by
// atomic adds that need no reply, so the thread waits on few round trips.
__device__ void commit_move(const DevTree& T, const Proposal& P) {
  if (!P.accepted) return;
  const int leafA = P.path_o[P.depth_o - 1];
  const int leafB = P.path_t[P.depth_t - 1];
  const int i = P.i_orig;
  const int s = P.slot;
  const double xt0 = P.xt[0], xt1 = P.xt[1], xt2 = P.xt[2], q = P.q;
  if (leafA == leafB) {
    if (s < T.n_slots) {
      T.sx[s] = xt0;
      T.sy[s] = xt1;
      T.sz[s] = xt2;
    } else {
      const int p = s - T.n_slots;
      T.px[p] = xt0;
      T.py[p] = xt1;
      T.pz[p] = xt2;
    }
    return;
  }
  const int cA = T.leaf_count[leafA], begA = T.node_begin[leafA];
  const int cB = T.leaf_count[leafB], begB = T.node_begin[leafB], endB = T.node_end[leafB];
  const int pn = *T.pool_n;
  // remove from the origin leaf (swap with its last particle) or the pool
  if (s < T.n_slots) {
    const int last = begA + cA - 1;
    const int ol = T.s_orig[last];
    const double lx = T.sx[last], ly = T.sy[last], lz = T.sz[last], lq = T.sq[last];
    const uint64_t pfx = T.node_prefix[leafA];
    const int lvl = T.node_level[leafA];
    if (s != last) {
      T.sx[s] = lx;
      T.sy[s] = ly;
      T.sz[s] = lz;
      T.sq[s] = lq;
      T.s_orig[s] = ol;
      T.orig_slot[ol] = s;
    }
    // a freed slot holds a zero charge at its leaf's centre
    T.sx[last] = center_of(T.L, lvl, int(compact3(pfx)));
    T.sy[last] = center_of(T.L, lvl, int(compact3(pfx >> 1)));
    T.sz[last] = center_of(T.L, lvl, int(compact3(pfx >> 2)));
    T.sq[last] = 0.0;
    T.s_orig[last] = -1;
    T.leaf_count[leafA] = cA - 1;
  } else {
    const int p = s - T.n_slots;
    T.p_orig[p] = -1;
    T.pq[p] = 0.0;
  }
  // insert into the target leaf, or park in the pool when it is full
  const int slot = begB + cB;
  if (slot < endB) {
    T.sx[slot] = xt0;
    T.sy[slot] = xt1;
    T.sz[slot] = xt2;
    T.sq[slot] = q;
    T.s_orig[slot] = i;
    T.orig_slot[i] = slot;
    T.leaf_count[leafB] = cB + 1;
  } else if (pn < T.pool_cap) {
    T.px[pn] = xt0;
    T.py[pn] = xt1;
    T.pz[pn] = xt2;
    T.pq[pn] = q;
    T.p_orig[pn] = i;
    T.p_leaf[pn] = leafB;
    T.orig_slot[i] = T.n_slots + pn;
    *T.pool_n = pn + 1;
  } else {
    *T.err = 1;  // pool exhausted: the host repacks and reports
  }
  for (int l = 0; l < P.depth_o; ++l) atomicAdd(T.node_count + P.path_o[l], -1);
  for (int l = 0; l < P.depth_t; ++l) atomicAdd(T.node_count + P.path_t[l], 1);
}


// ---------------------------------------------------------------------------
// Persistent Metropolis kernel: one cooperative launch runs a whole sequence
// of trial moves on every SM. Per move, every block resolves the proposal and
// builds both paths' phase tables itself (no broadcast needed), adds its share
// of the window, difference and near-field sums, and publishes 4 partials;
// after a grid barrier every block reduces all partials in the same fixed
// order, so all blocks reach the same dE and the same Metropolis decision. An
// accepted move is then applied by all blocks (receivers listed per block,
// one read-modify-write per mode and vector), block 0 commits the particle,
// and a second barrier orders the update before the next move. Barrier waits
// are bounded; a wait that gives up sets an error bit and every block returns.
constexpr int MC_T = 512;

struct McArgs {
  const int* idx;
  const double* disp;
  const double* u;
  double beta;
  int n_moves;
  double* dE_out;
  int* acc_out;
  double c_window;          // dk_0^3 / (2 pi)^3
  double* partials;         // [2][G][4], double-buffered by move parity
  unsigned int* arrivals;   // barrier arrivals, zero at launch
  long long spin_limit;     // polls before a barrier wait gives up
};

__device__ inline unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Grid barrier over a monotonically increasing arrival counter, as an
// arrival and a wait that may be apart; nbar counts the barriers this block
// has arrived at (kept by thread 0).
__device__ void mc_arrive(const McArgs& a, unsigned& nbar) {
  __syncthreads();
  if (threadIdx.x == 0) {
    ++nbar;
    // the release orders this block's writes (made visible to this thread by
    // the __syncthreads above) before the arrival; no reply is awaited
    asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(a.arrivals) : "memory");
  }
}

// Waits until every block has arrived at this block's last barrier. False
// when the wait gave up or another block reported a failure.
__device__ bool mc_wait(const DevTree& T, const McArgs& a, unsigned nbar) {
  __shared__ int s_ok;
  if (threadIdx.x == 0) {
    const unsigned target = nbar * gridDim.x;
    int ok = 1;
    for (long long it = 0;; ++it) {
      if (ld_acquire(a.arrivals) >= target) break;
      if (ldm<true>(T.err) & 2) {
        ok = 0;
        break;
      }
      if (it >= a.spin_limit) {
        atomicOr(T.err, 2);
        ok = 0;
        break;
      }
      __nanosleep(32);
    }
    // the acquire load above orders this thread after the other blocks'
    // releases; the barrier below passes that order on to the whole block
    s_ok = ok;
  }
  __syncthreads();
  return s_ok != 0;
}

__device__ bool mc_barrier(const DevTree& T, const McArgs& a, unsigned& nbar) {
  mc_arrive(a, nbar);
  return mc_wait(T, a, nbar);
}

// Source lists of one path's leaf for the near field: the leaf, its 26
// colleagues and 8 coarse neighbours, with their periodic offsets.
struct ResMeta {
  int beg[36], cnt[36], pre[37], lvl[36];
  unsigned long long pfx[36];
  double off[36][3];
};

__device__ void res_meta(const DevTree& T, int leaf, int l, const int* Xl, int src, ResMeta& M) {
  const double b = level_box(T, l);
  int j = -1;
  if (src == 0) j = leaf;
  else if (src <= 27) j = (src - 1 == 13) ? -1 : T.col27[size_t(leaf) * 27 + (src - 1)];
  else j = T.coarse8[size_t(leaf) * 8 + (src - 28)];
  int beg = 0, cnt = 0, lj = 0;
  unsigned long long pj = 0;
  double off[3] = {0, 0, 0};
  if (j >= 0) {
    lj = T.node_level[j];
    pj = T.node_prefix[j];
    const int ch = T.node_child0[j];
    beg = T.node_begin[j];
    const int end = ch < 0 ? beg + ldm<true>(T.leaf_count + j) : T.node_end[j];
    cnt = end - beg;
    const double bj = level_box(T, lj);
    const int Xj[3] = {int(compact3(pj)), int(compact3(pj >> 1)), int(compact3(pj >> 2))};
    for (int d = 0; d < 3; ++d)
      off[d] = -periodic_shift_d(center_of(T.L, l, Xl[d]), center_of(T.L, lj, Xj[d]), T.L, b, bj) * T.L;
  }
  M.beg[src] = beg;
  M.cnt[src] = j >= 0 ? cnt : -1;
  M.lvl[src] = lj;
  M.pfx[src] = pj;
  for (int d = 0; d < 3; ++d) M.off[src][d] = off[d];
}

template <int NP>
__global__ void __launch_bounds__(MC_T, 1) k_mc(DevTree T, McArgs a) {
  extern __shared__ double2 sm2[];
  __shared__ Header h;
  __shared__ double red[4][32];
  __shared__ double c_level[MAXLV + 2];
  __shared__ ResMeta meta[2];
  __shared__ Receiver rs[MAX_RECV];
  __shared__ Proposal P;
  __shared__ int s_acc;
  __shared__ int s_rounds[9];  // grid-stride rounds of H*g update units
  __shared__ int s_pn;         // overflow pool fill
  __shared__ int s_stale;      // the accepted move invalidated the preloaded next particle
  const ResidualPoly<NP> poly(T);
  if (threadIdx.x >= 1 && threadIdx.x <= 8) {
    const long units = long(T.H) * threadIdx.x, gs = long(gridDim.x) * blockDim.x;
    s_rounds[threadIdx.x] = int((units + gs - 1) / gs);
  }
  if (threadIdx.x >= 2 && threadIdx.x < MAXLV + 2) {
    const double dk = level_dk(T, threadIdx.x);
    c_level[threadIdx.x] = dk * dk * dk / (8.0 * 3.14159265358979323846 * 3.14159265358979323846 *
                                           3.14159265358979323846) * level_dscale(threadIdx.x);
  }
  const int G = gridDim.x;
  const int gt = blockIdx.x * blockDim.x + threadIdx.x, gstride = G * blockDim.x;
  // window and root items run from the end of the grid, the difference and
  // update units from its start, so no block carries both
  const int gtr = gstride - 1 - gt;
  unsigned nbar = 0;
  // warp 0 runs one proposal ahead: the next index and displacement are
  // loaded at the top of a move, the next slot after the sums and the
  // particle itself after the decision, so the next resolve starts from them
  // unless the accepted move changed that slot or particle
  int i_cur = threadIdx.x < 32 ? a.idx[0] : 0;
  double d_cur[3] = {0, 0, 0};
  if (threadIdx.x < 32)
    for (int c = 0; c < 3; ++c) d_cur[c] = a.disp[c];
  Preload pre{-1, 0, 0, 0, 0};
  // An accepted move ends with an arrival at a grid barrier whose wait is
  // deferred: the next move's resolve and phase tables read only the
  // preloaded particle and the static refinement bitmaps, so they run before
  // the wait; the near-field source lists, the pool fill and the sums, which
  // read what other blocks update or commit, run after it. When the accepted
  // move invalidated the preload, the wait comes first.
  bool pend = false;
  for (int m = 0; m < a.n_moves; ++m) {
    const bool more = threadIdx.x < 32 && m + 1 < a.n_moves;
    const int i_next = more ? a.idx[m + 1] : 0;
    double d_next[3] = {0, 0, 0};
    if (more)
      for (int c = 0; c < 3; ++c) d_next[c] = a.disp[3 * (m + 1) + c];
    if (pend && s_stale) {
      if (!mc_wait(T, a, nbar)) return;
      pend = false;
    }
    resolve<true>(T, i_cur, d_cur, h, &pre);
    const int lo_max = h.depth_o - 2, lt_max = h.depth_t - 2;
    // the incoming rows of both paths go to L2 while the tables are built
    for (int k = gt; k < T.H; k += gstride) {
      for (int l = 2; l <= lo_max; ++l)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(T.inc + size_t(h.path_o[l] - T.pw_base) * T.H + k));
      for (int l = 2; l <= lt_max; ++l)
        asm volatile("prefetch.global.L2 [%0];" ::"l"(T.inc + size_t(h.path_t[l] - T.pw_base) * T.H + k));
    }
    const int uo = min(h.depth_o - 1, T.pw_hi), ut = min(h.depth_t - 1, T.pw_hi);
    const int per = 3 * (2 * T.n_window + 1) + max(max(uo, ut) - 1, 0) * 3 * (2 * T.n_diff + 1);
    Tables to, oo;
    alloc_tables(sm2, T, oo);
    alloc_tables(sm2 + per, T, to);
    // near-field source lists on threads 0..71, phase tables on the rest
    auto source_lists = [&]() {
      if (threadIdx.x == 0) s_pn = __ldcg(T.pool_n);
      const int p = threadIdx.x / 36, src = threadIdx.x % 36;
      const int lv = (p == 0 ? h.depth_t : h.depth_o) - 1;
      res_meta(T, p == 0 ? h.path_t[lv] : h.path_o[lv], lv, p == 0 ? h.Xt[lv] : h.Xo[lv], src, meta[p]);
    };
    if (threadIdx.x < 72) {
      if (!pend) source_lists();
    } else {
      const int nthr = blockDim.x - 72, t = threadIdx.x - 72;
      build_tables(T, h.xo, h.q, h.Xo, uo, oo, t, nthr);
      build_tables(T, h.xt, h.q, h.Xt, ut, to, t, nthr);
    }
    if (pend) {
      if (!mc_wait(T, a, nbar)) return;
      pend = false;
      if (threadIdx.x < 72) source_lists();
    }
    __syncthreads();
    if (threadIdx.x < 2) {
      ResMeta& M = meta[threadIdx.x];
      int s = 0;
      for (int src = 0; src < 36; ++src) {
        M.pre[src] = s;
        s += max(M.cnt[src], 0);
      }
      M.pre[36] = s;
    }
    __syncthreads();
    double acc[4] = {0, 0, 0, 0};
    // near field of the target and the origin (src/energy_shift.cpp:233-302):
    // the pairs of both paths split evenly over the blocks. The first pair's
    // source is loaded before the mode sums so the two latencies overlap.
    const int nt = meta[0].pre[36], no = meta[1].pre[36], np = nt + no;
    const int e0 = int((long(blockIdx.x) * np) / G), e1 = int((long(blockIdx.x + 1) * np) / G);
    const double eps = 2.220446049250313e-16;
    int e = e0 + threadIdx.x;
    double4 src_first = make_double4(0, 0, 0, 0);
    int p_first = 0, srci_first = 0;
    if (e < e1) {
      p_first = e < nt ? 0 : 1;
      const ResMeta& M = meta[p_first];
      const int ee = p_first == 0 ? e : e - nt;
      int lo = 0, hi = 36;  // largest src with pre[src] <= ee
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (M.pre[mid] <= ee) lo = mid;
        else hi = mid;
      }
      srci_first = lo;
      const int sl = M.beg[lo] + (ee - M.pre[lo]);
      src_first = make_double4(__ldcg(T.sx + sl), __ldcg(T.sy + sl), __ldcg(T.sz + sl), __ldcg(T.sq + sl));
    }
    // window (src/energy_shift.cpp:72-90)
    for (int k = gtr; k < T.Hw; k += gstride) {
      const double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
      const double2 g = __ldcg(T.out_root + k);
      const double ar = t.x - o.x, ai = t.y - o.y, br = g.x - o.x, bi = g.y - o.y;
      acc[0] += (ar * br + ai * bi) * T.W[k];
    }
    // difference (src/energy_shift.cpp:92-140)
    {
      const int base = T.pw_base, d = T.dd;
      for (int k = gt; k < T.H; k += gstride) {
        const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
        double s = 0;
        for (int l = 2; l <= lo_max; ++l) {
          const double2 o = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
          const double2 c = __ldcg(T.inc + size_t(h.path_o[l] - base) * T.H + k);
          s -= (o.x * c.x - o.y * c.y - (o.x * o.x + o.y * o.y)) * c_level[l];
        }
        for (int l = 2; l <= lt_max; ++l) {
          const double2 t = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
          const double2 c = __ldcg(T.inc + size_t(h.path_t[l] - base) * T.H + k);
          s += (t.x * c.x - t.y * c.y) * c_level[l];
        }
        acc[1] += s * T.D2[k];
      }
    }
    {
      for (; e < e1; e += blockDim.x) {
        int p, srci;
        double4 v;
        if (e == e0 + int(threadIdx.x)) {
          p = p_first;
          srci = srci_first;
          v = src_first;
        } else {
          p = e < nt ? 0 : 1;
          const ResMeta& M = meta[p];
          const int ee = p == 0 ? e : e - nt;
          int lo = 0, hi = 36;
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (M.pre[mid] <= ee) lo = mid;
            else hi = mid;
          }
          srci = lo;
          const int sl = M.beg[lo] + (ee - M.pre[lo]);
          v = make_double4(__ldcg(T.sx + sl), __ldcg(T.sy + sl), __ldcg(T.sz + sl), __ldcg(T.sq + sl));
        }
        const ResMeta& M = meta[p];
        const int lv = (p == 0 ? h.depth_t : h.depth_o) - 1;
        const double b = level_box(T, lv);
        const double* x = p == 0 ? h.xt : h.xo;
        const double dx = x[0] - (v.x + M.off[srci][0]), dy = x[1] - (v.y + M.off[srci][1]),
                     dz = x[2] - (v.z + M.off[srci][2]);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > eps && r2 < b * b) acc[2 + p] += v.w * poly(sqrt(r2), b);
      }
      // arrivals parked in the overflow pool that belong to a source's subtree
      const int pn = s_pn;
      for (int e2 = gt; e2 < 2 * 36 * pn; e2 += gstride) {
        const int p = e2 / (36 * pn), sj = (e2 / pn) % 36, q = e2 % pn;
        const ResMeta& M = meta[p];
        if (M.cnt[sj] < 0 || __ldcg(T.p_orig + q) < 0) continue;
        const int pl = __ldcg(T.p_leaf + q);
        const int ll = T.node_level[pl], lj = M.lvl[sj];
        if (ll < lj || (T.node_prefix[pl] >> (3 * (ll - lj))) != M.pfx[sj]) continue;
        const int lv = (p == 0 ? h.depth_t : h.depth_o) - 1;
        const double b = level_box(T, lv);
        const double* x = p == 0 ? h.xt : h.xo;
        const double dx = x[0] - (__ldcg(T.px + q) + M.off[sj][0]), dy = x[1] - (__ldcg(T.py + q) + M.off[sj][1]),
                     dz = x[2] - (__ldcg(T.pz + q) + M.off[sj][2]);
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (r2 > eps && r2 < b * b) acc[2 + p] += __ldcg(T.pq + q) * poly(sqrt(r2), b);
      }
      acc[2] *= h.q;
      acc[3] *= h.q;
    }
    const int s_next = threadIdx.x < 32 ? __ldcg(T.orig_slot + i_next) : 0;
    block_sum4_t0(acc, red);
    double* part = a.partials + size_t(m & 1) * 4 * G;
    if (threadIdx.x == 0)
      for (int c = 0; c < 4; ++c) part[4 * blockIdx.x + c] = acc[c];
    if (!mc_barrier(T, a, nbar)) return;
    // every block reduces the same partials in the same order: one warp,
    // lane-strided sums then a shuffle tree into lane 0
    double tot[4] = {0, 0, 0, 0};
    if (threadIdx.x < 32) {
      for (int b = threadIdx.x; b < G; b += 32)
        for (int c = 0; c < 4; ++c) tot[c] += __ldcg(part + 4 * b + c);
#pragma unroll
      for (int c = 0; c < 4; ++c)
        for (int o = 16; o > 0; o >>= 1) tot[c] += __shfl_down_sync(0xffffffffu, tot[c], o);
    }
    if (threadIdx.x == 0) {
      const double dEw = tot[0] * a.c_window;
      double self = 0;
      if (h.dr != 0) self = poly(h.dr, level_box(T, 2)) * h.q * h.q;
      const double dE = dEw + tot[1] + tot[2] - tot[3] - self;
      const int accd = a.u[m] < exp(-a.beta * dE) ? 1 : 0;
      s_acc = accd;
      if (blockIdx.x == 0) {
        if (a.dE_out) a.dE_out[m] = dE;
        if (a.acc_out) a.acc_out[m] = accd;
        // algorithmic bytes of the dE evaluation: root and incoming rows, W and
        // D, 32 B per near-field source particle
        const int nlev = max(lo_max - 1, 0) + max(lt_max - 1, 0);
        atomicAdd(&T.work[2], 24ull * T.Hw + 16ull * nlev * T.H + 8ull * T.H +
                                  32ull * (unsigned long long)(meta[0].pre[36] + meta[1].pre[36]));
      }
    }
    __syncthreads();
    if (threadIdx.x < 32) {
      // the next particle's slot is stale when an accepted move changed leaves
      // (its own slot and the slot of the particle swapped into its place) or
      // moved that very particle
      const bool stale = s_acc && (h.path_o[h.depth_o - 1] != h.path_t[h.depth_t - 1] || i_next == h.i_orig);
      if (threadIdx.x == 0) s_stale = stale;
      // a kept slot is loaded now; an accepted move writes other slots only,
      // and the commit of a same-leaf move of this very particle marks it stale
      pre.s = -1;
      if (!stale) {
        pre.s = s_next;
        if (s_next < T.n_slots) {
          pre.x = __ldcg(T.sx + s_next);
          pre.y = __ldcg(T.sy + s_next);
          pre.z = __ldcg(T.sz + s_next);
          pre.q = __ldcg(T.sq + s_next);
        } else {
          const int pp = s_next - T.n_slots;
          pre.x = __ldcg(T.px + pp);
          pre.y = __ldcg(T.py + pp);
          pre.z = __ldcg(T.pz + pp);
          pre.q = __ldcg(T.pq + pp);
        }
      }
      i_cur = i_next;
      for (int c = 0; c < 3; ++c) d_cur[c] = d_next[c];
    }
    if (!s_acc) continue;
    // accept-and-update (src/tree.cpp:447-597)
    const int nr = build_receivers(T, h, rs);
    // receiver groups per mode: the g that minimises grid-stride rounds of
    // the H*g units times receivers per group
    int ng = 1;
    {
      int best = 1 << 30;
#pragma unroll
      for (int g = 1; g <= 8; ++g) {
        const int cost = s_rounds[g] * ((nr + g - 1) / g);
        if (cost < best) {
          best = cost;
          ng = g;
        }
      }
    }
    if (blockIdx.x == G / 2 && threadIdx.x == 0) {
      P.i_orig = h.i_orig;
      P.slot = h.slot;
      P.q = h.q;
      for (int c = 0; c < 3; ++c) {
        P.xo[c] = h.xo[c];
        P.xt[c] = h.xt[c];
      }
      P.depth_o = h.depth_o;
      P.depth_t = h.depth_t;
      for (int l = 0; l < MAXLV; ++l) {
        P.path_o[l] = l < h.depth_o ? h.path_o[l] : -1;
        P.path_t[l] = l < h.depth_t ? h.path_t[l] : -1;
      }
      P.accepted = 1;
      P.valid = 1;
      P.n_recv = nr;
      atomicAdd(&T.work[0], 1ull);
      atomicAdd(&T.work[1], 32ull * ((unsigned long long)T.Hw + (unsigned long long)nr * T.H));
      commit_move(T, P);
    }
    {
      // root window: out_root += t - o
      for (int k = gtr; k < T.Hw; k += gstride) {
        const double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
        double2 g = __ldcg(T.out_root + k);
        g = cadd(g, t);
        g = csub(g, o);
        T.out_root[k] = g;
      }
      // units (mode k, receiver group): a thread walks its group's receivers
      // in level runs. A periodic image multiplies a single-particle phase by
      // a cube root of unity w^-e, e = (k - n).f * 2^l mod 3, so each run
      // precomputes p, p w^-1, p w^-2 and a receiver only picks one.
      const int n = T.n_diff, d = T.dd;
      for (int u = gt; u < T.H * ng; u += gstride) {
        const int k = u % T.H, rg = u / T.H;
        const int r0 = (rg * nr) / ng, r1 = ((rg + 1) * nr) / ng;
        const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
        const int a0 = ((ix - n) % 3 + 3) % 3, a1 = ((iy - n) % 3 + 3) % 3, a2 = ((iz - n) % 3 + 3) % 3;
        int r = r0;
        while (r < r1) {
          const int l = rs[r].level;
          int re = r + 1;
          while (re < r1 && rs[re].level == l) ++re;
          const double2 pt0 = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
          const double2 po0 = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
          const double2 pt1 = cmul(pt0, root6(-2)), pt2 = cmul(pt0, root6(-4));
          const double2 po1 = cmul(po0, root6(-2)), po2 = cmul(po0, root6(-4));
          const int two_l = (l & 1) ? 2 : 1;
          for (; r < re; r += UPD_UNROLL) {
            double2 v[UPD_UNROLL];
            size_t off[UPD_UNROLL];
#pragma unroll
            for (int q = 0; q < UPD_UNROLL; ++q) {
              if (r + q < re) {
                const Receiver& R = rs[r + q];
                off[q] = size_t(R.off) * T.H + k;
                v[q] = R.is_out ? __ldcg(T.out + off[q]) : __ldcg(T.inc + off[q]);
              }
            }
#pragma unroll
            for (int q = 0; q < UPD_UNROLL; ++q) {
              if (r + q < re) {
                const Receiver& R = rs[r + q];
                // the exponent sum lies in [-12, 12]
                const int et = ((a0 * R.ft[0] + a1 * R.ft[1] + a2 * R.ft[2]) * two_l + 12) % 3;
                const int eo = ((a0 * R.fo[0] + a1 * R.fo[1] + a2 * R.fo[2]) * two_l + 12) % 3;
                double2 del = make_double2(0.0, 0.0);
                if (R.has_t) del = et == 0 ? pt0 : (et == 1 ? pt1 : pt2);
                if (R.has_o) del = csub(del, eo == 0 ? po0 : (eo == 1 ? po1 : po2));
                if (R.is_out) T.out[off[q]] = cadd(v[q], del);
                else T.inc[off[q]] = make_double2(v[q].x + del.x, v[q].y - del.y);
              }
            }
          }
          r = re;
        }
      }
    }
    mc_arrive(a, nbar);
    pend = true;
  }
}

// ---------------------------------------------------------------------------
// Replica sets: the Metropolis sequences of many independent trees in one
// launch, one thread block per tree (the block resolves, sums, decides,
// updates and commits its tree's moves with block barriers only). Small
// replicas do not need a whole GPU per move, so running them side by side
// fills the SMs with independent work.
constexpr int REP_T = 256;

template <int NP>
__global__ void __launch_bounds__(REP_T, 2) k_mc_rep(const DevTree* __restrict__ trees, int m, const int* __restrict__ idx,
                                                  const double* __restrict__ disp, const double* __restrict__ u,
                                                  double beta, double* __restrict__ dE_out, int* __restrict__ acc_out) {
  extern __shared__ double2 sm2[];
  __shared__ __align__(16) unsigned char ts_raw[sizeof(DevTree)];
  __shared__ Header h;
  __shared__ double red[4][32];
  __shared__ double c_level[MAXLV + 2];
  __shared__ Receiver rs[MAX_RECV];
  __shared__ Proposal P;
  __shared__ int s_acc;
  {
    const unsigned* src = reinterpret_cast<const unsigned*>(trees + blockIdx.x);
    unsigned* dst = reinterpret_cast<unsigned*>(ts_raw);
    for (int i = threadIdx.x; i < int(sizeof(DevTree) / 4); i += blockDim.x) dst[i] = src[i];
  }
  __syncthreads();
  const DevTree& T = *reinterpret_cast<const DevTree*>(ts_raw);
  const ResidualPoly<NP> poly(T);
  const double pi = 3.14159265358979323846;
  if (threadIdx.x >= 2 && threadIdx.x < MAXLV + 2) {
    const double dk = level_dk(T, threadIdx.x);
    c_level[threadIdx.x] = dk * dk * dk / (8.0 * pi * pi * pi) * level_dscale(threadIdx.x);
  }
  const double dk0 = T.delta_k[0];
  const double c_window = dk0 * dk0 * dk0 / (8.0 * pi * pi * pi);
  for (int mv = 0; mv < m; ++mv) {
    const size_t c = size_t(blockIdx.x) * m + mv;
    resolve(T, idx[c], disp + 3 * c, h);
    const int lo_max = h.depth_o - 2, lt_max = h.depth_t - 2;
    const int uo = min(h.depth_o - 1, T.pw_hi), ut = min(h.depth_t - 1, T.pw_hi);
    const int per = 3 * (2 * T.n_window + 1) + max(max(uo, ut) - 1, 0) * 3 * (2 * T.n_diff + 1);
    Tables to, oo;
    alloc_tables(sm2, T, oo);
    alloc_tables(sm2 + per, T, to);
    build_tables(T, h.xo, h.q, h.Xo, uo, oo, threadIdx.x, blockDim.x);
    build_tables(T, h.xt, h.q, h.Xt, ut, to, threadIdx.x, blockDim.x);
    __syncthreads();
    double acc[4] = {0, 0, 0, 0};
    for (int k = threadIdx.x; k < T.Hw; k += blockDim.x) {
      const double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
      const double2 g = T.out_root[k];
      const double ar = t.x - o.x, ai = t.y - o.y, br = g.x - o.x, bi = g.y - o.y;
      acc[0] += (ar * br + ai * bi) * T.W[k];
    }
    const int base = T.pw_base, d = T.dd, n = T.n_diff;
    for (int k = threadIdx.x; k < T.H; k += blockDim.x) {
      const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
      double sd = 0;
      for (int l = 2; l <= lo_max; ++l) {
        const double2 o = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
        const double2 cc = T.inc[size_t(h.path_o[l] - base) * T.H + k];
        sd -= (o.x * cc.x - o.y * cc.y - (o.x * o.x + o.y * o.y)) * c_level[l];
      }
      for (int l = 2; l <= lt_max; ++l) {
        const double2 t = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
        const double2 cc = T.inc[size_t(h.path_t[l] - base) * T.H + k];
        sd += (t.x * cc.x - t.y * cc.y) * c_level[l];
      }
      acc[1] += sd * T.D2[k];
    }
    const int lt = h.depth_t - 1, lo = h.depth_o - 1;
    acc[2] = residual_sum(T, poly, h.path_t[lt], lt, h.Xt[lt], h.xt);
    __syncthreads();  // the second call reuses the source-list arrays of the first
    acc[3] = residual_sum(T, poly, h.path_o[lo], lo, h.Xo[lo], h.xo);
    block_sum4(acc, red);
    if (threadIdx.x == 0) {
      double self = 0;
      if (h.dr != 0) self = poly(h.dr, level_box(T, 2)) * h.q * h.q;
      const double dE = acc[0] * c_window + acc[1] + (acc[2] - acc[3]) * h.q - self;
      const int accd = u[c] < exp(-beta * dE) ? 1 : 0;
      s_acc = accd;
      if (dE_out) dE_out[c] = dE;
      if (acc_out) acc_out[c] = accd;
    }
    __syncthreads();
    if (!s_acc) continue;
    // accept-and-update (src/tree.cpp:447-597) by this block
    const int nr = build_receivers(T, h, rs);
    if (threadIdx.x == 0) {
      P.i_orig = h.i_orig;
      P.slot = h.slot;
      P.q = h.q;
      for (int a = 0; a < 3; ++a) {
        P.xo[a] = h.xo[a];
        P.xt[a] = h.xt[a];
      }
      P.depth_o = h.depth_o;
      P.depth_t = h.depth_t;
      for (int l = 0; l < MAXLV; ++l) {
        P.path_o[l] = l < h.depth_o ? h.path_o[l] : -1;
        P.path_t[l] = l < h.depth_t ? h.path_t[l] : -1;
      }
      P.accepted = 1;
      P.valid = 1;
      P.n_recv = nr;
      atomicAdd(&T.work[0], 1ull);
      atomicAdd(&T.work[1], 32ull * ((unsigned long long)T.Hw + (unsigned long long)nr * T.H));
      commit_move(T, P);
    }
    for (int k = threadIdx.x; k < T.Hw; k += blockDim.x) {
      const double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
      T.out_root[k] = csub(cadd(T.out_root[k], t), o);
    }
    for (int k = threadIdx.x; k < T.H; k += blockDim.x) {
      const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
      const int a0 = ((ix - n) % 3 + 3) % 3, a1 = ((iy - n) % 3 + 3) % 3, a2 = ((iz - n) % 3 + 3) % 3;
      int r = 0;
      while (r < nr) {
        const int l = rs[r].level;
        int re = r + 1;
        while (re < nr && rs[re].level == l) ++re;
        const double2 pt0 = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
        const double2 po0 = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
        const double2 pt1 = cmul(pt0, root6(-2)), pt2 = cmul(pt0, root6(-4));
        const double2 po1 = cmul(po0, root6(-2)), po2 = cmul(po0, root6(-4));
        const int two_l = (l & 1) ? 2 : 1;
        for (; r < re; r += UPD_UNROLL) {
          double2 v[UPD_UNROLL];
          size_t off[UPD_UNROLL];
#pragma unroll
          for (int q = 0; q < UPD_UNROLL; ++q) {
            if (r + q < re) {
              const Receiver& R = rs[r + q];
              off[q] = size_t(R.off) * T.H + k;
              v[q] = R.is_out ? T.out[off[q]] : T.inc[off[q]];
            }
          }
#pragma unroll
          for (int q = 0; q < UPD_UNROLL; ++q) {
            if (r + q < re) {
              const Receiver& R = rs[r + q];
              // the exponent sum lies in [-12, 12]
              const int et = ((a0 * R.ft[0] + a1 * R.ft[1] + a2 * R.ft[2]) * two_l + 12) % 3;
              const int eo = ((a0 * R.fo[0] + a1 * R.fo[1] + a2 * R.fo[2]) * two_l + 12) % 3;
              double2 del = make_double2(0.0, 0.0);
              if (R.has_t) del = et == 0 ? pt0 : (et == 1 ? pt1 : pt2);
              if (R.has_o) del = csub(del, eo == 0 ? po0 : (eo == 1 ? po1 : po2));
              if (R.is_out) T.out[off[q]] = cadd(v[q], del);
              else T.inc[off[q]] = make_double2(v[q].x + del.x, v[q].y - del.y);
            }
          }
        }
        r = re;
      }
    }
    __syncthreads();
  }
}

using McRepKernel = void (*)(const DevTree*, int, const int*, const double*, const double*, double, double*, int*);
McRepKernel mc_rep_kernel(int np) {
  switch (np) {
    case 7: return k_mc_rep<7>;
    case 13: return k_mc_rep<13>;
    case 19: return k_mc_rep<19>;
    case 25: return k_mc_rep<25>;
    default: throw std::invalid_argument("unsupported residual polynomial");
  }
}

using McKernel = void (*)(DevTree, McArgs);
McKernel mc_kernel(int np) {
  switch (np) {
    case 7: return k_mc<7>;
    case 13: return k_mc<13>;
    case 19: return k_mc<19>;
    case 25: return k_mc<25>;
    default: throw std::invalid_argument("unsupported residual polynomial");
  }
}

// ---------------------------------------------------------------------------
// Many candidate moves against one state in one launch: one block per
// candidate evaluates its whole dE (resolve, phase tables, window and
// difference sums over all modes, both near-field sums, self term) and
// reduces it inside the block, so no grid-wide partials are needed and the
// candidates run side by side on all SMs. Candidates whose paths share boxes
// read the shared incoming rows through L2.
constexpr int SB_T = 256;

template <int NP>
__global__ void __launch_bounds__(SB_T) k_shift_batch(DevTree T, const int* __restrict__ idx,
                                                      const double* __restrict__ disp, double c_window,
                                                      double* __restrict__ dE_out) {
  extern __shared__ double2 sm2[];
  __shared__ Header h;
  __shared__ double red[4][32];
  __shared__ double c_level[MAXLV + 2];
  const ResidualPoly<NP> poly(T);
  if (threadIdx.x >= 2 && threadIdx.x < MAXLV + 2) {
    const double dk = level_dk(T, threadIdx.x);
    c_level[threadIdx.x] = dk * dk * dk / (8.0 * 3.14159265358979323846 * 3.14159265358979323846 *
                                           3.14159265358979323846) * level_dscale(threadIdx.x);
  }
  const int c = blockIdx.x;
  resolve(T, idx[c], disp + 3 * c, h);
  const int lo_max = h.depth_o - 2, lt_max = h.depth_t - 2;
  const int per = 3 * (2 * T.n_window + 1) + max(max(lo_max, lt_max) - 1, 0) * 3 * (2 * T.n_diff + 1);
  Tables to, oo;
  alloc_tables(sm2, T, oo);
  alloc_tables(sm2 + per, T, to);
  build_tables(T, h.xo, h.q, h.Xo, lo_max, oo, threadIdx.x, blockDim.x);
  build_tables(T, h.xt, h.q, h.Xt, lt_max, to, threadIdx.x, blockDim.x);
  __syncthreads();
  double acc[4] = {0, 0, 0, 0};
  for (int k = threadIdx.x; k < T.Hw; k += blockDim.x) {
    const double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
    const double2 g = T.out_root[k];
    const double ar = t.x - o.x, ai = t.y - o.y, br = g.x - o.x, bi = g.y - o.y;
    acc[0] += (ar * br + ai * bi) * T.W[k];
  }
  const int base = T.pw_base, d = T.dd;
  for (int k = threadIdx.x; k < T.H; k += blockDim.x) {
    const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
    double sd = 0;
    for (int l = 2; l <= lo_max; ++l) {
      const double2 o = cmul(oo.lev[l][2][iz], cmul(oo.lev[l][1][iy], oo.lev[l][0][ix]));
      const double2 cc = T.inc[size_t(h.path_o[l] - base) * T.H + k];
      sd -= (o.x * cc.x - o.y * cc.y - (o.x * o.x + o.y * o.y)) * c_level[l];
    }
    for (int l = 2; l <= lt_max; ++l) {
      const double2 t = cmul(to.lev[l][2][iz], cmul(to.lev[l][1][iy], to.lev[l][0][ix]));
      const double2 cc = T.inc[size_t(h.path_t[l] - base) * T.H + k];
      sd += (t.x * cc.x - t.y * cc.y) * c_level[l];
    }
    acc[1] += sd * T.D2[k];
  }
  const int lt = h.depth_t - 1, lo = h.depth_o - 1;
  acc[2] = residual_sum(T, poly, h.path_t[lt], lt, h.Xt[lt], h.xt);
  __syncthreads();  // the second call reuses the source-list arrays of the first
  acc[3] = residual_sum(T, poly, h.path_o[lo], lo, h.Xo[lo], h.xo);
  block_sum4(acc, red);
  if (threadIdx.x == 0) {
    double self = 0;
    if (h.dr != 0) self = poly(h.dr, level_box(T, 2)) * h.q * h.q;
    dE_out[c] = acc[0] * c_window + acc[1] + (acc[2] - acc[3]) * h.q - self;
  }
}

using ShiftBatchKernel = void (*)(DevTree, const int*, const double*, double, double*);
ShiftBatchKernel shift_batch_kernel(int np) {
  switch (np) {
    case 7: return k_shift_batch<7>;
    case 13: return k_shift_batch<13>;
    case 19: return k_shift_batch<19>;
    case 25: return k_shift_batch<25>;
    default: throw std::invalid_argument("unsupported residual polynomial");
  }
}

// ---------------------------------------------------------------------------
// Potential and field at particles (one block per particle): the same terms
// as an energy shift, for the particle's own position only. With unit-charge
// phases u(k) = exp(-i k.x) and the particle's charge q, the interaction with
// all other particles is
//   c_w sum_{k != 0} W Re(u conj(g - q u)) + sum_l c_l sum_k D (Re(u inc_l) - q |u|^2)
//       + sum_{j != i} q_j res(r_ij),
// and the returned potential adds 2 q C, C the particle's self terms of the
// energy (window: c_w/2 sum W - psi0(0)/(2 bs_2 C0); each difference level on
// its path: c_l/2 sum D_l - S_l), so that E = 1/2 sum_i q_i phi_i and
// phi_i = dE/dq_i. The field is -grad phi, each plane wave differentiating to
// -i k u.
template <int NP>
__global__ void __launch_bounds__(SB_T) k_potential_batch(DevTree T, const int* __restrict__ idx, double c_window,
                                                          double self_w, const double* __restrict__ Sl,
                                                          double* __restrict__ phi_out, double* __restrict__ field_out) {
  extern __shared__ double2 sm2[];
  __shared__ Header h;
  __shared__ double red[4][32];
  __shared__ double c_level[MAXLV + 2];
  const ResidualPoly<NP> poly(T);
  if (threadIdx.x >= 2 && threadIdx.x < MAXLV + 2) {
    const double dk = level_dk(T, threadIdx.x);
    c_level[threadIdx.x] = dk * dk * dk / (8.0 * 3.14159265358979323846 * 3.14159265358979323846 *
                                           3.14159265358979323846) * level_dscale(threadIdx.x);
  }
  const int c = blockIdx.x;
  const double zero3[3] = {0.0, 0.0, 0.0};
  resolve(T, idx[c], zero3, h);
  const int lo_max = h.depth_o - 2;
  Tables uu;
  alloc_tables(sm2, T, uu);
  build_tables(T, h.xo, 1.0, h.Xo, lo_max, uu, threadIdx.x, blockDim.x);
  __syncthreads();
  const double q = h.q;
  double v[4] = {0, 0, 0, 0};   // window, difference, residual
  double gw[4] = {0, 0, 0, 0};  // gradient of the window term
  double gd[4] = {0, 0, 0, 0};  // gradient of the difference terms
  double sums[4] = {0, 0, 0, 0};  // sum_{k != 0} W, sum D_2
  {
    const int dw = T.dw, nw = T.n_window;
    const double dk0 = T.delta_k[0];
    // the k = 0 mode is left out, as in Ewald summation: a neutral system has
    // g(0) = 0, but all particles but one carry the net charge -q, whose
    // k = 0 term is the uniform neutralising background's business
    const int k_zero = (nw * dw + nw) * dw + nw;
    for (int k = threadIdx.x; k < T.Hw; k += blockDim.x) {
      if (k == k_zero) continue;
      const double2 u = phase_at(uu.root, k, dw);
      const double2 g = T.out_root[k];
      const double bx = g.x - q * u.x, by = g.y - q * u.y;
      const double w = T.W[k];
      sums[0] += w;
      v[0] += (u.x * bx + u.y * by) * w;
      const double im = (u.y * bx - u.x * by) * w;  // Im(u conj(b))
      const int ix = k % dw, iy = (k / dw) % dw, iz = k / (dw * dw);
      gw[0] += dk0 * (ix - nw) * im;
      gw[1] += dk0 * (iy - nw) * im;
      gw[2] += dk0 * (iz - nw) * im;
    }
  }
  {
    const int base = T.pw_base, d = T.dd, n = T.n_diff;
    for (int k = threadIdx.x; k < T.H; k += blockDim.x) {
      const int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
      const double dd2 = T.D2[k];
      sums[1] += dd2;
      for (int l = 2; l <= lo_max; ++l) {
        const double2 u = cmul(uu.lev[l][2][iz], cmul(uu.lev[l][1][iy], uu.lev[l][0][ix]));
        const double2 cc = T.inc[size_t(h.path_o[l] - base) * T.H + k];
        const double f = c_level[l] * dd2;
        v[1] += (u.x * cc.x - u.y * cc.y - q * (u.x * u.x + u.y * u.y)) * f;
        const double im = (u.x * cc.y + u.y * cc.x) * f;  // Im(u cc)
        const double dkl = level_dk(T, l);
        gd[0] += dkl * (ix - n) * im;
        gd[1] += dkl * (iy - n) * im;
        gd[2] += dkl * (iz - n) * im;
      }
    }
  }
  // near field: the source lists of the particle's leaf, the particle itself excluded
  double gr[3] = {0, 0, 0};
  {
    const int lv = h.depth_o - 1;
    const int leaf = h.path_o[lv];
    const double b = level_box(T, lv);
    const double eps = 2.220446049250313e-16;
    __shared__ int m_beg[36], m_pre[37];
    __shared__ double m_off[36][3];
    if (threadIdx.x < 36) {
      const int src = threadIdx.x;
      int j = -1;
      if (src == 0) j = leaf;
      else if (src <= 27) j = (src - 1 == 13) ? -1 : T.col27[size_t(leaf) * 27 + (src - 1)];
      else j = T.coarse8[size_t(leaf) * 8 + (src - 28)];
      int beg = 0, cnt = 0;
      double off[3] = {0, 0, 0};
      if (j >= 0) {
        const int lj = T.node_level[j];
        const unsigned long long pj = T.node_prefix[j];
        beg = T.node_begin[j];
        cnt = (T.node_child0[j] < 0 ? beg + T.leaf_count[j] : T.node_end[j]) - beg;
        const double bj = level_box(T, lj);
        const int Xj[3] = {int(compact3(pj)), int(compact3(pj >> 1)), int(compact3(pj >> 2))};
        for (int a = 0; a < 3; ++a)
          off[a] = -periodic_shift_d(center_of(T.L, lv, h.Xo[lv][a]), center_of(T.L, lj, Xj[a]), T.L, b, bj) * T.L;
      }
      m_beg[src] = beg;
      m_pre[src] = cnt;
      for (int a = 0; a < 3; ++a) m_off[src][a] = off[a];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int acc = 0;
      for (int src = 0; src < 36; ++src) {
        const int nn = m_pre[src];
        m_pre[src] = acc;
        acc += nn;
      }
      m_pre[36] = acc;
    }
    __syncthreads();
    const int total = m_pre[36];
    for (int e = threadIdx.x; e < total; e += blockDim.x) {
      int lo = 0, hi = 36;
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (m_pre[mid] <= e) lo = mid;
        else hi = mid;
      }
      const int s = m_beg[lo] + (e - m_pre[lo]);
      const double dx = h.xo[0] - (T.sx[s] + m_off[lo][0]), dy = h.xo[1] - (T.sy[s] + m_off[lo][1]),
                   dz = h.xo[2] - (T.sz[s] + m_off[lo][2]);
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > eps && r2 < b * b) {
        const double r = sqrt(r2), qj = T.sq[s];
        v[2] += qj * poly(r, b);
        const double g = qj * poly.deriv(r, b) / r;
        gr[0] += g * dx;
        gr[1] += g * dy;
        gr[2] += g * dz;
      }
    }
    // arrivals parked in the overflow pool that belong to a source's subtree
    // are folded into the slots by the host before this kernel runs
  }
  double v4[4] = {v[0], v[1], v[2], 0.0};
  block_sum4(v4, red);
  double w4[4] = {gw[0], gw[1], gw[2], 0.0};
  block_sum4(w4, red);
  double d4[4] = {gd[0], gd[1], gd[2], 0.0};
  block_sum4(d4, red);
  double r4[4] = {gr[0], gr[1], gr[2], 0.0};
  block_sum4(r4, red);
  block_sum4(sums, red);
  if (threadIdx.x == 0) {
    double cself = 0.5 * c_window * sums[0] - self_w;
    for (int l = 2; l <= lo_max; ++l) cself += 0.5 * c_level[l] * sums[1] - Sl[l];
    phi_out[c] = v4[0] * c_window + v4[1] + v4[2] + 2.0 * q * cself;
    if (field_out)
      for (int a = 0; a < 3; ++a) field_out[3 * size_t(c) + a] = -(w4[a] * c_window + d4[a] + r4[a]);
  }
}

using PotentialKernel = void (*)(DevTree, const int*, double, double, const double*, double*, double*);
PotentialKernel potential_kernel(int np) {
  switch (np) {
    case 7: return k_potential_batch<7>;
    case 13: return k_potential_batch<13>;
    case 19: return k_potential_batch<19>;
    case 25: return k_potential_batch<25>;
    default: throw std::invalid_argument("unsupported residual polynomial");
  }
}

// the shift kernel for a residual polynomial of np coefficients (3, 6, 9, 12 digits)
using ShiftKernel = void (*)(DevTree, ShiftArgs);
ShiftKernel shift_kernel(int np) {
  switch (np) {
    case 7: return k_shift<7>;
    case 13: return k_shift<13>;
    case 19: return k_shift<19>;
    case 25: return k_shift<25>;
    default: throw std::invalid_argument("unsupported residual polynomial");
  }
}

size_t tables_smem(const DevTree& T, int lmax, int copies) {
  size_t per = 3 * size_t(2 * T.n_window + 1) + size_t(std::max(lmax - 1, 0)) * 3 * (2 * T.n_diff + 1);
  return per * copies * sizeof(double2);
}

}  // namespace

// ---------------------------------------------------------------------------
void DmkTree::launch_shift(const int* d_idx, const double* d_disp, const double* d_u, double beta, int move, int mode,
                           double* d_dE, int* d_acc) {
  DevTree& D = dev_;
  const double pi = 3.14159265358979323846;
  ShiftArgs a{};
  a.idx = d_idx;
  a.disp = d_disp;
  a.u = d_u;
  a.beta = beta;
  a.move = move;
  a.mode = mode;
  a.dE_out = d_dE;
  a.acc_out = d_acc;
  a.c_window = std::pow(D.delta_k[0], 3) / std::pow(2 * pi, 3);
  a.partials = D.partials;
  a.counter = D.counter;
  a.prop = D.prop;
  ensure_move_resources();
  a.cur = use_cursor_ ? d_cursor_ : nullptr;
  a.ptab = ptab_;
  a.ptab_per = ptab_per_;
  size_t smem = tables_smem(D, D.max_depth, 2);
  time_begin(0);
  shift_kernel(D.n_poly)<<<unsigned(shift_grid_), SH_T, smem, st_>>>(D, a);
  PDMK_LAUNCH_CHECK();
  time_end(0);
}

void DmkTree::launch_shift_cursor(int move) {
  // proposals, outputs, mode and beta come from *d_cursor_ at run time
  use_cursor_ = true;
  launch_shift(nullptr, nullptr, nullptr, 0.0, move, 1, nullptr, nullptr);
  use_cursor_ = false;
}

// Per-tree resources of the move kernels, set up before any graph capture
// (no allocation or attribute change may happen inside a capture).
void DmkTree::ensure_move_resources() {
  DevTree& D = dev_;
  if (!ptab_) {
    ptab_per_ = 3L * (2 * D.n_window + 1) + long(MAX_LEVELS + 1) * 3 * (2 * D.n_diff + 1);
    ptab_ = static_cast<double2*>(alloc(sizeof(double2) * 2 * size_t(ptab_per_)));
    d_cursor_ = static_cast<MoveCursor*>(alloc(sizeof(MoveCursor)));
  }
  ensure_shift_config();
}

// Grid size and dynamic shared memory limit of the shift kernel (no allocation).
void DmkTree::ensure_shift_config() {
  DevTree& D = dev_;
  if (shift_grid_ == 0) {
    int dev = 0, sms = 148;
    PDMK_CUDA(cudaGetDevice(&dev));
    PDMK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    shift_grid_ = 2 + sms;
    const size_t smem = tables_smem(D, D.max_depth, 2);
    raise_smem_limit(reinterpret_cast<const void*>(shift_kernel(D.n_poly)), smem);
  }
}

// Capture kGraphMoves sequential moves (shift, update, commit) into one
// executable graph; with timed != 0 external event records bracket each
// update so its duration can be read after the graph ran.
void DmkTree::build_mc_graph(int timed) {
  ensure_move_resources();
  if (timed && graph_ev_.empty()) {
    graph_ev_.resize(2 * kGraphMoves);
    for (auto& e : graph_ev_) PDMK_CUDA(cudaEventCreate(&e));
  }
  cudaGraph_t g;
  const long long launches0 = g_launch_count.load();  // captured launches do not run here
  capturing_ = true;
  PDMK_CUDA(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
  try {
    for (int b = 0; b < kGraphMoves; ++b) {
      launch_shift_cursor(b);
      if (timed) PDMK_CUDA(cudaEventRecordWithFlags(graph_ev_[2 * b], st_, cudaEventRecordExternal));
      launch_update();
      if (timed) PDMK_CUDA(cudaEventRecordWithFlags(graph_ev_[2 * b + 1], st_, cudaEventRecordExternal));
    }
  } catch (...) {
    capturing_ = false;
    cudaStreamEndCapture(st_, &g);
    throw;
  }
  PDMK_CUDA(cudaStreamEndCapture(st_, &g));
  capturing_ = false;
  g_launch_count.store(launches0);
  PDMK_CUDA(cudaGraphInstantiate(&mc_graph_[timed], g, 0));
  PDMK_CUDA(cudaGraphDestroy(g));
}

void DmkTree::launch_update() {
  DevTree& D = dev_;
  const int levels = std::max(D.pw_hi - 1, 0);
  // rows: root, up to 2 x 28 receivers per expansion level, commit
  // x: one mode per thread; y: receiver ranges, enough for ~16 warps per SM
  const int gx = (std::max(D.H, D.Hw) + UPD_T - 1) / UPD_T;
  const int gy = std::max(1, std::min(8, (16 * (shift_grid_ - 2) * 32 / UPD_T + gx - 1) / std::max(gx, 1)));
  (void)levels;
  const dim3 grid{unsigned(gx), unsigned(gy), 1u};
  time_begin(1);
  k_update<<<grid, UPD_T, 0, st_>>>(D, ptab_, ptab_per_);
  PDMK_LAUNCH_CHECK();
  time_end(1);
}


cudaEvent_t DmkTree::take_event() {
  if (!ev_pool_.empty()) {
    cudaEvent_t e = ev_pool_.back();
    ev_pool_.pop_back();
    return e;
  }
  cudaEvent_t e;
  PDMK_CUDA(cudaEventCreate(&e));
  return e;
}

void DmkTree::time_begin(int cls) {
  if (!timing_ || capturing_) return;
  ev_cur_[cls] = take_event();
  PDMK_CUDA(cudaEventRecord(ev_cur_[cls], st_));
}

void DmkTree::time_end(int cls) {
  if (!timing_ || capturing_ || !ev_cur_[cls]) return;
  cudaEvent_t e = take_event();
  PDMK_CUDA(cudaEventRecord(e, st_));
  ev_open_.push_back({cls, {ev_cur_[cls], e}});
  ev_cur_[cls] = nullptr;
}

void DmkTree::get_timing(double* out, bool reset) {
  PDMK_CUDA(cudaStreamSynchronize(st_));
  for (auto& o : ev_open_) {
    float ms = 0;
    PDMK_CUDA(cudaEventElapsedTime(&ms, o.second.first, o.second.second));
    t_ms_[o.first] += ms;
    t_cnt_[o.first] += 1;
    ev_pool_.push_back(o.second.first);
    ev_pool_.push_back(o.second.second);
  }
  ev_open_.clear();
  for (int c = 0; c < 4; ++c) {
    out[2 * c] = t_ms_[c];
    out[2 * c + 1] = double(t_cnt_[c]);
    if (reset) {
      t_ms_[c] = 0;
      t_cnt_[c] = 0;
    }
  }
}

void DmkTree::get_work(double* out) {
  unsigned long long w[3];
  PDMK_CUDA(cudaMemcpyAsync(w, dev_.work, sizeof(w), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  for (int c = 0; c < 3; ++c) out[c] = double(w[c]);
}

void DmkTree::reset_work() { PDMK_CUDA(cudaMemsetAsync(dev_.work, 0, 3 * sizeof(unsigned long long), st_)); }

double DmkTree::eval_shift_energy(long i, double dx, double dy, double dz, double* parts) {
  double disp[3] = {dx, dy, dz};
  int ii = int(i);
  PDMK_CUDA(cudaMemcpyAsync(d_one_idx_, &ii, sizeof(int), cudaMemcpyHostToDevice, st_));
  PDMK_CUDA(cudaMemcpyAsync(d_one_disp_, disp, sizeof(disp), cudaMemcpyHostToDevice, st_));
  launch_shift(d_one_idx_, d_one_disp_, nullptr, 0.0, 0, 0, nullptr, nullptr);
  Proposal P;
  PDMK_CUDA(cudaMemcpyAsync(&P, dev_.prop, sizeof(Proposal), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  if (parts)
    for (int c = 0; c < 5; ++c) parts[c] = P.parts[c];
  last_i_ = i;
  last_d_[0] = dx;
  last_d_[1] = dy;
  last_d_[2] = dz;
  last_valid_ = true;
  return P.dE;
}

void DmkTree::update_shift(long i, double dx, double dy, double dz) {
  // the reference requires the same arguments as the preceding
  // eval_shift_energy (src/tree.cpp:471-489); recompute when they differ
  if (!(last_valid_ && last_i_ == i && last_d_[0] == dx && last_d_[1] == dy && last_d_[2] == dz))
    eval_shift_energy(i, dx, dy, dz, nullptr);
  int one = 1;
  PDMK_CUDA(cudaMemcpyAsync(&dev_.prop->accepted, &one, sizeof(int), cudaMemcpyHostToDevice, st_));
  launch_update();
  PDMK_CUDA(cudaStreamSynchronize(st_));
  last_valid_ = false;
  diff_cached_ = false;
  moved_ = true;
}

// One cooperative launch per kMcChunk moves on every SM (k_mc). The grid is
// the SM count, which the occupancy query confirms can be co-resident; the
// cooperative launch refuses to start otherwise, so the grid barriers inside
// cannot wait on a block that never runs.
void DmkTree::mc_run_persistent(int n_moves, const int* d_idx, const double* d_disp, const double* d_u, double beta,
                                double* d_dE, int* d_acc) {
  DevTree& D = dev_;
  const size_t smem = tables_smem(D, D.max_depth, 2);
  const McKernel kern = mc_kernel(D.n_poly);
  if (mc_grid_ == 0) {
    int dev = 0, sms = 0, coop = 0;
    PDMK_CUDA(cudaGetDevice(&dev));
    PDMK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PDMK_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
    if (!coop) throw CudaError("device does not support cooperative launches");
    raise_smem_limit(reinterpret_cast<const void*>(kern), smem);
    int per_sm = 0;
    PDMK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, MC_T, smem));
    if (per_sm < 1) throw CudaError("persistent Metropolis kernel does not fit on one SM");
    mc_partials_ = static_cast<double*>(alloc(sizeof(double) * 8 * size_t(sms)));
    mc_sync_ = static_cast<unsigned int*>(alloc(64));
    mc_grid_ = sms;
  }
  const double pi = 3.14159265358979323846;
  for (int m0 = 0; m0 < n_moves; m0 += kMcChunk) {
    const int cnt = std::min(kMcChunk, n_moves - m0);
    PDMK_CUDA(cudaMemsetAsync(mc_sync_, 0, 64, st_));
    McArgs a{};
    a.idx = d_idx + m0;
    a.disp = d_disp + 3 * size_t(m0);
    a.u = d_u + m0;
    a.beta = beta;
    a.n_moves = cnt;
    a.dE_out = d_dE ? d_dE + m0 : nullptr;
    a.acc_out = d_acc ? d_acc + m0 : nullptr;
    a.c_window = std::pow(D.delta_k[0], 3) / std::pow(2 * pi, 3);
    a.partials = mc_partials_;
    a.arrivals = mc_sync_;
    a.spin_limit = 1LL << 21;  // about a second of polling
    void* args[] = {&D, &a};
    time_begin(2);
    PDMK_CUDA(cudaLaunchCooperativeKernel(reinterpret_cast<const void*>(kern), dim3(unsigned(mc_grid_)),
                                          dim3(unsigned(MC_T)), args, smem, st_));
    PDMK_LAUNCH_CHECK();
    time_end(2);
  }
}

void DmkTree::mc_run_device(int n_moves, const int* d_idx, const double* d_disp, const double* d_u, double beta,
                            double* d_dE, int* d_acc) {
  if (mc_mode_ == 0) {
    if (n_moves > 0) mc_run_persistent(n_moves, d_idx, d_disp, d_u, beta, d_dE, d_acc);
    last_valid_ = false;
    diff_cached_ = false;
    moved_ = true;
    return;
  }
  ensure_move_resources();
  int m = 0;
  // whole batches run as one captured graph each; with timing on, one batch
  // in kTimedEvery runs the graph variant whose updates are bracketed by
  // event records (those records slow the graph, so only a sample carries them)
  while (n_moves - m >= kGraphMoves) {
    const int timed = (timing_ && (timed_batches_++ % kTimedEvery) == 0) ? 1 : 0;
    if (!mc_graph_[timed]) build_mc_graph(timed);
    MoveCursor c{d_idx, d_disp, d_u, d_dE, d_acc, m, 1, beta};
    PDMK_CUDA(cudaMemcpyAsync(d_cursor_, &c, sizeof(c), cudaMemcpyHostToDevice, st_));
    PDMK_CUDA(cudaGraphLaunch(mc_graph_[timed], st_));
    g_launch_count.fetch_add(2 * kGraphMoves, std::memory_order_relaxed);  // shift + update per move
    if (timed) {
      // the events are reused by the next launch: read them now
      PDMK_CUDA(cudaStreamSynchronize(st_));
      for (int b = 0; b < kGraphMoves; ++b) {
        float ms = 0;
        PDMK_CUDA(cudaEventElapsedTime(&ms, graph_ev_[2 * b], graph_ev_[2 * b + 1]));
        t_ms_[1] += ms;
        t_cnt_[1] += 1;
      }
    }
    m += kGraphMoves;
  }
  for (; m < n_moves; ++m) {
    launch_shift(d_idx, d_disp, d_u, beta, m, 1, d_dE, d_acc);
    launch_update();
  }
  last_valid_ = false;
  diff_cached_ = false;
  moved_ = true;
}

// All candidates in one launch of k_shift_batch (one block per candidate).
void DmkTree::shift_batch_device(int m, const int* d_idx, const double* d_disp, double* d_dE) {
  DevTree& D = dev_;
  if (m <= 0) return;
  const size_t smem = tables_smem(D, D.max_depth, 2);
  const ShiftBatchKernel kern = shift_batch_kernel(D.n_poly);
  raise_smem_limit(reinterpret_cast<const void*>(kern), smem);
  const double pi = 3.14159265358979323846;
  const double c_window = std::pow(D.delta_k[0], 3) / std::pow(2 * pi, 3);
  kern<<<unsigned(m), SB_T, smem, st_>>>(D, d_idx, d_disp, c_window, d_dE);
  PDMK_LAUNCH_CHECK();
  last_valid_ = false;
}


// ---------------------------------------------------------------------------
// Candidate batch through a fixed static device buffer. For callers that may
// not allocate device memory once the tree exists (a process that budgets its
// device memory up front, a host thread that must not enter the allocator
// between steps): the candidates' indices and displacements are staged into
// g_static_scratch and their energy shifts come back through it, and the
// batch is the same single launch of k_shift_batch as the allocating batch
// (one block per candidate; its phase tables live in shared memory). The
// array's device address is looked up once per device, with that device
// current. Nothing in the buffer has to start at zero: every call writes the
// inputs it reads, and the kernel writes every output before it is read.
// Calls that overlap in time on one device (two host threads, two trees on
// different streams) share the buffer and race; serialise them.
namespace {
constexpr int kStaticMaxMoves = 4096;  // candidates per call
constexpr size_t kOffIdx = 0;
constexpr size_t kOffDisp = kOffIdx + sizeof(int) * kStaticMaxMoves;
constexpr size_t kOffDE = kOffDisp + sizeof(double) * 3 * kStaticMaxMoves;
constexpr size_t kStaticBytes = kOffDE + sizeof(double) * kStaticMaxMoves;  // 144 KB

static __device__ __align__(256) unsigned char g_static_scratch[kStaticBytes];

unsigned char* static_scratch() {
  static std::mutex mu;
  static void* addr[64] = {};
  int dev = 0;
  PDMK_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) throw std::runtime_error("device ordinal out of range for the static scratch table");
  std::lock_guard<std::mutex> lock(mu);
  if (!addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_static_scratch);
    if (e != cudaSuccess || !p)
      throw CudaError(std::string("cudaGetSymbolAddress(static shift scratch): ") + cudaGetErrorString(e));
    addr[dev] = p;
  }
  return static_cast<unsigned char*>(addr[dev]);
}
}  // namespace

void DmkTree::shift_batch_static(int m, const long* h_idx, const double* h_disp, double* h_dE) {
  DevTree& D = dev_;
  if (m < 0 || m > kStaticMaxMoves)
    throw std::invalid_argument("static scratch holds at most " + std::to_string(kStaticMaxMoves) +
                                " candidates per call, got " + std::to_string(m));
  if (m == 0) return;
  unsigned char* base = static_scratch();
  int* s_idx = reinterpret_cast<int*>(base + kOffIdx);
  double* s_disp = reinterpret_cast<double*>(base + kOffDisp);
  double* s_dE = reinterpret_cast<double*>(base + kOffDE);
  // indices narrowed through a stack buffer (pageable copies are staged
  // before cudaMemcpyAsync returns, so the buffer may be reused at once)
  int chunk[512];
  for (int c0 = 0; c0 < m; c0 += 512) {
    const int nc = std::min(512, m - c0);
    for (int c = 0; c < nc; ++c) chunk[c] = int(h_idx[c0 + c]);
    PDMK_CUDA(cudaMemcpyAsync(s_idx + c0, chunk, sizeof(int) * nc, cudaMemcpyHostToDevice, st_));
  }
  PDMK_CUDA(cudaMemcpyAsync(s_disp, h_disp, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, st_));
  const size_t smem = tables_smem(D, D.max_depth, 2);
  const ShiftBatchKernel kern = shift_batch_kernel(D.n_poly);
  raise_smem_limit(reinterpret_cast<const void*>(kern), smem);
  const double pi = 3.14159265358979323846;
  const double c_window = std::pow(D.delta_k[0], 3) / std::pow(2 * pi, 3);
  kern<<<unsigned(m), SB_T, smem, st_>>>(D, s_idx, s_disp, c_window, s_dE);
  PDMK_LAUNCH_CHECK();
  PDMK_CUDA(cudaMemcpyAsync(h_dE, s_dE, sizeof(double) * m, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
}

// Metropolis sequences of many trees in one launch (k_mc_rep), ordered after
// all their streams' earlier work on the first tree's stream.
void DmkTree::replicas_mc_run(const std::vector<DmkTree*>& ts, int m, const int* d_idx, const double* d_disp,
                              const double* d_u, double beta, double* d_dE, int* d_acc) {
  if (ts.empty() || m <= 0) return;
  const int np = ts[0]->dev_.n_poly;
  size_t smem = 0;
  std::vector<DevTree> hd;
  for (DmkTree* t : ts) {
    if (t->dev_.n_poly != np) throw std::invalid_argument("replicas must share the digits setting");
    t->ensure_packed();
    smem = std::max(smem, tables_smem(t->dev_, t->dev_.max_depth, 2));
    hd.push_back(t->dev_);
  }
  cudaStream_t st = ts[0]->st_;
  std::vector<cudaEvent_t> evs(ts.size());
  for (auto& e : evs) PDMK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
  for (size_t i = 1; i < ts.size(); ++i) {
    PDMK_CUDA(cudaEventRecord(evs[i], ts[i]->st_));
    PDMK_CUDA(cudaStreamWaitEvent(st, evs[i], 0));
  }
  DevTree* d_trees = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_trees), sizeof(DevTree) * hd.size(), st));
  PDMK_CUDA(cudaMemcpyAsync(d_trees, hd.data(), sizeof(DevTree) * hd.size(), cudaMemcpyHostToDevice, st));
  const McRepKernel kern = mc_rep_kernel(np);
  raise_smem_limit(reinterpret_cast<const void*>(kern), smem);
  kern<<<unsigned(ts.size()), REP_T, smem, st>>>(d_trees, m, d_idx, d_disp, d_u, beta, d_dE, d_acc);
  PDMK_LAUNCH_CHECK();
  PDMK_CUDA(cudaFreeAsync(d_trees, st));
  PDMK_CUDA(cudaEventRecord(evs[0], st));
  for (size_t i = 1; i < ts.size(); ++i) PDMK_CUDA(cudaStreamWaitEvent(ts[i]->st_, evs[0], 0));
  for (auto& e : evs) PDMK_CUDA(cudaEventDestroy(e));  // released once the waits resolve
  for (DmkTree* t : ts) {
    t->last_valid_ = false;
    t->diff_cached_ = false;
    t->moved_ = true;
  }
}

// Potentials and fields at many particles in one launch (k_potential_batch).
void DmkTree::potential_batch(int m, const int* d_idx, double* d_phi, double* d_field) {
  DevTree& D = dev_;
  if (m <= 0) return;
  ensure_packed();  // the near-field source lists read the slots only
  prepare_box_lists();  // the per-level self terms S_l
  const size_t smem = tables_smem(D, D.max_depth, 1);
  const PotentialKernel kern = potential_kernel(D.n_poly);
  raise_smem_limit(reinterpret_cast<const void*>(kern), smem);
  const double pi = 3.14159265358979323846;
  const double c_window = std::pow(D.delta_k[0], 3) / std::pow(2 * pi, 3);
  const double self_w = ps_.psi0_0 / (2 * D.boxsize[2] * ps_.C0);
  kern<<<unsigned(m), SB_T, smem, st_>>>(D, d_idx, c_window, self_w, d_Sl_, d_phi, d_field);
  PDMK_LAUNCH_CHECK();
}

}  // namespace pdmk
