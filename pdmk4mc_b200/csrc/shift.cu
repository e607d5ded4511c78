// Single-particle energy shift, accept-and-update, and the device-side
// Metropolis loop (FP64).
//
// Reference counterparts: eval_shift_energy and its window / difference /
// residual parts (src/energy_shift.cpp:18-302), locate_particle
// (src/tree.cpp:204-236), form_outgoing_pw_single (src/planewave.cpp:157-181)
// and update_shift (src/tree.cpp:447-597).
//
// One trial move runs as: k_shift (grid-wide partial sums, the last block
// finishes dE and the Metropolis test and writes the Proposal record),
// k_update for the target path and then for the origin path (the two never
// race on a vector), and k_commit (particle membership). Every kernel reads
// the Proposal record, so the whole sequence is stream-ordered and can be
// captured in a CUDA graph.
#include <algorithm>
#include <cmath>
#include <vector>

#include "common.cuh"
#include "tree.hpp"

namespace pdmk {
namespace {

constexpr int SH_T = 256;
constexpr int MAXLV = MAX_LEVELS;

__device__ inline bool bm_get(const uint32_t* bm, uint64_t cell) { return (bm[cell >> 5] >> (cell & 31)) & 1u; }

__device__ inline int bm_rank(const DevTree& T, int level, uint64_t cell) {
  uint32_t w = T.bm[level][cell >> 5];
  return T.wprefix[level][cell >> 5] + __popc(w & ((1u << (cell & 31)) - 1u));
}

// Leaf path of a point: lane l resolves level l from the refinement bitmaps.
// Must be called by a full warp; returns the path length (leaf level + 1).
__device__ inline int warp_path(const DevTree& T, double x, double y, double z, int* path) {
  const int lane = threadIdx.x & 31;
  const uint64_t key = morton3(grid_coord(x, T.L), grid_coord(y, T.L), grid_coord(z, T.L));
  bool is_leaf = false;
  int node = -1;
  if (lane < T.max_depth) {
    const int l = lane;
    const uint64_t cell = l == 0 ? 0 : key >> (3 * (KEY_BITS - l));
    bool exists = l <= 1 || bm_get(T.bm[l - 1], cell >> 3);
    if (exists) {
      node = l == 0 ? 0 : (l == 1 ? 1 + int(cell) : T.level_start[l] + 8 * bm_rank(T, l - 1, cell >> 3) + int(cell & 7));
      bool refined = l <= T.maxref && bm_get(T.bm[l], cell);
      is_leaf = !refined;
    }
  }
  unsigned leaves = __ballot_sync(0xffffffffu, is_leaf);
  int leaf_level = __ffs(leaves) - 1;
  if (lane <= leaf_level) path[lane] = node;
  __syncwarp();
  return leaf_level + 1;
}

__device__ inline void node_center(const DevTree& T, int node, double* c, int* X) {
  uint64_t p = T.node_prefix[node];
  int l = T.node_level[node];
  double scale = ldexp(1.0, -l);
  X[0] = int(compact3(p));
  X[1] = int(compact3(p >> 1));
  X[2] = int(compact3(p >> 2));
  for (int d = 0; d < 3; ++d) c[d] = T.L * (double(X[d]) * scale + 0.5 * scale);
}

__device__ inline int periodic_shift_d(double xi, double xj, double L, double bi, double bj) {
  if (xi < bi && xj > (L - bj)) return 1;
  if (xi > (L - bi) && xj < bj) return -1;
  return 0;
}

__device__ inline double poly_res(const DevTree& T, double r, double b) {
  double xs = (r / b - 0.5) * 2.0;
  if (fabs(xs) >= 1.0) return 0;
  double v = 0;
  for (int i = 0; i < T.n_poly; ++i) v = fma(v, xs, T.poly[i]);
  return v / r;
}

// Phase tables exp(-i m dk_l x) per axis for one point on its path: slot 0
// is the root (window modes), slot l (2 <= l <= pw_hi) the level-l box on the
// path. The box-centred form uses the exact decentring root of unity.
struct Tables {
  double2* root[3];
  double2* lev[MAXLV + 2][3];
};

__device__ inline void axis_table(double xr, double dk, int M, int X, int n, int cnt, double scale, double2* dst,
                                  int part, int nparts) {
  // entries m = -n .. -n+cnt-1, split in nparts contiguous pieces
  int per = (cnt + nparts - 1) / nparts;
  int a = part * per, b = min(cnt, a + per);
  if (a >= b) return;
  int m0 = -n + a;
  double th = dk * xr;
  double s, c;
  sincos(-double(m0) * th, &s, &c);
  double2 v = make_double2(c * scale, s * scale);
  sincos(-th, &s, &c);
  const double2 step = make_double2(c, s);
  const int dec = M * (2 * X + 1);
  for (int t = a; t < b; ++t) {
    dst[t] = cmul(v, root6(-dec * (m0 + t - a)));
    v = cmul(v, step);
  }
}

// Fill tables for point x with path (levels 2..lmax); block-cooperative.
__device__ void build_tables(const DevTree& T, const double* x, double q, const int* path, int lmax, Tables& tb) {
  const int NP = 4;  // pieces per axis
  const int nlev = lmax >= 2 ? lmax - 1 : 0;
  const int ntask = (1 + nlev) * 3 * NP;
  for (int t = threadIdx.x; t < ntask; t += blockDim.x) {
    int part = t % NP, axis = (t / NP) % 3, slot = t / (3 * NP);
    if (slot == 0) {
      int n = T.n_window;
      int cnt = axis == 2 ? n + 1 : 2 * n + 1;
      axis_table(x[axis] - 0.5 * T.L, T.delta_k[0], 3, 0, n, cnt, axis == 2 ? q : 1.0, tb.root[axis], part, NP);
    } else {
      int l = slot + 1;
      int node = path[l];
      double c[3];
      int X[3];
      node_center(T, node, c, X);
      int n = T.n_diff;
      int cnt = axis == 2 ? n + 1 : 2 * n + 1;
      axis_table(x[axis] - c[axis], T.delta_k[l], 1, X[axis], n, cnt, axis == 2 ? q : 1.0, tb.lev[l][axis], part, NP);
    }
  }
}

__device__ inline double2 phase_at(double2* const* ax, int k, int d) {
  int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
  return cmul(ax[2][iz], cmul(ax[1][iy], ax[0][ix]));
}

struct Header {
  int i_orig, slot;
  double q;
  double xo[3], xt[3];
  double dr;
  int depth_o, depth_t;
  int path_o[MAXLV], path_t[MAXLV];
};

// resolve the proposal: particle, positions, paths (first warp of the block)
__device__ void resolve(const DevTree& T, int i, const double* disp, Header& h) {
  const int lane = threadIdx.x & 31;
  if (threadIdx.x < 32) {
    if (lane == 0) {
      h.i_orig = i;
      int s = T.orig_slot[i];
      h.slot = s;
      double x, y, z, q;
      if (s < T.n_slots) {
        x = T.sx[s];
        y = T.sy[s];
        z = T.sz[s];
        q = T.sq[s];
      } else {
        int p = s - T.n_slots;
        x = T.px[p];
        y = T.py[p];
        z = T.pz[p];
        q = T.pq[p];
      }
      h.q = q;
      h.xo[0] = x;
      h.xo[1] = y;
      h.xo[2] = z;
      // my_mod wrap and minimum-image distance (src/energy_shift.cpp:30-41)
      const double L = T.L;
      h.xt[0] = wrap_mod(x + disp[0], L);
      h.xt[1] = wrap_mod(y + disp[1], L);
      h.xt[2] = wrap_mod(z + disp[2], L);
      double dr = sqrt(disp[0] * disp[0] + disp[1] * disp[1] + disp[2] * disp[2]);
      for (int mx = -1; mx <= 1; mx++)
        for (int my = -1; my <= 1; my++)
          for (int mz = -1; mz <= 1; mz++) {
            double ax = h.xt[0] - (x + mx * L), ay = h.xt[1] - (y + my * L), az = h.xt[2] - (z + mz * L);
            dr = fmin(dr, sqrt(ax * ax + ay * ay + az * az));
          }
      h.dr = dr;
    }
    __syncwarp();
    int dt = warp_path(T, h.xt[0], h.xt[1], h.xt[2], h.path_t);
    int dO = warp_path(T, h.xo[0], h.xo[1], h.xo[2], h.path_o);
    if (lane == 0) {
      h.depth_t = dt;
      h.depth_o = dO;
    }
  }
  __syncthreads();
}

// q * sum_{j in N(leaf)} q_j res(|x - x_j|; bs_leaf), masked r^2 in (eps, b^2)
// (eval_shift_energy_res_vec + direct_eval, src/energy_shift.cpp:233-302)
__device__ double residual_sum(const DevTree& T, int leaf, const double* x) {
  const int l = T.node_level[leaf];
  const double b = T.boxsize[l];
  const double b2 = b * b;
  const double eps = 2.220446049250313e-16;
  double ci[3];
  int Xi[3];
  node_center(T, leaf, ci, Xi);
  double acc = 0;
  // sources: self (0), colleagues (1..27), coarse (28..35)
  for (int src = threadIdx.x >> 5; src < 36; src += blockDim.x >> 5) {
    int j;
    if (src == 0) j = leaf;
    else if (src <= 27) {
      if (src - 1 == 13) continue;
      j = T.col27[size_t(leaf) * 27 + (src - 1)];
    } else {
      j = T.coarse8[size_t(leaf) * 8 + (src - 28)];
    }
    if (j < 0) continue;
    double cj[3];
    int Xj[3];
    node_center(T, j, cj, Xj);
    const double bj = T.boxsize[T.node_level[j]];
    double off[3];
    for (int d = 0; d < 3; ++d) off[d] = -periodic_shift_d(ci[d], cj[d], T.L, b, bj) * T.L;
    const bool is_leaf = T.node_child0[j] < 0;
    const int sb = T.node_begin[j];
    const int se = is_leaf ? sb + T.leaf_count[j] : T.node_end[j];
    for (int s = sb + (threadIdx.x & 31); s < se; s += 32) {
      double dx = x[0] - (T.sx[s] + off[0]), dy = x[1] - (T.sy[s] + off[1]), dz = x[2] - (T.sz[s] + off[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > eps && r2 < b2) acc += T.sq[s] * poly_res(T, sqrt(r2), b);
    }
    // arrivals parked in the overflow pool that belong to j's subtree
    const int pn = *T.pool_n;
    const int lj = T.node_level[j];
    const uint64_t pj = T.node_prefix[j];
    for (int p = threadIdx.x & 31; p < pn; p += 32) {
      if (T.p_orig[p] < 0) continue;
      int pl = T.p_leaf[p];
      int ll = T.node_level[pl];
      if (ll < lj || (T.node_prefix[pl] >> (3 * (ll - lj))) != pj) continue;
      double dx = x[0] - (T.px[p] + off[0]), dy = x[1] - (T.py[p] + off[1]), dz = x[2] - (T.pz[p] + off[2]);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > eps && r2 < b2) acc += T.pq[p] * poly_res(T, sqrt(r2), b);
    }
  }
  return acc;
}

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
  __syncthreads();
  return s;
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
  double c_level[MAXLV + 2];  // dk_l^3 / (2 pi)^3 * dscale_l
  double* partials;
  unsigned int* counter;
  Proposal* prop;
};

__device__ inline void alloc_tables(double2* sm, const DevTree& T, Tables& tb, int lmax) {
  double2* p = sm;
  for (int a = 0; a < 3; ++a) {
    tb.root[a] = p;
    p += 2 * T.n_window + 1;
  }
  for (int l = 2; l <= lmax; ++l)
    for (int a = 0; a < 3; ++a) {
      tb.lev[l][a] = p;
      p += 2 * T.n_diff + 1;
    }
}

// Grid: blocks [0, G-2) do the plane-wave sums; block G-2 the target
// residual, block G-1 the origin residual. The last block to finish reduces.
__global__ void __launch_bounds__(SH_T) k_shift(DevTree T, ShiftArgs a) {
  extern __shared__ double2 sm2[];
  __shared__ Header h;
  __shared__ double red[32];
  __shared__ bool is_last;
  const int move = a.move;
  resolve(T, a.idx[move], a.disp + 3 * move, h);
  const int G = gridDim.x;
  const int Gpw = G - 2;
  double acc_w = 0, acc_d = 0, res_t = 0, res_o = 0;
  if (blockIdx.x < Gpw) {
    // non-leaf path levels: 2 .. depth-2
    const int lo_max = h.depth_o - 2, lt_max = h.depth_t - 2;
    Tables to, oo;
    const int lmax = max(lo_max, lt_max);
    const int per = 3 * (2 * T.n_window + 1) + (lmax >= 2 ? (lmax - 1) : 0) * 3 * (2 * T.n_diff + 1);
    alloc_tables(sm2, T, oo, lmax);
    alloc_tables(sm2 + per, T, to, lmax);
    build_tables(T, h.xo, h.q, h.path_o, lo_max, oo);
    build_tables(T, h.xt, h.q, h.path_t, lt_max, to);
    __syncthreads();
    const int stride = Gpw * blockDim.x;
    const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
    // window (src/energy_shift.cpp:72-90)
    for (int k = t0; k < T.Hw; k += stride) {
      double2 t = phase_at(to.root, k, T.dw), o = phase_at(oo.root, k, T.dw);
      double2 g = T.out_root[k];
      double ar = t.x - o.x, ai = t.y - o.y, br = g.x - o.x, bi = g.y - o.y;
      acc_w += (ar * br + ai * bi) * T.W[k];
    }
    // difference (src/energy_shift.cpp:92-140)
    const int base = T.level_start[T.pw_lo];
    for (int l = 2; l <= lo_max; ++l) {
      const double2* inc = T.inc + size_t(h.path_o[l] - base) * T.H;
      double s = 0;
      for (int k = t0; k < T.H; k += stride) {
        double2 o = phase_at(oo.lev[l], k, T.dd);
        double2 c = inc[k];
        s += (o.x * c.x - o.y * c.y - (o.x * o.x + o.y * o.y)) * T.D2[k];
      }
      acc_d -= s * a.c_level[l];
    }
    for (int l = 2; l <= lt_max; ++l) {
      const double2* inc = T.inc + size_t(h.path_t[l] - base) * T.H;
      double s = 0;
      for (int k = t0; k < T.H; k += stride) {
        double2 t = phase_at(to.lev[l], k, T.dd);
        double2 c = inc[k];
        s += (t.x * c.x - t.y * c.y) * T.D2[k];
      }
      acc_d += s * a.c_level[l];
    }
  } else if (blockIdx.x == Gpw) {
    res_t = residual_sum(T, h.path_t[h.depth_t - 1], h.xt) * h.q;
  } else {
    res_o = residual_sum(T, h.path_o[h.depth_o - 1], h.xo) * h.q;
  }
  double sw = block_sum(acc_w, red), sd = block_sum(acc_d, red);
  double st = block_sum(res_t, red), so = block_sum(res_o, red);
  if (threadIdx.x == 0) {
    double* pp = a.partials + 4 * size_t(blockIdx.x);
    pp[0] = sw;
    pp[1] = sd;
    pp[2] = st;
    pp[3] = so;
    __threadfence();
    unsigned prev = atomicAdd(a.counter, 1u);
    is_last = (prev == unsigned(G - 1));
  }
  __syncthreads();
  if (is_last && threadIdx.x == 0) {
    __threadfence();
    double w = 0, d = 0, rt = 0, ro = 0;
    for (int b = 0; b < G; ++b) {
      const double* pp = a.partials + 4 * size_t(b);
      w += __ldcg(pp);
      d += __ldcg(pp + 1);
      rt += __ldcg(pp + 2);
      ro += __ldcg(pp + 3);
    }
    double dEw = 2.0 * w * 0.5 * a.c_window;
    double r = h.dr;
    double self = 0;
    if (r != 0) self = poly_res(T, r, T.boxsize[2]) * h.q * h.q;
    double dE = dEw + d + rt - ro - self;
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
    int acc = 0;
    if (a.mode == 1) {
      double u = a.u[move];
      acc = u < exp(-a.beta * dE) ? 1 : 0;
      if (a.acc_out) a.acc_out[move] = acc;
    }
    if (a.dE_out) a.dE_out[move] = dE;
    P->accepted = acc;
    P->valid = 1;
    *a.counter = 0u;
  }
}

// ---------------------------------------------------------------------------
// update_shift (src/tree.cpp:447-597) for one path: sign +1 target, -1 origin
__global__ void __launch_bounds__(SH_T) k_update(DevTree T, int which, double c_unused) {
  extern __shared__ double2 sm2[];
  __shared__ int rnode[MAXLV * 28];
  __shared__ signed char rflag[MAXLV * 28][4];  // is_out, px, py, pz
  __shared__ int rlevel[MAXLV * 28];
  __shared__ int nrecv;
  __shared__ Proposal P;
  if (threadIdx.x == 0) P = *T.prop;
  __syncthreads();
  if (!P.accepted) return;
  const bool tgt = which == 0;
  const double sign = tgt ? 1.0 : -1.0;
  const int depth = tgt ? P.depth_t : P.depth_o;
  const int* path = tgt ? P.path_t : P.path_o;
  const double* x = tgt ? P.xt : P.xo;
  const int lmax = min(depth - 1, T.pw_hi);  // path levels 2..leaf level carrying expansions
  // receivers per level: own out, own inc, non-leaf colleagues' inc
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    if (lane == 0) nrecv = 0;
    __syncwarp();
    for (int l = 2; l <= lmax; ++l) {
      const int node = path[l];
      uint64_t p = T.node_prefix[node];
      int X[3] = {int(compact3(p)), int(compact3(p >> 1)), int(compact3(p >> 2))};
      int j = -1;
      bool ok = false;
      if (lane < 27 && lane != 13) {
        j = T.col27[size_t(node) * 27 + lane];
        ok = j >= 0 && T.node_child0[j] >= 0;
      }
      unsigned m = __ballot_sync(0xffffffffu, ok);
      int base = nrecv;
      if (ok) {
        int pos = base + 2 + __popc(m & ((1u << lane) - 1u));
        rnode[pos] = j;
        rlevel[pos] = l;
        rflag[pos][0] = 0;
        int dv[3] = {lane % 3 - 1, (lane / 3) % 3 - 1, lane / 9 - 1};
        for (int d = 0; d < 3; ++d) {
          // source-centric image flag: periodic_shift(c_source, c_receiver)
          int v = X[d] + dv[d];
          rflag[pos][1 + d] = v < 0 ? 1 : (v >= (1 << l) ? -1 : 0);
        }
      }
      if (lane < 2) {
        rnode[base + lane] = node;
        rlevel[base + lane] = l;
        rflag[base + lane][0] = lane == 0 ? 1 : 0;
        rflag[base + lane][1] = rflag[base + lane][2] = rflag[base + lane][3] = 0;
      }
      __syncwarp();
      if (lane == 0) nrecv = base + 2 + __popc(m);
      __syncwarp();
    }
  }
  __syncthreads();
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    // algorithmic update traffic: one read and one write of 16 B per complex
    unsigned long long b = 32ull * (unsigned long long)nrecv * (unsigned long long)T.H;
    if (tgt) {
      b += 32ull * (unsigned long long)T.Hw;
      atomicAdd(&T.work[0], 1ull);
    }
    atomicAdd(&T.work[1], b);
  }
  // tables: this path's levels, plus both roots (window) for the target pass
  Tables tb, tb_o;
  const int per = 3 * (2 * T.n_window + 1) + (lmax >= 2 ? (lmax - 1) : 0) * 3 * (2 * T.n_diff + 1);
  alloc_tables(sm2, T, tb, lmax);
  alloc_tables(sm2 + per, T, tb_o, 0);
  build_tables(T, x, P.q, path, lmax, tb);
  if (tgt) build_tables(T, P.xo, P.q, P.path_o, 0, tb_o);
  __syncthreads();
  const int stride = gridDim.x * blockDim.x;
  const int t0 = blockIdx.x * blockDim.x + threadIdx.x;
  if (tgt) {
    // root: out += t; out -= o (src/tree.cpp:479-480)
    for (int k = t0; k < T.Hw; k += stride) {
      double2 t = phase_at(tb.root, k, T.dw), o = phase_at(tb_o.root, k, T.dw);
      double2 g = T.out_root[k];
      g = cadd(g, t);
      g = csub(g, o);
      T.out_root[k] = g;
    }
  }
  const int base = T.level_start[T.pw_lo];
  const int n = T.n_diff, d = T.dd;
  const long total = long(nrecv) * T.H;
  for (long e = t0; e < total; e += stride) {
    const int r = int(e / T.H), k = int(e % T.H);
    const int l = rlevel[r];
    double2 p = phase_at(tb.lev[l], k, d);
    const int is_out = rflag[r][0];
    const size_t off = size_t(rnode[r] - base) * T.H + k;
    if (is_out) {
      double2 v = T.out[off];
      T.out[off] = make_double2(v.x + sign * p.x, v.y + sign * p.y);
    } else {
      const int px = rflag[r][1], py = rflag[r][2], pz = rflag[r][3];
      if (px | py | pz) {
        int ix = k % d, iy = (k / d) % d, iz = k / (d * d);
        int sgn = ((ix - n) * px + (iy - n) * py + (iz - n) * pz) * ((l & 1) ? 2 : 1);
        p = cmul(p, root6(-2 * (sgn % 3)));
      }
      double2 v = T.inc[off];
      T.inc[off] = make_double2(v.x + sign * p.x, v.y - sign * p.y);
    }
  }
}

// particle membership and position (exact on every level)
__global__ void k_commit(DevTree T) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const Proposal P = *T.prop;
  if (!P.accepted) return;
  const int leafA = P.path_o[P.depth_o - 1];
  const int leafB = P.path_t[P.depth_t - 1];
  const int i = P.i_orig;
  int s = P.slot;
  if (leafA == leafB) {
    if (s < T.n_slots) {
      T.sx[s] = P.xt[0];
      T.sy[s] = P.xt[1];
      T.sz[s] = P.xt[2];
    } else {
      int p = s - T.n_slots;
      T.px[p] = P.xt[0];
      T.py[p] = P.xt[1];
      T.pz[p] = P.xt[2];
    }
    return;
  }
  // remove from the origin leaf (swap with its last particle) or the pool
  if (s < T.n_slots) {
    int cA = T.leaf_count[leafA];
    int last = T.node_begin[leafA] + cA - 1;
    if (s != last) {
      int ol = T.s_orig[last];
      T.sx[s] = T.sx[last];
      T.sy[s] = T.sy[last];
      T.sz[s] = T.sz[last];
      T.sq[s] = T.sq[last];
      T.s_orig[s] = ol;
      T.orig_slot[ol] = s;
    }
    double c[3];
    int X[3];
    node_center(T, leafA, c, X);
    T.sx[last] = c[0];
    T.sy[last] = c[1];
    T.sz[last] = c[2];
    T.sq[last] = 0.0;
    T.s_orig[last] = -1;
    T.leaf_count[leafA] = cA - 1;
  } else {
    int p = s - T.n_slots;
    T.p_orig[p] = -1;
    T.pq[p] = 0.0;
  }
  // insert into the target leaf, or park in the pool when it is full
  int cB = T.leaf_count[leafB];
  int slot = T.node_begin[leafB] + cB;
  if (slot < T.node_end[leafB]) {
    T.sx[slot] = P.xt[0];
    T.sy[slot] = P.xt[1];
    T.sz[slot] = P.xt[2];
    T.sq[slot] = P.q;
    T.s_orig[slot] = i;
    T.orig_slot[i] = slot;
    T.leaf_count[leafB] = cB + 1;
  } else {
    int p = *T.pool_n;
    if (p < T.pool_cap) {
      T.px[p] = P.xt[0];
      T.py[p] = P.xt[1];
      T.pz[p] = P.xt[2];
      T.pq[p] = P.q;
      T.p_orig[p] = i;
      T.p_leaf[p] = leafB;
      T.orig_slot[i] = T.n_slots + p;
      *T.pool_n = p + 1;
    } else {
      *T.err = 1;  // pool exhausted: the host repacks and reports
    }
  }
  for (int l = 0; l < P.depth_o; ++l) T.node_count[P.path_o[l]] -= 1;
  for (int l = 0; l < P.depth_t; ++l) T.node_count[P.path_t[l]] += 1;
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
  for (int l = 0; l < MAX_LEVELS + 2; ++l) a.c_level[l] = std::pow(D.delta_k[l], 3) / std::pow(2 * pi, 3) * D.dscale[l];
  a.partials = D.partials;
  a.counter = D.counter;
  a.prop = D.prop;
  size_t smem = tables_smem(D, D.max_depth, 2);
  if (shift_grid_ == 0) {
    int dev = 0, sms = 148;
    PDMK_CUDA(cudaGetDevice(&dev));
    PDMK_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    shift_grid_ = 2 + sms;
    static size_t smem_set = 0;  // the attribute is per function, shared by all trees
    if (smem > smem_set) {
      PDMK_CUDA(cudaFuncSetAttribute(k_shift, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      PDMK_CUDA(cudaFuncSetAttribute(k_update, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
      smem_set = smem;
    }
  }
  time_begin(0);
  k_shift<<<unsigned(shift_grid_), SH_T, smem, st_>>>(D, a);
  PDMK_LAUNCH_CHECK();
  time_end(0);
}

void DmkTree::launch_update() {
  DevTree& D = dev_;
  size_t smem = tables_smem(D, D.max_depth, 2);
  if (update_grid_ == 0) update_grid_ = 2 * 148;
  time_begin(1);
  k_update<<<unsigned(update_grid_), SH_T, smem, st_>>>(D, 0, 0.0);
  PDMK_LAUNCH_CHECK();
  k_update<<<unsigned(update_grid_), SH_T, smem, st_>>>(D, 1, 0.0);
  PDMK_LAUNCH_CHECK();
  time_end(1);
}

void DmkTree::launch_commit() {
  time_begin(2);
  k_commit<<<1, 32, 0, st_>>>(dev_);
  PDMK_LAUNCH_CHECK();
  time_end(2);
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
  if (!timing_) return;
  ev_cur_[cls] = take_event();
  PDMK_CUDA(cudaEventRecord(ev_cur_[cls], st_));
}

void DmkTree::time_end(int cls) {
  if (!timing_ || !ev_cur_[cls]) return;
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
  unsigned long long w[2];
  PDMK_CUDA(cudaMemcpyAsync(w, dev_.work, sizeof(w), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  out[0] = double(w[0]);
  out[1] = double(w[1]);
}

void DmkTree::reset_work() { PDMK_CUDA(cudaMemsetAsync(dev_.work, 0, 2 * sizeof(unsigned long long), st_)); }

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
  launch_commit();
  PDMK_CUDA(cudaStreamSynchronize(st_));
  last_valid_ = false;
  diff_cached_ = false;
}

void DmkTree::mc_run_device(int n_moves, const int* d_idx, const double* d_disp, const double* d_u, double beta,
                            double* d_dE, int* d_acc) {
  for (int m = 0; m < n_moves; ++m) {
    launch_shift(d_idx, d_disp, d_u, beta, m, 1, d_dE, d_acc);
    launch_update();
    launch_commit();
  }
  last_valid_ = false;
  diff_cached_ = false;
}

void DmkTree::shift_batch_device(int m, const int* d_idx, const double* d_disp, double* d_dE) {
  for (int c = 0; c < m; ++c) launch_shift(d_idx, d_disp, nullptr, 0.0, c, 0, d_dE, nullptr);
  last_valid_ = false;
}

}  // namespace pdmk
