// ORACLE — test infrastructure only (see oracle_core.hpp). A plain CPU
// restatement of the reference's DMK energy path. Every routine names the
// reference file:line it follows. The tree is built from a documented
// restatement of the SCTL PtTree semantics the reference relies on (the SCTL
// sources are not vendored with the reference):
//   * particles are binned by a 21-bit-per-axis Morton key of r/L and stably
//     sorted by it;
//   * a node is refined when it holds more than n_per_leaf particles (and is
//     above level 10), every node above level 2 is refined (the reference
//     throws or drops leaves above level 2), and the tree is then closed under
//     periodic 2:1 balance over all 26 neighbours;
//   * nodes are numbered level by level, in Morton order within a level.
#include "oracle_core.hpp"

#include <omp.h>

#include <algorithm>
#include <array>
#include <limits>
#include <cmath>
#include <complex>
#include <cstring>
#include <map>
#include <numeric>
#include <random>
#include <set>
#include <vector>

namespace {

using cd = std::complex<double>;
constexpr int KEY_BITS = 21;   // Morton bits per axis
constexpr int MAX_LEVEL = 10;  // deepest level a node may be refined to

inline uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffff;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}
inline uint32_t compact3(uint64_t x) {
  x &= 0x1249249249249249ULL;
  x = (x ^ (x >> 2)) & 0x10c30c30c30c30c3ULL;
  x = (x ^ (x >> 4)) & 0x100f00f00f00f00fULL;
  x = (x ^ (x >> 8)) & 0x1f0000ff0000ffULL;
  x = (x ^ (x >> 16)) & 0x1f00000000ffffULL;
  x = (x ^ (x >> 32)) & 0x1fffffULL;
  return static_cast<uint32_t>(x);
}
inline uint64_t morton(uint32_t ix, uint32_t iy, uint32_t iz) {
  return spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
}
inline uint32_t grid_coord(double x, double L) {
  double u = x / L;
  double s = std::floor(u * double(1u << KEY_BITS));
  if (s < 0) s = 0;
  if (s > double((1u << KEY_BITS) - 1)) s = double((1u << KEY_BITS) - 1);
  return static_cast<uint32_t>(s);
}

// my_mod (include/utils.hpp:96-105)
inline double my_mod(double x, double L) {
  while (x < 0) x += L;
  while (x >= L) x -= L;
  return x;
}
// periodic_shift (include/utils.hpp:58-67)
inline int periodic_shift(double xi, double xj, double L, double bi, double bj) {
  if (xi < bi && xj > (L - bj)) return 1;
  if (xi > (L - bi) && xj < bj) return -1;
  return 0;
}
inline double sq(double x) { return x * x; }

struct Node {
  int level;
  uint64_t prefix;
  long parent;
  long child0;  // first of 8 consecutive children, -1 for a leaf
  bool leaf;
  double center[3];
};

struct Tree {
  double L;
  int n_per_leaf, digits;
  long n;
  // PSWF constants (oracle/pswf.py)
  std::vector<double> leg, poly;
  double c, lambda, C0, diff0, psi0_0;
  int n_window, n_diff;
  int max_depth;
  std::vector<double> boxsize, sigmas, delta_k;
  std::vector<Node> nodes;
  std::vector<std::vector<long>> level_indices;
  std::map<std::pair<int, uint64_t>, long> index;
  std::vector<double> r;  // sorted, xyz interleaved
  std::vector<double> q;  // sorted
  std::vector<long> orig_of_sorted, sorted_of_orig;
  std::vector<std::vector<long>> node_particles;
  std::vector<std::array<int, 27>> nbr;
  std::vector<std::vector<long>> colleague, coarse;
  double Q;
  std::vector<double> W;
  std::vector<std::vector<double>> D;  // indexed by level
  std::vector<std::vector<cd>> out, inc;
  // proposal scratch (the reference keeps these on the tree, include/tree.hpp:68-72)
  std::vector<long> path_o, path_t;
  std::vector<std::vector<cd>> pw_o, pw_t;

  double psi0(double x) const {
    // Legendre series on [-1,1]; zero outside, as the reference's prol0eva
    // does for c below its threshold 45 (src/pswf.cpp:976-982)
    if (std::fabs(x) > 1) return 0.0;
    double p0 = 1.0, p1 = x, s = leg[0];
    if (leg.size() > 1) s += leg[1] * x;
    for (size_t k = 1; k + 1 < leg.size(); ++k) {
      double p2 = ((2.0 * k + 1.0) * x * p1 - double(k) * p0) / double(k + 1);
      s += leg[k + 1] * p2;
      p0 = p1;
      p1 = p2;
    }
    return s;
  }
  // PolyFun::eval (include/pswf.hpp:70-78)
  double poly_eval(double x) const {
    double xs = (x - 0.5) * 2.0;
    if (std::fabs(xs) >= 1.0) return 0.0;
    double v = 0;
    for (double cf : poly) v = v * xs + cf;
    return v;
  }
  // residual_kernel (include/kernels.hpp:50-58)
  double res_kernel(double rr, double cutoff) const {
    if (rr == 0) return 0;
    return poly_eval(rr / cutoff) / rr;
  }
  int dims_window() const { return (2 * n_window + 1) * (2 * n_window + 1) * (n_window + 1); }
  int dims_diff() const { return (2 * n_diff + 1) * (2 * n_diff + 1) * (n_diff + 1); }
};

// ---------------------------------------------------------------------------
// tree build (src/tree.cpp:267-444 with the SCTL semantics above)
struct BuildNode {
  bool refined = false;
};

void build_tree(Tree& t, const double* r_in, const double* q_in) {
  const long n = t.n;
  std::vector<uint64_t> key(n);
  for (long i = 0; i < n; ++i)
    key[i] = morton(grid_coord(r_in[3 * i], t.L), grid_coord(r_in[3 * i + 1], t.L), grid_coord(r_in[3 * i + 2], t.L));
  std::vector<long> ord(n);
  std::iota(ord.begin(), ord.end(), 0);
  std::stable_sort(ord.begin(), ord.end(), [&](long a, long b) { return key[a] < key[b]; });
  std::vector<uint64_t> skey(n);
  t.r.resize(3 * n);
  t.q.resize(n);
  t.orig_of_sorted = ord;
  t.sorted_of_orig.assign(n, 0);
  for (long s = 0; s < n; ++s) {
    long i = ord[s];
    skey[s] = key[i];
    t.r[3 * s] = r_in[3 * i];
    t.r[3 * s + 1] = r_in[3 * i + 1];
    t.r[3 * s + 2] = r_in[3 * i + 2];
    t.q[s] = q_in[i];
    t.sorted_of_orig[i] = s;
  }
  auto count_of = [&](int level, uint64_t prefix) -> long {
    int sh = 3 * (KEY_BITS - level);
    uint64_t lo = prefix << sh, hi = (prefix + 1) << sh;
    auto a = std::lower_bound(skey.begin(), skey.end(), lo);
    auto b = (level == 0) ? skey.end() : std::lower_bound(skey.begin(), skey.end(), hi);
    return long(b - a);
  };
  // count-driven refinement, top down
  std::map<std::pair<int, uint64_t>, BuildNode> bn;
  std::vector<std::pair<int, uint64_t>> frontier{{0, 0}};
  bn[{0, 0}] = BuildNode();
  while (!frontier.empty()) {
    std::vector<std::pair<int, uint64_t>> next;
    for (auto& nd : frontier) {
      int lv = nd.first;
      long cnt = count_of(lv, nd.second);
      bool refine = (lv < 2) || (cnt > t.n_per_leaf && lv < MAX_LEVEL);
      if (refine) {
        bn[nd].refined = true;
        for (int ch = 0; ch < 8; ++ch) {
          std::pair<int, uint64_t> c{lv + 1, (nd.second << 3) | uint64_t(ch)};
          bn[c] = BuildNode();
          next.push_back(c);
        }
      }
    }
    frontier.swap(next);
  }
  // periodic 2:1 balance over 26 neighbours, to a fixed point
  auto ensure_refined = [&](int level, uint64_t prefix) -> bool {
    bool changed = false;
    for (int lv = 0; lv <= level; ++lv) {
      uint64_t p = prefix >> (3 * (level - lv));
      auto it = bn.find({lv, p});
      // existence of (lv,p) is guaranteed by refining its ancestors first
      if (!it->second.refined) {
        it->second.refined = true;
        changed = true;
        for (int ch = 0; ch < 8; ++ch) bn[{lv + 1, (p << 3) | uint64_t(ch)}] = BuildNode();
      }
    }
    return changed;
  };
  bool changed = true;
  while (changed) {
    changed = false;
    std::vector<std::pair<int, uint64_t>> all;
    all.reserve(bn.size());
    for (auto& kv : bn) all.push_back(kv.first);
    for (auto& nd : all) {
      int m = nd.first;
      if (m < 2) continue;
      uint32_t ix = compact3(nd.second), iy = compact3(nd.second >> 1), iz = compact3(nd.second >> 2);
      uint32_t mask = (1u << m) - 1;
      for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
          for (int dx = -1; dx <= 1; ++dx) {
            if (!dx && !dy && !dz) continue;
            uint32_t nx = (ix + dx) & mask, ny = (iy + dy) & mask, nz = (iz + dz) & mask;
            uint64_t anc = morton(nx >> 2, ny >> 2, nz >> 2);
            changed |= ensure_refined(m - 2, anc);
          }
    }
  }
  // enumerate: level-major, Morton order within a level (std::map order)
  int maxlev = 0;
  for (auto& kv : bn) maxlev = std::max(maxlev, kv.first.first);
  t.max_depth = maxlev + 1;
  t.level_indices.assign(t.max_depth, {});
  for (auto& kv : bn) {
    Node nd;
    nd.level = kv.first.first;
    nd.prefix = kv.first.second;
    nd.leaf = !kv.second.refined;
    nd.parent = -1;
    nd.child0 = -1;
    long id = long(t.nodes.size());
    t.nodes.push_back(nd);
    t.index[kv.first] = id;
    t.level_indices[nd.level].push_back(id);
  }
  // map order is (level, prefix): already level-major
  for (auto& nd : t.nodes) {
    if (nd.level > 0) nd.parent = t.index.at({nd.level - 1, nd.prefix >> 3});
    if (!nd.leaf) nd.child0 = t.index.at({nd.level + 1, nd.prefix << 3});
  }
  // box sizes and centres (src/tree.cpp:364-381)
  t.boxsize.assign(t.max_depth + 1, 0);
  t.boxsize[0] = t.L;
  for (int i = 1; i < t.max_depth + 1; ++i) t.boxsize[i] = 0.5 * t.boxsize[i - 1];
  for (auto& nd : t.nodes) {
    double scale = std::ldexp(1.0, -nd.level);
    uint32_t c3[3] = {compact3(nd.prefix), compact3(nd.prefix >> 1), compact3(nd.prefix >> 2)};
    for (int d = 0; d < 3; ++d) nd.center[d] = t.L * (double(c3[d]) * scale + 0.5 * scale);
  }
  // membership: the whole subtree, in sorted order (src/tree.cpp:117-133)
  t.node_particles.assign(t.nodes.size(), {});
  for (size_t id = 0; id < t.nodes.size(); ++id) {
    auto& nd = t.nodes[id];
    int sh = 3 * (KEY_BITS - nd.level);
    uint64_t lo = nd.prefix << sh, hi = (nd.prefix + 1) << sh;
    long a = long(std::lower_bound(skey.begin(), skey.end(), lo) - skey.begin());
    long b = nd.level == 0 ? n : long(std::lower_bound(skey.begin(), skey.end(), hi) - skey.begin());
    for (long s = a; s < b; ++s) t.node_particles[id].push_back(s);
  }
  t.Q = 0;
  for (long i = 0; i < n; ++i) t.Q += q_in[i] * q_in[i];  // src/tree.cpp:306-309
}

// node_shift (src/tree.cpp:169-201)
void node_shift(const Tree& t, long i, long j, double* s) {
  const Node& a = t.nodes[i];
  const Node& b = t.nodes[j];
  for (int d = 0; d < 3; ++d) {
    int p = periodic_shift(a.center[d], b.center[d], t.L, t.boxsize[a.level], t.boxsize[b.level]);
    s[d] = b.center[d] - (a.center[d] + p * t.L);
  }
}

// collect_neighbors (src/tree.cpp:136-165); nbr[27] ordered dx fastest
void build_neighbors(Tree& t) {
  const long nn = long(t.nodes.size());
  t.nbr.assign(nn, {});
  t.colleague.assign(nn, {});
  t.coarse.assign(nn, {});
  for (long id = 0; id < nn; ++id) {
    auto& nd = t.nodes[id];
    t.nbr[id].fill(-1);
    if (nd.level < 1) continue;
    uint32_t ix = compact3(nd.prefix), iy = compact3(nd.prefix >> 1), iz = compact3(nd.prefix >> 2);
    uint32_t mask = (1u << nd.level) - 1;
    for (int dz = -1; dz <= 1; ++dz)
      for (int dy = -1; dy <= 1; ++dy)
        for (int dx = -1; dx <= 1; ++dx) {
          uint64_t p = morton((ix + dx) & mask, (iy + dy) & mask, (iz + dz) & mask);
          auto it = t.index.find({nd.level, p});
          t.nbr[id][(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)] = it == t.index.end() ? -1 : int(it->second);
        }
  }
  for (int l = 2; l < t.max_depth; ++l)
    for (long id : t.level_indices[l]) {
      for (int k = 0; k < 27; ++k) {
        long j = t.nbr[id][k];
        if (j != -1 && j != id) t.colleague[id].push_back(j);
      }
      if (t.colleague[id].size() < 26) {
        long par = t.nodes[id].parent;
        double s_i2p[3];
        node_shift(t, par, id, s_i2p);
        for (int k = 0; k < 27; ++k) {
          long j = t.nbr[par][k];
          if (j != -1 && j != par && t.nodes[j].leaf) {
            double s_n2p[3];
            node_shift(t, par, j, s_n2p);
            if (s_i2p[0] * s_n2p[0] >= 0 && s_i2p[1] * s_n2p[1] >= 0 && s_i2p[2] * s_n2p[2] >= 0)
              t.coarse[id].push_back(j);
          }
        }
      }
    }
}

// form_wavenumbers (src/tree.cpp:17-81) and interaction matrices
// (src/tree.cpp:84-100, include/kernels.hpp:15-114)
void build_setup(Tree& t) {
  t.psi0_0 = t.psi0(0.0);
  t.sigmas.assign(t.max_depth + 1, 0);
  t.sigmas[0] = t.L / t.c;
  for (int i = 1; i < t.max_depth + 1; ++i) t.sigmas[i] = 0.5 * t.sigmas[i - 1];
  t.delta_k.assign(t.max_depth + 1, 0);
  t.delta_k[0] = t.delta_k[1] = 2 * M_PI / t.L;
  for (int i = 2; i < t.max_depth + 1; ++i) t.delta_k[i] = (2.0 * M_PI / 3.0) / t.boxsize[i];
  auto fourier = [&](double x) { return 2 * M_PI * t.lambda * t.psi0(x) / t.C0; };
  {
    int nk = t.n_window, d = 2 * nk + 1;
    double dk = t.delta_k[1], sigma = t.sigmas[2];
    t.W.assign(d * d * (nk + 1), 0);
    for (int k = 0; k < nk + 1; ++k)
      for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
          double kx = (i - nk) * dk, ky = (j - nk) * dk, kz = (k - nk) * dk;
          double k2 = kx * kx + ky * ky + kz * kz;
          double val = 0;
          if (k2 != 0) val = fourier(std::sqrt(k2) * sigma) / k2;
          t.W[k * d * d + j * d + i] = (k == nk) ? val : 2 * val;
        }
  }
  t.D.assign(t.max_depth + 1, {});
  for (int l = 2; l < t.max_depth - 1; ++l) {
    int nk = t.n_diff, d = 2 * nk + 1;
    double dk = t.delta_k[l], sl = t.sigmas[l], slp1 = t.sigmas[l + 1];
    auto& D = t.D[l];
    D.assign(d * d * (nk + 1), 0);
    for (int k = 0; k < nk + 1; ++k)
      for (int j = 0; j < d; ++j)
        for (int i = 0; i < d; ++i) {
          double kx = (i - nk) * dk, ky = (j - nk) * dk, kz = (k - nk) * dk;
          double k2 = kx * kx + ky * ky + kz * kz;
          double val;
          if (k2 == 0) {
            val = t.diff0 * (slp1 * slp1 - sl * sl);
          } else {
            double kk = std::sqrt(k2);
            val = (fourier(kk * slp1) - fourier(kk * sl)) / k2;
          }
          D[k * d * d + j * d + i] = (k == nk) ? val : 2 * val;
        }
  }
  // expansion storage (src/tree.cpp:414-443)
  t.out.assign(t.nodes.size(), {});
  t.inc.assign(t.nodes.size(), {});
  int dw = 2 * t.n_window + 1;
  t.out[0].assign(size_t(dw) * dw * dw, cd(0));
  t.inc[0].assign(size_t(dw) * dw * dw, cd(0));
  int dd = 2 * t.n_diff + 1;
  for (int l = 2; l < t.max_depth - 1; ++l)
    for (long id : t.level_indices[l]) {
      t.out[id].assign(size_t(dd) * dd * dd, cd(0));
      t.inc[id].assign(size_t(dd) * dd * dd, cd(0));
    }
  t.pw_o.assign(t.max_depth, {});
  t.pw_t.assign(t.max_depth, {});
  t.pw_o[0].assign(size_t(dw) * dw * (t.n_window + 1), cd(0));
  t.pw_t[0] = t.pw_o[0];
  for (int l = 2; l < t.max_depth - 1; ++l) {
    t.pw_o[l].assign(size_t(dd) * dd * (t.n_diff + 1), cd(0));
    t.pw_t[l] = t.pw_o[l];
  }
}

// nudft3d1_halfplane (include/nudft.hpp:66-123), accumulating into f
void nudft_halfplane(long M, const double* x, const double* y, const double* z, const double* c, int N, cd* f) {
  const int nh = (N + 1) / 2 + (N % 2 == 0);
  std::vector<cd> xc(N), yc(N), zc(nh);
  const double kmin = -double(N / 2);
  for (long i = 0; i < M; ++i) {
    cd ex = std::exp(cd(0, -x[i])), ey = std::exp(cd(0, -y[i])), ez = std::exp(cd(0, -z[i]));
    xc[0] = std::exp(cd(0, -x[i] * kmin)) * cd(c[i], 0);
    for (int l = 1; l < N; ++l) xc[l] = xc[l - 1] * ex;
    yc[0] = std::exp(cd(0, -y[i] * kmin));
    for (int m = 1; m < N; ++m) yc[m] = yc[m - 1] * ey;
    zc[0] = std::exp(cd(0, -z[i] * kmin));
    for (int k = 1; k < nh; ++k) zc[k] = zc[k - 1] * ez;
    for (int k = 0; k < nh; ++k)
      for (int m = 0; m < N; ++m) {
        cd zy = zc[k] * yc[m];
        cd* fp = f + (size_t(k) * N + m) * N;
        for (int l = 0; l < N; ++l) fp[l] += zy * xc[l];
      }
  }
}

// nudft3d1_single_halfplane (include/nudft.hpp:125-167)
void nudft_single(double x, double y, double z, double q, int N, cd* f) {
  const int nh = (N % 2 == 0) ? (N / 2 + 1) : ((N + 1) / 2);
  std::vector<cd> xc(N), yc(N), zc(nh);
  const double kmin = -double(N / 2);
  cd ex = std::exp(cd(0, -x)), ey = std::exp(cd(0, -y)), ez = std::exp(cd(0, -z));
  xc[0] = std::exp(cd(0, -x * kmin)) * cd(q, 0);
  for (int l = 1; l < N; ++l) xc[l] = xc[l - 1] * ex;
  yc[0] = std::exp(cd(0, -y * kmin));
  for (int m = 1; m < N; ++m) yc[m] = yc[m - 1] * ey;
  zc[0] = std::exp(cd(0, -z * kmin));
  for (int k = 1; k < nh; ++k) zc[k] = zc[k - 1] * ez;
  for (int k = 0; k < nh; ++k)
    for (int m = 0; m < N; ++m) {
      cd zy = zc[k] * yc[m];
      cd* fp = f + (size_t(k) * N + m) * N;
      for (int l = 0; l < N; ++l) fp[l] = zy * xc[l];
    }
}

// the incoming-shift phase exp(-i k.p L) of ShiftMatrix (include/shiftmat.hpp:16-38)
inline cd shift_phase(int ix, int iy, int iz, int n, double dk, double L, int px, int py, int pz) {
  double kx = (ix - n) * dk * px, ky = (iy - n) * dk * py, kz = (iz - n) * dk * pz;
  return std::exp(-cd(0, kx * L + ky * L + kz * L));
}

void gather_xyzq(const Tree& t, const std::vector<long>& idx, double dk, std::vector<double>& x,
                 std::vector<double>& y, std::vector<double>& z, std::vector<double>& c) {
  size_t m = idx.size();
  x.resize(m);
  y.resize(m);
  z.resize(m);
  c.resize(m);
  for (size_t k = 0; k < m; ++k) {
    long s = idx[k];
    x[k] = t.r[3 * s] * dk;
    y[k] = t.r[3 * s + 1] * dk;
    z[k] = t.r[3 * s + 2] * dk;
    c[k] = t.q[s];
  }
}

// outgoing_pw_root + outgoing_pw_direct (src/planewave.cpp:24-84); the root
// uses the same half-plane direct NUDFT over all particles in place of finufft
void form_outgoing(Tree& t, int nthreads) {
  const int dw = 2 * t.n_window + 1;
  const int hw = dw * dw * (t.n_window + 1);
  std::fill(t.out[0].begin(), t.out[0].end(), cd(0));
  {
    std::vector<std::vector<cd>> part(nthreads, std::vector<cd>(hw, cd(0)));
    const long n = t.n;
#pragma omp parallel num_threads(nthreads)
    {
      int tid = omp_get_thread_num();
      long b = n * tid / nthreads, e = n * (tid + 1) / nthreads;
      std::vector<long> idx;
      for (long s = b; s < e; ++s) idx.push_back(s);
      std::vector<double> x, y, z, c;
      gather_xyzq(t, idx, t.delta_k[0], x, y, z, c);
      nudft_halfplane(long(idx.size()), x.data(), y.data(), z.data(), c.data(), dw, part[tid].data());
    }
    for (int th = 0; th < nthreads; ++th)
      for (int k = 0; k < hw; ++k) t.out[0][k] += part[th][k];
  }
  const int dd = 2 * t.n_diff + 1;
  std::vector<long> work;
  for (int l = 2; l < t.max_depth - 1; ++l)
    for (long id : t.level_indices[l]) work.push_back(id);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long w = 0; w < long(work.size()); ++w) {
    long id = work[w];
    std::fill(t.out[id].begin(), t.out[id].end(), cd(0));
    if (t.node_particles[id].empty()) continue;
    std::vector<double> x, y, z, c;
    gather_xyzq(t, t.node_particles[id], t.delta_k[t.nodes[id].level], x, y, z, c);
    nudft_halfplane(long(x.size()), x.data(), y.data(), z.data(), c.data(), dd, t.out[id].data());
  }
}

// form_incoming_pw (src/planewave.cpp:99-155)
void form_incoming(Tree& t, int nthreads) {
  const int n = t.n_diff, d = 2 * n + 1;
  const int dims = d * d * (n + 1);
  std::vector<long> work;
  for (int l = 2; l < t.max_depth - 1; ++l)
    for (long id : t.level_indices[l])
      if (!t.nodes[id].leaf) work.push_back(id);
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (long w = 0; w < long(work.size()); ++w) {
    long i = work[w];
    const Node& ni = t.nodes[i];
    int l = ni.level;
    double bs = t.boxsize[l], dk = t.delta_k[l];
    auto& inc = t.inc[i];
    if (!t.node_particles[i].empty()) {
      for (int k = 0; k < dims; ++k) inc[k] = std::conj(t.out[i][k]);
    } else {
      std::fill(inc.begin(), inc.begin() + dims, cd(0));
    }
    for (long j : t.colleague[i]) {
      if (t.node_particles[j].empty()) continue;
      const Node& nj = t.nodes[j];
      int px = periodic_shift(nj.center[0], ni.center[0], t.L, bs, bs);
      int py = periodic_shift(nj.center[1], ni.center[1], t.L, bs, bs);
      int pz = periodic_shift(nj.center[2], ni.center[2], t.L, bs, bs);
      const auto& oj = t.out[j];
      if (!px && !py && !pz) {
        for (int k = 0; k < dims; ++k) inc[k] += std::conj(oj[k]);
      } else {
        for (int iz = 0; iz <= n; ++iz)
          for (int iy = 0; iy < d; ++iy)
            for (int ix = 0; ix < d; ++ix) {
              int k = (iz * d + iy) * d + ix;
              inc[k] += std::conj(oj[k] * shift_phase(ix, iy, iz, n, dk, t.L, px, py, pz));
            }
      }
    }
  }
}

// eval_energy_window (src/energy.cpp:21-39)
double energy_window(const Tree& t) {
  const int dims = t.dims_window();
  double e = 0;
  for (int k = 0; k < dims; ++k) e += std::norm(t.out[0][k]) * t.W[k];
  e *= 1 / (2 * std::pow(2 * M_PI, 3)) * std::pow(t.delta_k[0], 3);
  double rc = t.boxsize[2];
  e -= t.Q * t.psi0_0 / (2 * rc * t.C0);
  return e;
}

// eval_energy_diff (src/energy.cpp:42-79)
double energy_diff(const Tree& t, int nthreads) {
  const int dims = t.dims_diff();
  double e = 0;
  for (int l = 2; l < t.max_depth - 1; ++l) {
    const auto& D = t.D[l];
    double Cl = 1 / (2 * std::pow(2 * M_PI, 3)) * std::pow(t.delta_k[l], 3);
    double Sl = t.psi0_0 * (1 / (2 * t.boxsize[l + 1] * t.C0) - 1 / (2 * t.boxsize[l] * t.C0));
    const auto& lv = t.level_indices[l];
#pragma omp parallel for reduction(+ : e) schedule(dynamic, 4) num_threads(nthreads)
    for (long w = 0; w < long(lv.size()); ++w) {
      long id = lv[w];
      if (t.nodes[id].leaf || t.node_particles[id].empty()) continue;
      double tri = 0;
      for (int k = 0; k < dims; ++k) {
        const cd& a = t.out[id][k];
        const cd& b = t.inc[id][k];
        tri += (a.real() * b.real() - a.imag() * b.imag()) * D[k];
      }
      double Qi = 0;
      for (long s : t.node_particles[id]) Qi += t.q[s] * t.q[s];
      e += Cl * tri - Qi * Sl;
    }
  }
  return e;
}

// eval_energy_res / _res_i / _res_ij (src/energy.cpp:82-173)
double energy_res(const Tree& t, int nthreads) {
  std::vector<long> leaves;
  for (int l = 2; l < t.max_depth; ++l)
    for (long id : t.level_indices[l])
      if (t.nodes[id].leaf && !t.node_particles[id].empty()) leaves.push_back(id);
  double e = 0;
#pragma omp parallel for reduction(+ : e) schedule(dynamic, 8) num_threads(nthreads)
  for (long w = 0; w < long(leaves.size()); ++w) {
    long i = leaves[w];
    const Node& ni = t.nodes[i];
    double b = t.boxsize[ni.level];
    const auto& P = t.node_particles[i];
    double el = 0;
    for (size_t a = 0; a + 1 < P.size(); ++a)
      for (size_t c = a + 1; c < P.size(); ++c) {
        long s = P[a], u = P[c];
        double rr = std::sqrt(sq(t.r[3 * s] - t.r[3 * u]) + sq(t.r[3 * s + 1] - t.r[3 * u + 1]) +
                              sq(t.r[3 * s + 2] - t.r[3 * u + 2]));
        if (rr <= b) el += t.q[s] * t.q[u] * t.res_kernel(rr, b);
      }
    auto pair_sum = [&](long j) {
      double sh[3];
      node_shift(t, i, j, sh);
      const Node& nj = t.nodes[j];
      double acc = 0;
      for (long s : P) {
        double xi = t.r[3 * s] - ni.center[0] - sh[0];
        double yi = t.r[3 * s + 1] - ni.center[1] - sh[1];
        double zi = t.r[3 * s + 2] - ni.center[2] - sh[2];
        for (long u : t.node_particles[j]) {
          double xj = t.r[3 * u] - nj.center[0], yj = t.r[3 * u + 1] - nj.center[1], zj = t.r[3 * u + 2] - nj.center[2];
          double rr = std::sqrt(sq(xi - xj) + sq(yi - yj) + sq(zi - zj));
          if (rr <= b) acc += t.q[s] * t.q[u] * t.res_kernel(rr, b) / 2;
        }
      }
      return acc;
    };
    for (long j : t.coarse[i])
      if (!t.node_particles[j].empty()) el += pair_sum(j);
    for (long j : t.colleague[i])
      if (!t.node_particles[j].empty()) el += pair_sum(j);
    e += el;
  }
  return e;
}

// leaf path by Morton descent (the reference's locate_particle,
// src/tree.cpp:204-236, under the floor binning of the sort)
void locate(const Tree& t, double x, double y, double z, std::vector<long>& path) {
  uint64_t key = morton(grid_coord(x, t.L), grid_coord(y, t.L), grid_coord(z, t.L));
  path.clear();
  long id = 0;
  path.push_back(id);
  while (!t.nodes[id].leaf) {
    int lv = t.nodes[id].level + 1;
    int ch = int((key >> (3 * (KEY_BITS - lv))) & 7);
    id = t.nodes[id].child0 + ch;
    path.push_back(id);
  }
}

void form_pw_single(Tree& t, std::vector<std::vector<cd>>& pw, const std::vector<long>& path, double x, double y,
                    double z, double q) {
  // form_outgoing_pw_single (src/planewave.cpp:157-181)
  for (int i = 0; i < int(path.size()); ++i) {
    int nk;
    double dk;
    if (i == 0) {
      nk = t.n_window;
      dk = t.delta_k[0];
    } else if (i == 1 || i == t.max_depth - 1) {
      continue;
    } else {
      nk = t.n_diff;
      dk = t.delta_k[i];
    }
    nudft_single(dk * x, dk * y, dk * z, q, 2 * nk + 1, pw[i].data());
  }
}

// eval_shift_energy_res_vec + direct_eval (src/energy_shift.cpp:233-302,
// include/direct_eval.hpp:308-434) with an exact reciprocal square root
double shift_res(const Tree& t, const std::vector<long>& path, double x, double y, double z, double q) {
  long i = path.back();
  const Node& ni = t.nodes[i];
  double b = t.boxsize[ni.level];
  double thresh2 = std::numeric_limits<double>::epsilon();
  double b2 = b * b;
  double u = 0;
  auto add = [&](long j, double ox, double oy, double oz) {
    for (long s : t.node_particles[j]) {
      double dx = x - (t.r[3 * s] + ox), dy = y - (t.r[3 * s + 1] + oy), dz = z - (t.r[3 * s + 2] + oz);
      double r2 = dx * dx + dy * dy + dz * dz;
      if (r2 > thresh2 && r2 < b2) {
        double rr = std::sqrt(r2);
        u += t.q[s] * (t.poly_eval(rr / b) / rr);
      }
    }
  };
  add(i, 0, 0, 0);
  auto nbr_add = [&](long j) {
    double sh[3];
    node_shift(t, i, j, sh);
    const Node& nj = t.nodes[j];
    add(j, ni.center[0] - nj.center[0] + sh[0], ni.center[1] - nj.center[1] + sh[1],
        ni.center[2] - nj.center[2] + sh[2]);
  };
  for (long j : t.colleague[i]) nbr_add(j);
  for (long j : t.coarse[i]) nbr_add(j);
  return u * q;
}

// eval_shift_energy (src/energy_shift.cpp:18-140)
double shift_energy(Tree& t, long i_orig, double dx, double dy, double dz, double* parts) {
  long s = t.sorted_of_orig[i_orig];
  double q = t.q[s];
  double xo = t.r[3 * s], yo = t.r[3 * s + 1], zo = t.r[3 * s + 2];
  double xt = my_mod(xo + dx, t.L), yt = my_mod(yo + dy, t.L), zt = my_mod(zo + dz, t.L);
  double dr = std::sqrt(dx * dx + dy * dy + dz * dz);
  for (int mx = -1; mx <= 1; mx++)
    for (int my = -1; my <= 1; my++)
      for (int mz = -1; mz <= 1; mz++)
        dr = std::min(dr, std::sqrt(sq(xt - (xo + mx * t.L)) + sq(yt - (yo + my * t.L)) + sq(zt - (zo + mz * t.L))));
  locate(t, xt, yt, zt, t.path_t);
  locate(t, xo, yo, zo, t.path_o);
  form_pw_single(t, t.pw_o, t.path_o, xo, yo, zo, q);
  form_pw_single(t, t.pw_t, t.path_t, xt, yt, zt, q);
  // window (src/energy_shift.cpp:72-90)
  double dEw = 0;
  {
    const int dims = t.dims_window();
    double acc = 0;
    for (int k = 0; k < dims; ++k) {
      cd a = t.pw_t[0][k] - t.pw_o[0][k];
      cd b = t.out[0][k] - t.pw_o[0][k];
      acc += (a.real() * b.real() + a.imag() * b.imag()) * t.W[k];
    }
    dEw = 2.0 * acc * (1 / (2 * std::pow(2 * M_PI, 3)) * std::pow(t.delta_k[0], 3));
  }
  // difference (src/energy_shift.cpp:92-140)
  const int dims = t.dims_diff();
  double dEo = 0, dEt = 0;
  for (int l = 2; l < int(t.path_o.size()) - 1; ++l) {
    const auto& o = t.pw_o[l];
    const auto& inc = t.inc[t.path_o[l]];
    const auto& D = t.D[l];
    double acc = 0;
    for (int k = 0; k < dims; ++k)
      acc += (o[k].real() * inc[k].real() - o[k].imag() * inc[k].imag() - std::norm(o[k])) * D[k];
    dEo += acc / std::pow(2 * M_PI, 3) * std::pow(t.delta_k[l], 3);
  }
  for (int l = 2; l < int(t.path_t.size()) - 1; ++l) {
    const auto& tt = t.pw_t[l];
    const auto& inc = t.inc[t.path_t[l]];
    const auto& D = t.D[l];
    double acc = 0;
    for (int k = 0; k < dims; ++k) acc += (tt[k].real() * inc[k].real() - tt[k].imag() * inc[k].imag()) * D[k];
    dEt += acc / std::pow(2 * M_PI, 3) * std::pow(t.delta_k[l], 3);
  }
  double rt = shift_res(t, t.path_t, xt, yt, zt, q);
  double ro = shift_res(t, t.path_o, xo, yo, zo, q);
  double self = t.res_kernel(dr, t.boxsize[2]) * q * q;
  if (parts) {
    parts[0] = dEw;
    parts[1] = dEt - dEo;
    parts[2] = rt;
    parts[3] = ro;
    parts[4] = self;
  }
  return dEw + (dEt - dEo) + rt - ro - self;
}

// update_shift (src/tree.cpp:447-597); membership is kept exact on every
// level of both paths (the reference patches only the lowest two levels)
void update_shift(Tree& t, long i_orig, double dx, double dy, double dz, int nthreads) {
  // recompute the proposal so the call does not depend on a preceding shift
  shift_energy(t, i_orig, dx, dy, dz, nullptr);
  long s = t.sorted_of_orig[i_orig];
  double xo = t.r[3 * s], yo = t.r[3 * s + 1], zo = t.r[3 * s + 2];
  t.r[3 * s] = my_mod(xo + dx, t.L);
  t.r[3 * s + 1] = my_mod(yo + dy, t.L);
  t.r[3 * s + 2] = my_mod(zo + dz, t.L);
  const int dw = t.dims_window();
  for (int k = 0; k < dw; ++k) t.out[0][k] += t.pw_t[0][k];
  for (int k = 0; k < dw; ++k) t.out[0][k] -= t.pw_o[0][k];
  const int n = t.n_diff, d = 2 * n + 1, dims = t.dims_diff();
  auto apply = [&](const std::vector<long>& path, std::vector<std::vector<cd>>& pw, double sign) {
    for (int l = 2; l < int(path.size()); ++l) {
      if (l == t.max_depth - 1) continue;
      long ni = path[l];
      const auto& p = pw[l];
      for (int k = 0; k < dims; ++k) t.out[ni][k] += sign * p[k];
      for (int k = 0; k < dims; ++k) t.inc[ni][k] += sign * std::conj(p[k]);
      const Node& a = t.nodes[ni];
      double bs = t.boxsize[l], dk = t.delta_k[l];
      std::vector<long> targets;
      for (long j : t.colleague[ni])
        if (!t.nodes[j].leaf) targets.push_back(j);
#pragma omp parallel for num_threads(nthreads) schedule(static, 1)
      for (long w = 0; w < long(targets.size()); ++w) {
        long j = targets[w];
        const Node& b = t.nodes[j];
        int px = periodic_shift(a.center[0], b.center[0], t.L, bs, bs);
        int py = periodic_shift(a.center[1], b.center[1], t.L, bs, bs);
        int pz = periodic_shift(a.center[2], b.center[2], t.L, bs, bs);
        auto& inc = t.inc[j];
        if (!px && !py && !pz) {
          for (int k = 0; k < dims; ++k) inc[k] += sign * std::conj(p[k]);
        } else {
          for (int iz = 0; iz <= n; ++iz)
            for (int iy = 0; iy < d; ++iy)
              for (int ix = 0; ix < d; ++ix) {
                int k = (iz * d + iy) * d + ix;
                inc[k] += sign * std::conj(p[k] * shift_phase(ix, iy, iz, n, dk, t.L, px, py, pz));
              }
        }
      }
    }
  };
  apply(t.path_t, t.pw_t, 1.0);
  apply(t.path_o, t.pw_o, -1.0);
  for (long id : t.path_o) {
    auto& v = t.node_particles[id];
    v.erase(std::find(v.begin(), v.end(), s));
  }
  for (long id : t.path_t) t.node_particles[id].push_back(s);
}

// energy_direct.cpp restatements (src/energy_direct.cpp:20-186)
void energy_direct(const Tree& t, int nthreads, double* parts) {
  // window: explicit full k-cube sum
  double ew = 0;
  {
    int nk = t.n_window;
    double dk0 = t.delta_k[0], sigma = t.sigmas[2];
    int d = 2 * nk + 1;
#pragma omp parallel for reduction(+ : ew) collapse(2) num_threads(nthreads)
    for (int i = 0; i < d; ++i)
      for (int j = 0; j < d; ++j)
        for (int k = 0; k < d; ++k) {
          double kx = (i - nk) * dk0, ky = (j - nk) * dk0, kz = (k - nk) * dk0;
          double k2 = kx * kx + ky * ky + kz * kz;
          cd rho = 0;
          for (long s = 0; s < t.n; ++s)
            rho += std::exp(cd(0, kx * t.r[3 * s] + ky * t.r[3 * s + 1] + kz * t.r[3 * s + 2])) * t.q[s];
          double wk = 0;
          if (k2 != 0) wk = 2 * M_PI * t.lambda * t.psi0(std::sqrt(k2) * sigma) / t.C0 / k2;
          ew += std::norm(rho) * wk;
        }
    ew *= 1 / (2 * std::pow(2 * M_PI, 3)) * std::pow(dk0, 3);
    ew -= t.Q * t.psi0_0 / (2 * t.boxsize[2] * t.C0);
  }
  auto img_sum = [&](long s, auto&& kern) {
    double acc = 0;
    for (long u = 0; u < t.n; ++u) {
      if (u == s) continue;
      for (int mx = -1; mx <= 1; mx++)
        for (int my = -1; my <= 1; my++)
          for (int mz = -1; mz <= 1; mz++) {
            double rr = std::sqrt(sq(t.r[3 * s] - (t.r[3 * u] + mx * t.L)) + sq(t.r[3 * s + 1] - (t.r[3 * u + 1] + my * t.L)) +
                                  sq(t.r[3 * s + 2] - (t.r[3 * u + 2] + mz * t.L)));
            acc += t.q[s] * t.q[u] * kern(rr) / 2;
          }
    }
    return acc;
  };
  double ed = 0, er = 0;
  for (int l = 2; l < t.max_depth; ++l) {
    const auto& lv = t.level_indices[l];
    double bl = t.boxsize[l], bl1 = t.boxsize[l + 1];
    for (long id : lv) {
      if (t.node_particles[id].empty()) continue;
      const auto& P = t.node_particles[id];
      if (!t.nodes[id].leaf) {
#pragma omp parallel for reduction(+ : ed) num_threads(nthreads)
        for (long w = 0; w < long(P.size()); ++w)
          ed += img_sum(P[w], [&](double rr) { return -(t.poly_eval(rr / bl1) - t.poly_eval(rr / bl)) / rr; });
      } else {
#pragma omp parallel for reduction(+ : er) num_threads(nthreads)
        for (long w = 0; w < long(P.size()); ++w) er += img_sum(P[w], [&](double rr) { return t.res_kernel(rr, bl); });
      }
    }
  }
  parts[0] = ew;
  parts[1] = ed;
  parts[2] = er;
}

}  // namespace

extern "C" {

void* or_create(double L, int n_per_leaf, int digits, long n, const double* r, const double* q, int n_leg,
                const double* leg, double c, double lambda, double C0, double diff0, int n_poly, const double* poly,
                int n_window, int n_diff) {
  auto* t = new Tree();
  t->L = L;
  t->n_per_leaf = n_per_leaf;
  t->digits = digits;
  t->n = n;
  t->leg.assign(leg, leg + n_leg);
  t->poly.assign(poly, poly + n_poly);
  t->c = c;
  t->lambda = lambda;
  t->C0 = C0;
  t->diff0 = diff0;
  t->n_window = n_window;
  t->n_diff = n_diff;
  build_tree(*t, r, q);
  build_neighbors(*t);
  build_setup(*t);
  return t;
}

void or_destroy(void* h) { delete static_cast<Tree*>(h); }

void or_info(void* h, long* info) {
  auto* t = static_cast<Tree*>(h);
  info[0] = t->max_depth;
  info[1] = long(t->nodes.size());
  info[2] = t->n;
  info[3] = t->dims_window();
  info[4] = t->dims_diff();
  info[5] = t->n_window;
  info[6] = t->n_diff;
}

void or_form_outgoing(void* h, int nthreads) { form_outgoing(*static_cast<Tree*>(h), nthreads); }
void or_form_incoming(void* h, int nthreads) { form_incoming(*static_cast<Tree*>(h), nthreads); }

void or_energy(void* h, int nthreads, double* parts) {
  auto* t = static_cast<Tree*>(h);
  parts[0] = energy_window(*t);
  parts[1] = energy_diff(*t, nthreads);
  parts[2] = energy_res(*t, nthreads);
}

void or_energy_direct(void* h, int nthreads, double* parts) { energy_direct(*static_cast<Tree*>(h), nthreads, parts); }

double or_shift(void* h, long i, double dx, double dy, double dz, double* parts) {
  return shift_energy(*static_cast<Tree*>(h), i, dx, dy, dz, parts);
}
void or_update(void* h, long i, double dx, double dy, double dz, int nthreads) {
  update_shift(*static_cast<Tree*>(h), i, dx, dy, dz, nthreads);
}

void or_tree_nodes(void* h, int* level, uint64_t* prefix, int* is_leaf, long* count) {
  auto* t = static_cast<Tree*>(h);
  for (size_t i = 0; i < t->nodes.size(); ++i) {
    level[i] = t->nodes[i].level;
    prefix[i] = t->nodes[i].prefix;
    is_leaf[i] = t->nodes[i].leaf ? 1 : 0;
    count[i] = long(t->node_particles[i].size());
  }
}

void or_tree_neighbors(void* h, int* col27, int* coarse8) {
  auto* t = static_cast<Tree*>(h);
  for (size_t i = 0; i < t->nodes.size(); ++i) {
    for (int k = 0; k < 27; ++k) {
      int j = t->nodes[i].level >= 2 ? t->nbr[i][k] : -1;
      col27[i * 27 + k] = (j == int(i)) ? -1 : j;
    }
    for (int k = 0; k < 8; ++k) coarse8[i * 8 + k] = k < int(t->coarse[i].size()) ? int(t->coarse[i][k]) : -1;
  }
}

void or_sorted_order(void* h, long* out) {
  auto* t = static_cast<Tree*>(h);
  std::copy(t->orig_of_sorted.begin(), t->orig_of_sorted.end(), out);
}

void or_positions(void* h, double* out) {
  auto* t = static_cast<Tree*>(h);
  for (long s = 0; s < t->n; ++s) {
    long i = t->orig_of_sorted[s];
    out[3 * i] = t->r[3 * s];
    out[3 * i + 1] = t->r[3 * s + 1];
    out[3 * i + 2] = t->r[3 * s + 2];
  }
}

void or_get_pw(void* h, long node, int which, double* out) {
  auto* t = static_cast<Tree*>(h);
  const auto& v = which == 0 ? t->out[node] : t->inc[node];
  int dims = node == 0 ? t->dims_window() : t->dims_diff();
  for (int k = 0; k < dims && k < int(v.size()); ++k) {
    out[2 * k] = v[k].real();
    out[2 * k + 1] = v[k].imag();
  }
}

void or_get_W(void* h, double* out) {
  auto* t = static_cast<Tree*>(h);
  std::copy(t->W.begin(), t->W.end(), out);
}
void or_get_D(void* h, int level, double* out) {
  auto* t = static_cast<Tree*>(h);
  std::copy(t->D[level].begin(), t->D[level].end(), out);
}

void or_leaf_path(void* h, double x, double y, double z, long* path, int* depth) {
  auto* t = static_cast<Tree*>(h);
  std::vector<long> p;
  locate(*t, x, y, z, p);
  *depth = int(p.size());
  std::copy(p.begin(), p.end(), path);
}

// Ewald (src/ewald.cpp:17-223)
double or_ewald_energy(double L, double s, double alpha, long n, const double* r, const double* q, int nthreads) {
  double rc = s / alpha, kc = 2 * s * alpha, V = L * L * L;
  int nk = int(std::ceil(kc / (2 * M_PI / L)));
  int d = 2 * nk + 1;
  double dk = 2 * M_PI / L;
  double es = 0;
#pragma omp parallel for reduction(+ : es) schedule(dynamic, 16) num_threads(nthreads)
  for (long i = 0; i < n; ++i)
    for (long j = 0; j < n; ++j)
      for (int mx = -1; mx <= 1; mx++)
        for (int my = -1; my <= 1; my++)
          for (int mz = -1; mz <= 1; mz++) {
            if (i == j && !mx && !my && !mz) continue;
            double rr = std::sqrt(sq(r[3 * i] - r[3 * j] - mx * L) + sq(r[3 * i + 1] - r[3 * j + 1] - my * L) +
                                  sq(r[3 * i + 2] - r[3 * j + 2] - mz * L));
            if (rr <= rc) es += q[i] * q[j] * std::erfc(alpha * rr) / rr;
          }
  es /= 2.0;
  // long range: separable structure factor over the full cube
  std::vector<double> el_part(nthreads, 0.0);
  std::vector<cd> rho(size_t(d) * d * d, cd(0));
  {
    std::vector<std::vector<cd>> part(nthreads, std::vector<cd>(size_t(d) * d * d, cd(0)));
#pragma omp parallel num_threads(nthreads)
    {
      int tid = omp_get_thread_num();
      long b = n * tid / nthreads, e = n * (tid + 1) / nthreads;
      std::vector<cd> ex(d), ey(d), ez(d);
      for (long i = b; i < e; ++i) {
        cd x0 = std::exp(-cd(0, 1) * dk * r[3 * i]), y0 = std::exp(-cd(0, 1) * dk * r[3 * i + 1]),
           z0 = std::exp(-cd(0, 1) * dk * r[3 * i + 2]);
        for (int a = -nk; a <= nk; a++) {
          ex[a + nk] = std::pow(x0, a);
          ey[a + nk] = std::pow(y0, a);
          ez[a + nk] = std::pow(z0, a);
        }
        for (int ix = 0; ix < d; ix++)
          for (int iy = 0; iy < d; iy++) {
            cd t2 = ey[iy] * ex[ix];
            for (int iz = 0; iz < d; iz++) part[tid][(size_t(ix) * d + iy) * d + iz] += q[i] * (ez[iz] * t2);
          }
      }
    }
    for (int th = 0; th < nthreads; ++th)
      for (size_t k = 0; k < rho.size(); ++k) rho[k] += part[th][k];
  }
  double el = 0;
  for (int ix = 0; ix < d; ix++)
    for (int iy = 0; iy < d; iy++)
      for (int iz = 0; iz < d; iz++) {
        double kx = (ix - nk) * dk, ky = (iy - nk) * dk, kz = (iz - nk) * dk;
        double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 == 0) continue;
        el += std::exp(-k2 / (4 * alpha * alpha)) / k2 * std::norm(rho[(size_t(ix) * d + iy) * d + iz]);
      }
  el *= 2 * M_PI / V;
  double eself = 0;
  for (long i = 0; i < n; ++i) eself += -q[i] * q[i] * alpha / std::sqrt(M_PI);
  return es + el + eself;
}

// potential at (x,y,z) of all charges except `exclude` (src/ewald.cpp:225-308)
double or_ewald_potential(double L, double s, double alpha, long n, const double* r, const double* q, double x,
                          double y, double z, long exclude, int nthreads) {
  double rc = s / alpha, kc = 2 * s * alpha, V = L * L * L;
  int nk = int(std::ceil(kc / (2 * M_PI / L)));
  double dk = 2 * M_PI / L;
  double ps = 0, pl = 0;
#pragma omp parallel for reduction(+ : ps, pl) schedule(static) num_threads(nthreads)
  for (long i = 0; i < n; ++i) {
    if (i == exclude) continue;
    for (int mx = -1; mx <= 1; mx++)
      for (int my = -1; my <= 1; my++)
        for (int mz = -1; mz <= 1; mz++) {
          double rr = std::sqrt(sq(r[3 * i] + mx * L - x) + sq(r[3 * i + 1] + my * L - y) + sq(r[3 * i + 2] + mz * L - z));
          if (rr <= rc && rr > 0) ps += q[i] * std::erfc(alpha * rr) / rr;
        }
    // reciprocal part: sum over k of e^{-k^2/4a^2}/k^2 * Re(q e^{-ik.(r_i - x)})
    double ddx = r[3 * i] - x, ddy = r[3 * i + 1] - y, ddz = r[3 * i + 2] - z;
    double acc = 0;
    for (int a = -nk; a <= nk; ++a)
      for (int b = -nk; b <= nk; ++b)
        for (int c = -nk; c <= nk; ++c) {
          double kx = a * dk, ky = b * dk, kz = c * dk;
          double k2 = kx * kx + ky * ky + kz * kz;
          if (k2 == 0) continue;
          acc += std::exp(-k2 / (4 * alpha * alpha)) / k2 * std::cos(kx * ddx + ky * ddy + kz * ddz);
        }
    pl += q[i] * acc;
  }
  pl *= 4 * M_PI / V;
  return ps + pl;
}

// Stateful Ewald for sequential moves: keeps the structure factor rho(k) of
// the full cube (src/ewald.cpp:103-176) so the exact energy change of a move
// costs O(N + K) instead of two full potentials.
struct EwaldState {
  double L, s, alpha, rc;
  int nk, d;
  double dk;
  std::vector<double> r, q, f;
  std::vector<cd> rho;
};

static void ewald_phases(const EwaldState& e, double x, double y, double z, std::vector<cd>& ex, std::vector<cd>& ey,
                         std::vector<cd>& ez) {
  cd x0 = std::exp(-cd(0, 1) * e.dk * x), y0 = std::exp(-cd(0, 1) * e.dk * y), z0 = std::exp(-cd(0, 1) * e.dk * z);
  for (int a = -e.nk; a <= e.nk; a++) {
    ex[a + e.nk] = std::pow(x0, a);
    ey[a + e.nk] = std::pow(y0, a);
    ez[a + e.nk] = std::pow(z0, a);
  }
}

void* or_ewald_create(double L, double s, double alpha, long n, const double* r, const double* q, int nthreads) {
  auto* e = new EwaldState();
  e->L = L;
  e->s = s;
  e->alpha = alpha;
  e->rc = s / alpha;
  e->nk = int(std::ceil(2 * s * alpha / (2 * M_PI / L)));
  e->d = 2 * e->nk + 1;
  e->dk = 2 * M_PI / L;
  e->r.assign(r, r + 3 * n);
  e->q.assign(q, q + n);
  const int d = e->d;
  e->f.assign(size_t(d) * d * d, 0.0);
  for (int ix = 0; ix < d; ix++)
    for (int iy = 0; iy < d; iy++)
      for (int iz = 0; iz < d; iz++) {
        double kx = (ix - e->nk) * e->dk, ky = (iy - e->nk) * e->dk, kz = (iz - e->nk) * e->dk;
        double k2 = kx * kx + ky * ky + kz * kz;
        if (k2 != 0) e->f[(size_t(ix) * d + iy) * d + iz] = std::exp(-k2 / (4 * alpha * alpha)) / k2;
      }
  e->rho.assign(size_t(d) * d * d, cd(0));
  std::vector<std::vector<cd>> part(nthreads, std::vector<cd>(e->rho.size(), cd(0)));
#pragma omp parallel num_threads(nthreads)
  {
    int tid = omp_get_thread_num();
    long b = n * tid / nthreads, en = n * (tid + 1) / nthreads;
    std::vector<cd> ex(d), ey(d), ez(d);
    for (long i = b; i < en; ++i) {
      ewald_phases(*e, r[3 * i], r[3 * i + 1], r[3 * i + 2], ex, ey, ez);
      for (int ix = 0; ix < d; ix++)
        for (int iy = 0; iy < d; iy++) {
          cd t2 = ey[iy] * ex[ix];
          for (int iz = 0; iz < d; iz++) part[tid][(size_t(ix) * d + iy) * d + iz] += q[i] * (ez[iz] * t2);
        }
    }
  }
  for (int th = 0; th < nthreads; ++th)
    for (size_t k = 0; k < e->rho.size(); ++k) e->rho[k] += part[th][k];
  return e;
}

void or_ewald_destroy(void* h) { delete static_cast<EwaldState*>(h); }

// exact Ewald energy change of moving particle i by (dx,dy,dz) wrapped into
// the box; with apply != 0 the move is committed
double or_ewald_move(void* h, long i, double dx, double dy, double dz, int apply) {
  auto* e = static_cast<EwaldState*>(h);
  const long n = long(e->q.size());
  const double L = e->L;
  double xo = e->r[3 * i], yo = e->r[3 * i + 1], zo = e->r[3 * i + 2];
  double xn = my_mod(xo + dx, L), yn = my_mod(yo + dy, L), zn = my_mod(zo + dz, L);
  double ds = 0;
  for (long j = 0; j < n; ++j) {
    if (j == i) continue;
    for (int mx = -1; mx <= 1; mx++)
      for (int my = -1; my <= 1; my++)
        for (int mz = -1; mz <= 1; mz++) {
          double xj = e->r[3 * j] + mx * L, yj = e->r[3 * j + 1] + my * L, zj = e->r[3 * j + 2] + mz * L;
          double rn = std::sqrt(sq(xn - xj) + sq(yn - yj) + sq(zn - zj));
          double ro = std::sqrt(sq(xo - xj) + sq(yo - yj) + sq(zo - zj));
          if (rn <= e->rc) ds += e->q[j] * std::erfc(e->alpha * rn) / rn;
          if (ro <= e->rc) ds -= e->q[j] * std::erfc(e->alpha * ro) / ro;
        }
  }
  ds *= e->q[i];
  const int d = e->d;
  std::vector<cd> exo(d), eyo(d), ezo(d), exn(d), eyn(d), ezn(d);
  ewald_phases(*e, xo, yo, zo, exo, eyo, ezo);
  ewald_phases(*e, xn, yn, zn, exn, eyn, ezn);
  double dl = 0;
  std::vector<cd> delta(apply ? e->rho.size() : 0);
  for (int ix = 0; ix < d; ix++)
    for (int iy = 0; iy < d; iy++)
      for (int iz = 0; iz < d; iz++) {
        size_t k = (size_t(ix) * d + iy) * d + iz;
        cd del = e->q[i] * (exn[ix] * eyn[iy] * ezn[iz] - exo[ix] * eyo[iy] * ezo[iz]);
        dl += e->f[k] * (2 * (std::conj(e->rho[k]) * del).real() + std::norm(del));
        if (apply) delta[k] = del;
      }
  dl *= 2 * M_PI / (L * L * L);
  if (apply) {
    for (size_t k = 0; k < e->rho.size(); ++k) e->rho[k] += delta[k];
    e->r[3 * i] = xn;
    e->r[3 * i + 1] = yn;
    e->r[3 * i + 2] = zn;
  }
  return ds + dl;
}

// primitives exported for the golden-vector checks
void or_nudft_halfplane(long M, const double* x, const double* y, const double* z, const double* c, int N, double* f) {
  nudft_halfplane(M, x, y, z, c, N, reinterpret_cast<cd*>(f));
}
void or_nudft_single(double x, double y, double z, double q, int N, double* f) {
  nudft_single(x, y, z, q, N, reinterpret_cast<cd*>(f));
}
void or_shift_phases(int n, double dk, double L, int px, int py, int pz, double* out) {
  int d = 2 * n + 1;
  for (int iz = 0; iz <= n; ++iz)
    for (int iy = 0; iy < d; ++iy)
      for (int ix = 0; ix < d; ++ix) {
        cd v = shift_phase(ix, iy, iz, n, dk, L, px, py, pz);
        size_t k = (size_t(iz) * d + iy) * d + ix;
        out[2 * k] = v.real();
        out[2 * k + 1] = v.imag();
      }
}
double or_res_kernel(int n_poly, const double* poly, double r, double cutoff) {
  Tree t;
  t.poly.assign(poly, poly + n_poly);
  return t.res_kernel(r, cutoff);
}
double or_my_mod(double x, double L) { return my_mod(x, L); }
int or_periodic_shift(double xi, double xj, double L, double bi, double bj) { return periodic_shift(xi, xj, L, bi, bj); }

// the reference tests' trial-move stream: a fresh default-seeded
// std::mt19937 drawing dx, dy, dz from uniform_real_distribution(0, L) and
// the particle from uniform_int_distribution(0, n-1), per trial
// (test/hpdmk_test.cpp:407-418, :498-507)
void or_reference_trials(long ntrials, double L, long n, double* d, long* idx) {
  std::mt19937 gen;
  std::uniform_real_distribution<double> dist(0, L);
  std::uniform_int_distribution<int> di(0, int(n - 1));
  for (long t = 0; t < ntrials; ++t) {
    d[3 * t] = dist(gen);
    d[3 * t + 1] = dist(gen);
    d[3 * t + 2] = dist(gen);
    idx[t] = di(gen);
  }
}

void or_random_init(long n, double lo, double hi, double* out) {
  std::mt19937 gen;
  std::uniform_real_distribution<double> dist(lo, hi);
  for (long i = 0; i < n; ++i) out[i] = dist(gen);
}
}
