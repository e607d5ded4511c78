// Tree build on the GPU: Morton keys, radix sort, count-driven refinement,
// periodic 2:1 balance on per-level refinement bitmaps, node enumeration,
// neighbour lists, and the slotted particle layout.
//
// Reference counterpart: the HPDMKPtTree constructor (src/tree.cpp:267-444)
// on top of SCTL's PtTree::UpdateRefinement(pts, n_per_leaf, balance21=true,
// periodic=true), collect_particles (src/tree.cpp:117-133) and
// collect_neighbors / node_shift (src/tree.cpp:136-201). The tree rules are:
// refine a node holding more than n_per_leaf particles (down to level 10);
// refine every node above level 2; close under periodic 2:1 balance over all
// 26 neighbours; number nodes level by level in Morton order.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <map>
#include <mutex>
#include <stdexcept>

#include "common.cuh"
#include "hostpar.hpp"
#include "sort.cuh"
#include "tree.hpp"

namespace pdmk {
namespace {

constexpr int TPB = 256;

inline unsigned grid_for(long n, int tpb = TPB) { return unsigned(std::max<long>(1, (n + tpb - 1) / tpb)); }

// Small host values reach the device as a kernel argument: a cudaMemcpyAsync
// from pageable host memory would first wait for the stream to drain.
struct SmallWords {
  int n;
  uint32_t w[256];
};

__global__ void k_put_words(uint32_t* dst, SmallWords v) {
  for (int i = threadIdx.x; i < v.n; i += blockDim.x) dst[i] = v.w[i];
}

void put_small(void* dst, const void* src, size_t bytes, cudaStream_t st) {
  SmallWords v;
  if (bytes % 4 != 0 || bytes > sizeof(v.w)) throw std::logic_error("put_small: size");
  v.n = int(bytes / 4);
  std::memcpy(v.w, src, bytes);
  k_put_words<<<1, 64, 0, st>>>(static_cast<uint32_t*>(dst), v);
  PDMK_LAUNCH_CHECK();
}

// ---------------------------------------------------------------------------
__global__ void k_keys(const double* r, long n, double L, uint64_t* key, int* val) {
  long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  key[i] = morton3(grid_coord(r[3 * i], L), grid_coord(r[3 * i + 1], L), grid_coord(r[3 * i + 2], L));
  val[i] = int(i);
}

__global__ void k_gather_sorted(const double* r, const double* q, const int* ord, long n, double* x, double* y,
                                double* z, double* c) {
  long s = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int i = ord[s];
  x[s] = r[3 * i];
  y[s] = r[3 * i + 1];
  z[s] = r[3 * i + 2];
  c[s] = q[i];
}

__device__ inline long lower_bound_u64(const uint64_t* a, long n, uint64_t v) {
  long lo = 0, hi = n;
  while (lo < hi) {
    long mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

__device__ inline void cell_range(const uint64_t* keys, long n, int level, uint64_t prefix, long* lo, long* hi) {
  if (level == 0) {
    *lo = 0;
    *hi = n;
    return;
  }
  int sh = 3 * (KEY_BITS - level);
  *lo = lower_bound_u64(keys, n, prefix << sh);
  *hi = lower_bound_u64(keys, n, (prefix + 1) << sh);
}

__device__ inline bool bit_get(const uint32_t* bm, uint64_t cell) { return (bm[cell >> 5] >> (cell & 31)) & 1u; }
__device__ inline void bit_set(uint32_t* bm, uint64_t cell) {
  uint32_t m = 1u << (cell & 31);
  if (!(bm[cell >> 5] & m)) atomicOr(&bm[cell >> 5], m);
}

struct Bitmaps {
  uint32_t* bm[MAX_LEVELS];
  int* wprefix[MAX_LEVELS];  // exclusive prefix of word popcounts
};

// refined-cell rank within its level (Morton order)
__device__ inline int cell_rank(const Bitmaps& B, int level, uint64_t cell) {
  uint32_t w = B.bm[level][cell >> 5];
  return B.wprefix[level][cell >> 5] + __popc(w & ((1u << (cell & 31)) - 1u));
}

// candidates at `level` are the 8 children of each refined cell of the level above
// The parent count comes from the device (the previous level's out_n), so
// levels can be launched back to back; lists hold at most list_cap cells and
// the host checks the counts for overflow when it reads them.
__global__ void k_refine_level(const uint64_t* keys, long n, int level, int n_per_leaf, const uint64_t* parents,
                               const int* n_parents, int list_cap, uint32_t* bm, uint64_t* out_list, int* out_n) {
  long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const int np = min(*n_parents, list_cap);
  if (t >= long(np) * 8) return;
  uint64_t cell = (parents[t >> 3] << 3) | uint64_t(t & 7);
  long lo, hi;
  cell_range(keys, n, level, cell, &lo, &hi);
  bool refine = (level < 2) || ((hi - lo) > n_per_leaf && level < MAX_LEVEL);
  if (refine) {
    bit_set(bm, cell);
    int k = atomicAdd(out_n, 1);
    if (k < list_cap) out_list[k] = cell;
  }
}

// 2:1 balance: a refined cell at level k needs all 26 neighbours at level k
// to exist, i.e. their parents (level k-1) and all ancestors refined. One
// thread per (cell, neighbour) pair where that fits in kBalanceFanThreads
// threads, one thread per cell with a loop over its 26 neighbours on deeper,
// larger levels. A walk up the ancestors stops at the first cell already
// refined: a refined cell's ancestors are refined too, or are being set by the
// thread that refined it, so the bitmaps at the end are the same union.
constexpr long kBalanceFanThreads = 1L << 24;

__global__ void k_balance_level(Bitmaps B, int level, int fan) {
  const long ncells = 1L << (3 * level);
  const long t = long(blockIdx.x) * blockDim.x + threadIdx.x;
  const long cell = t / fan;
  if (cell >= ncells || !bit_get(B.bm[level], uint64_t(cell))) return;
  const int k0 = fan == 26 ? int(t % 26) : 0, k1 = fan == 26 ? k0 + 1 : 26;
  const uint32_t mask = (1u << level) - 1u;
  const uint32_t X = compact3(uint64_t(cell)), Y = compact3(uint64_t(cell) >> 1), Z = compact3(uint64_t(cell) >> 2);
  for (int k = k0; k < k1; ++k) {
    const int j = k < 13 ? k : k + 1;  // 3x3x3 offsets without the centre (13)
    const int dx = j % 3 - 1, dy = (j / 3) % 3 - 1, dz = j / 9 - 1;
    uint64_t nb = morton3((X + dx) & mask, (Y + dy) & mask, (Z + dz) & mask);
    for (int lv = level - 1; lv >= 0; --lv) {
      nb >>= 3;
      uint32_t* wp = B.bm[lv] + (nb >> 5);
      const uint32_t m = 1u << (nb & 31);
      if (*wp & m) break;
      if (atomicOr(wp, m) & m) break;
    }
  }
}

__global__ void k_word_popc(const uint32_t* bm, long nwords, int* out) {
  long w = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w < nwords) out[w] = __popc(bm[w]);
}

__global__ void k_level_total(const uint32_t* bm, const int* wprefix, long nwords, int* total) {
  *total = wprefix[nwords - 1] + __popc(bm[nwords - 1]);
}

struct NodeArrays {
  uint64_t* prefix;
  int* level;
  int* parent;
  int* child0;
};

__global__ void k_enum_nodes(Bitmaps B, int level, int maxref, const int* level_start, NodeArrays na) {
  // nodes at `level` are the children of refined cells at level-1
  int pl = level - 1;
  long nwords = (1L << (3 * pl)) >> 5;
  if (nwords < 1) nwords = 1;
  long w = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (w >= nwords) return;
  uint32_t bits = B.bm[pl][w];
  while (bits) {
    int b = __ffs(bits) - 1;
    bits &= bits - 1;
    uint64_t pc = (uint64_t(w) << 5) | uint64_t(b);
    int r = cell_rank(B, pl, pc);
    int pid = (pl == 0) ? 0 : level_start[pl] + 8 * cell_rank(B, pl - 1, pc >> 3) + int(pc & 7);
    for (int c = 0; c < 8; ++c) {
      int id = level_start[level] + 8 * r + c;
      uint64_t cell = (pc << 3) | uint64_t(c);
      na.prefix[id] = cell;
      na.level[id] = level;
      na.parent[id] = pid;
      int ch = -1;
      if (level <= maxref && bit_get(B.bm[level], cell)) ch = level_start[level + 1] + 8 * cell_rank(B, level, cell);
      na.child0[id] = ch;
    }
  }
}

__device__ inline double center_coord(double L, int level, uint32_t ic) {
  double scale = ldexp(1.0, -level);
  return L * (double(ic) * scale + 0.5 * scale);
}

// periodic_shift (include/utils.hpp:58-67)
__device__ inline int periodic_shift_dev(double xi, double xj, double L, double bi, double bj) {
  if (xi < bi && xj > (L - bj)) return 1;
  if (xi > (L - bi) && xj < bj) return -1;
  return 0;
}

// same-level neighbour cell -> node id or -1
__device__ inline int nbr_node(const Bitmaps& B, const int* level_start, int level, uint64_t cell) {
  if (level == 0) return 0;
  uint64_t pc = cell >> 3;
  if (level >= 2 && !bit_get(B.bm[level - 1], pc)) return -1;
  int pr = (level == 1) ? 0 : cell_rank(B, level - 1, pc);
  return level_start[level] + 8 * pr + int(cell & 7);
}

__global__ void k_neighbors(Bitmaps B, const int* level_start, int n_nodes, int lo_node, double L, const double* boxsize,
                            const uint64_t* prefix, const int* level, const int* parent, const int* child0, int* col27,
                            int* coarse8) {
  int id = lo_node + blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n_nodes) return;
  int l = level[id];
  uint64_t p = prefix[id];
  uint32_t X = compact3(p), Y = compact3(p >> 1), Z = compact3(p >> 2);
  uint32_t mask = (1u << l) - 1u;
  int ncol = 0;
  for (int k = 0; k < 27; ++k) {
    int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
    int j = -1;
    if (k != 13) j = nbr_node(B, level_start, l, morton3((X + dx) & mask, (Y + dy) & mask, (Z + dz) & mask));
    col27[long(id) * 27 + k] = j;
    ncol += (j >= 0);
  }
  for (int k = 0; k < 8; ++k) coarse8[long(id) * 8 + k] = -1;
  if (ncol < 26) {
    int par = parent[id];
    int pl = l - 1;
    uint64_t pp = prefix[par];
    uint32_t PX = compact3(pp), PY = compact3(pp >> 1), PZ = compact3(pp >> 2);
    uint32_t pmask = (1u << pl) - 1u;
    double bs_i = boxsize[l], bs_p = boxsize[pl];
    double ci[3] = {center_coord(L, l, X), center_coord(L, l, Y), center_coord(L, l, Z)};
    double cp[3] = {center_coord(L, pl, PX), center_coord(L, pl, PY), center_coord(L, pl, PZ)};
    double s_i2p[3];
    for (int d = 0; d < 3; ++d) {
      int ps = periodic_shift_dev(cp[d], ci[d], L, bs_p, bs_i);
      s_i2p[d] = ci[d] - (cp[d] + ps * L);
    }
    int nc = 0;
    for (int k = 0; k < 27; ++k) {
      if (k == 13) continue;
      int dx = k % 3 - 1, dy = (k / 3) % 3 - 1, dz = k / 9 - 1;
      uint32_t NX = (PX + dx) & pmask, NY = (PY + dy) & pmask, NZ = (PZ + dz) & pmask;
      int j = nbr_node(B, level_start, pl, morton3(NX, NY, NZ));
      if (j < 0 || j == par || child0[j] >= 0) continue;
      double cn[3] = {center_coord(L, pl, NX), center_coord(L, pl, NY), center_coord(L, pl, NZ)};
      bool ok = true;
      for (int d = 0; d < 3; ++d) {
        int ps = periodic_shift_dev(cp[d], cn[d], L, bs_p, bs_p);
        double s_n2p = cn[d] - (cp[d] + ps * L);
        ok = ok && (s_i2p[d] * s_n2p >= 0);
      }
      if (ok && nc < 8) coarse8[long(id) * 8 + nc++] = j;
    }
  }
}

__global__ void k_node_ranges(const uint64_t* keys, long n, int n_nodes, const uint64_t* prefix, const int* level,
                              long* lo, long* hi) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n_nodes) return;
  long a, b;
  cell_range(keys, n, level[id], prefix[id], &a, &b);
  lo[id] = a;
  hi[id] = b;
}

__global__ void k_collect_leaves(int n_nodes, const uint64_t* prefix, const int* level, const int* child0,
                                 uint64_t* lkey, int* lid, int* nleaf) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n_nodes || child0[id] >= 0) return;
  int k = atomicAdd(nleaf, 1);
  lkey[k] = prefix[id] << (3 * (KEY_BITS - level[id]));
  lid[k] = id;
}

// per DFS leaf j: source range and capacity
__global__ void k_leaf_caps(int nl, const int* lid, const long* lo, const long* hi, int slack, int* cnt, int* cap,
                            long* src_lo) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nl) return;
  int id = lid[j];
  cnt[j] = int(hi[id] - lo[id]);
  cap[j] = cnt[j] + slack;
  src_lo[j] = lo[id];
}

__global__ void k_fill_slots(int n_slots, int nl, const int* begin, const int* cnt, const long* src_lo, const int* lid,
                             const uint64_t* prefix, const int* level, double L, const double* dx, const double* dy,
                             const double* dz, const double* dq, const int* dorig, double* sx, double* sy, double* sz,
                             double* sq, int* s_orig, int* orig_slot) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_slots) return;
  int lo = 0, hi = nl;  // last j with begin[j] <= s
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if (begin[mid] <= s) lo = mid;
    else hi = mid;
  }
  int j = lo;
  int local = s - begin[j];
  if (local < cnt[j]) {
    long src = src_lo[j] + local;
    sx[s] = dx[src];
    sy[s] = dy[src];
    sz[s] = dz[src];
    sq[s] = dq[src];
    int o = dorig[src];
    s_orig[s] = o;
    orig_slot[o] = s;
  } else {
    int id = lid[j];
    int l = level[id];
    uint64_t p = prefix[id];
    sx[s] = center_coord(L, l, compact3(p));
    sy[s] = center_coord(L, l, compact3(p >> 1));
    sz[s] = center_coord(L, l, compact3(p >> 2));
    sq[s] = 0.0;
    s_orig[s] = -1;
  }
}

__global__ void k_leaf_dfs_index(int nl, const int* lid, int* dfs_of_node) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nl) dfs_of_node[lid[j]] = j;
}

__global__ void k_node_slots(int n_nodes, const int* child0, const int* dfs_of_node, const int* begin, const int* cap,
                             const int* cnt, const int* cnt_prefix, int* node_begin, int* node_end, int* leaf_count,
                             int* node_count) {
  int id = blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= n_nodes) return;
  int f = id, g = id;
  while (child0[f] >= 0) f = child0[f];
  while (child0[g] >= 0) g = child0[g] + 7;
  int jf = dfs_of_node[f], jg = dfs_of_node[g];
  node_begin[id] = begin[jf];
  node_end[id] = begin[jg] + cap[jg];
  leaf_count[id] = (child0[id] < 0) ? cnt[jf] : 0;
  node_count[id] = cnt_prefix[jg] + cnt[jg] - cnt_prefix[jf];
}

// repack: gather live particles leaf by leaf (slots, then pool entries)
__global__ void k_repack_counts(int pool_used, const int* p_leaf, const int* p_orig, const int* dfs_of_node, int* cnt) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= pool_used || p_orig[p] < 0) return;
  atomicAdd(&cnt[dfs_of_node[p_leaf[p]]], 1);
}

__global__ void k_repack_gather_slots(int nl, const int* lid, const int* node_begin, const int* leaf_count,
                                      const int* dense_begin, const double* sx, const double* sy, const double* sz,
                                      const double* sq, const int* s_orig, double* dx, double* dy, double* dz,
                                      double* dq, int* dorig) {
  int j = blockIdx.x;
  if (j >= nl) return;
  int id = lid[j];
  int b = node_begin[id], c = leaf_count[id];
  for (int t = threadIdx.x; t < c; t += blockDim.x) {
    int s = b + t;
    long d = dense_begin[j] + t;
    dx[d] = sx[s];
    dy[d] = sy[s];
    dz[d] = sz[s];
    dq[d] = sq[s];
    dorig[d] = s_orig[s];
  }
}

__global__ void k_repack_gather_pool(int pool_used, const int* p_leaf, const int* p_orig, const double* px,
                                     const double* py, const double* pz, const double* pq, const int* dfs_of_node,
                                     const int* dense_begin, const int* old_cnt, int* fill, double* dx, double* dy,
                                     double* dz, double* dq, int* dorig) {
  // one thread: pool order is preserved within each leaf
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int p = 0; p < pool_used; ++p) {
    if (p_orig[p] < 0) continue;
    int j = dfs_of_node[p_leaf[p]];
    long d = dense_begin[j] + old_cnt[j] + fill[j]++;
    dx[d] = px[p];
    dy[d] = py[p];
    dz[d] = pz[p];
    dq[d] = pq[p];
    dorig[d] = p_orig[p];
  }
}

__global__ void k_leaf_counts_from_nodes(int nl, const int* lid, const int* leaf_count, int* cnt) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < nl) cnt[j] = leaf_count[lid[j]];
}

__global__ void k_caps_from_counts(int nl, const int* cnt, int slack, int* cap, long* src_lo, const int* dense_begin) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= nl) return;
  cap[j] = cnt[j] + slack;
  src_lo[j] = dense_begin[j];
}

__global__ void k_validate(const double* r, const double* q, long n, double L, int* bad) {
  long i = long(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  bool ok = isfinite(q[i]);
  for (int d = 0; d < 3; ++d) ok = ok && (r[3 * i + d] >= 0.0 && r[3 * i + d] < L);
  if (!ok) atomicAdd(bad, 1);
}

}  // namespace


// ---------------------------------------------------------------------------
// Tree-lifetime allocations come from the device's stream-ordered pool, kept
// cached across trees (the release threshold is raised once per device), so
// building a fresh tree per full-energy evaluation costs no driver
// allocations in steady state.
void* DmkTree::alloc(size_t bytes) {
  static bool pool_ready[64] = {false};
  int dev = 0;
  PDMK_CUDA(cudaGetDevice(&dev));
  if (dev < 64 && !pool_ready[dev]) {
    cudaMemPool_t pool;
    PDMK_CUDA(cudaDeviceGetDefaultMemPool(&pool, dev));
    uint64_t thr = ~uint64_t(0);
    PDMK_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
    pool_ready[dev] = true;
  }
  void* p = nullptr;
  if (bytes == 0) bytes = 16;
  cudaError_t e = cudaMallocAsync(&p, bytes, st_);
  if (e != cudaSuccess) throw CudaError(std::string("cudaMallocAsync: ") + cudaGetErrorString(e));
  allocs_.push_back(p);
  return p;
}

DmkTree::DmkTree(double L, int n_per_leaf, int digits, long n, const double* r, const double* q,
                 bool inputs_on_device, const TreeOptions& opt, cudaStream_t stream)
    : L_(L), n_per_leaf_(n_per_leaf), digits_(digits), N_(n), opt_(opt), st_(stream) {
  ps_ = make_prolate_setup(digits);
  try {
    build(r, q, inputs_on_device);
    build_setup();
  } catch (...) {
    cudaStreamSynchronize(st_);
    for (void* p : allocs_) cudaFreeAsync(p, st_);
    allocs_.clear();
    if (slot_block_) cudaFreeAsync(slot_block_, st_);
    slot_block_ = nullptr;
    throw;
  }
}

DmkTree::~DmkTree() {
  cudaStreamSynchronize(st_);
  if (aux_) {
    cudaStreamSynchronize(aux_);
    cudaStreamDestroy(aux_);
    cudaEventDestroy(ev_fork_);
    cudaEventDestroy(ev_join_);
  }
  for (auto& gx : mc_graph_)
    if (gx) cudaGraphExecDestroy(gx);
  for (cudaEvent_t e : graph_ev_) cudaEventDestroy(e);
  for (cudaEvent_t e : ev_pool_) cudaEventDestroy(e);
  for (auto& o : ev_open_) {
    cudaEventDestroy(o.second.first);
    cudaEventDestroy(o.second.second);
  }
  for (void* p : allocs_) cudaFreeAsync(p, st_);
  if (slot_block_) cudaFreeAsync(slot_block_, st_);
}

void DmkTree::synchronize() const { PDMK_CUDA(cudaStreamSynchronize(st_)); }

void DmkTree::build(const double* r_in, const double* q_in, bool on_device) {
  const long n = N_;
  DevTree& D = dev_;
  D.L = L_;
  D.N = int(n);
  // inputs
  double* r = nullptr;
  double* q = nullptr;
  void* tmp_in = nullptr;
  if (on_device) {
    r = const_cast<double*>(r_in);
    q = const_cast<double*>(q_in);
  } else {
    PDMK_CUDA(cudaMallocAsync(&tmp_in, size_t(4 * n) * sizeof(double), st_));
    r = static_cast<double*>(tmp_in);
    q = r + 3 * n;
    staged_h2d(r, {{r_in, size_t(3 * n) * sizeof(double)}, {q_in, size_t(n) * sizeof(double)}}, st_);
  }
  // refined cells per level (level 0: the root) and, in the last word, the
  // count of invalid device inputs; read back together after the shallow
  // refinement levels
  constexpr int kBadWord = MAX_LEVEL + 2;
  int* d_lvl;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_lvl), sizeof(int) * (kBadWord + 1), st_));
  PDMK_CUDA(cudaMemsetAsync(d_lvl, 0, sizeof(int) * (kBadWord + 1), st_));
  if (on_device) {
    // keys clamp every coordinate to the grid, so a build from invalid data
    // stays in bounds until the check below rejects it
    k_validate<<<grid_for(n), TPB, 0, st_>>>(r, q, n, L_, d_lvl + kBadWord);
    PDMK_LAUNCH_CHECK();
  }
  // keys, sort
  uint64_t* keys;
  int* ord;
  void* sort_scr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&keys), size_t(n) * sizeof(uint64_t) + 16, st_));
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&ord), size_t(n) * sizeof(int) + 16, st_));
  PDMK_CUDA(cudaMallocAsync(&sort_scr, radix_sort_scratch_bytes(std::max<long>(n, 64)), st_));
  k_keys<<<grid_for(n), TPB, 0, st_>>>(r, n, L_, keys, ord);
  PDMK_LAUNCH_CHECK();
  radix_sort_pairs(keys, ord, n, 8, sort_scr, st_);
  double *dsx, *dsy, *dsz, *dsq;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dsx), size_t(4 * n) * sizeof(double) + 64, st_));
  dsy = dsx + n;
  dsz = dsy + n;
  dsq = dsz + n;
  k_gather_sorted<<<grid_for(n), TPB, 0, st_>>>(r, q, ord, n, dsx, dsy, dsz, dsq);
  PDMK_LAUNCH_CHECK();
  if (tmp_in) PDMK_CUDA(cudaFreeAsync(tmp_in, st_));

  // count-driven refinement, level by level
  Bitmaps B{};
  std::vector<long> nwords(MAX_LEVELS);
  for (int l = 0; l < MAX_LEVELS; ++l) nwords[l] = std::max<long>(1, (1L << (3 * l)) >> 5);
  uint64_t* lists[2];
  int* d_cnt;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_cnt), 64, st_));
  long list_cap = std::max<long>(1024, 8 * (n / std::max(1, n_per_leaf_) + 64) + 4096);
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&lists[0]), size_t(list_cap) * 8, st_));
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&lists[1]), size_t(list_cap) * 8, st_));
  uint64_t zero = 0;
  put_small(lists[0], &zero, 8, st_);
  int maxref = 0;  // deepest level holding a refined cell
  {
    const int one = 1;
    put_small(d_lvl, &one, 4, st_);
    // root: refined (all nodes above level 2 are refined)
    B.bm[0] = static_cast<uint32_t*>(alloc(4));
    put_small(B.bm[0], &one, 4, st_);
    auto refine = [&](int l, unsigned grid) {
      if (l < MAX_LEVEL) {
        B.bm[l] = static_cast<uint32_t*>(alloc(size_t(nwords[l]) * 4));
        PDMK_CUDA(cudaMemsetAsync(B.bm[l], 0, size_t(nwords[l]) * 4, st_));
      }
      k_refine_level<<<grid, TPB, 0, st_>>>(keys, n, l, n_per_leaf_, lists[(l - 1) & 1], d_lvl + (l - 1), int(list_cap),
                                             l < MAX_LEVEL ? B.bm[l] : nullptr, lists[l & 1], d_lvl + l);
      PDMK_LAUNCH_CHECK();
    };
    // the shallow levels (bitmaps of at most 32 KB) go back to back with one
    // read-back; deeper trees continue level by level
    constexpr int kEager = 6;
    for (int l = 1; l <= kEager; ++l) refine(l, grid_for(list_cap));
    int cnt[kBadWord + 1] = {0};
    PDMK_CUDA(cudaMemcpyAsync(cnt, d_lvl, sizeof(cnt), cudaMemcpyDeviceToHost, st_));
    PDMK_CUDA(cudaStreamSynchronize(st_));
    if (cnt[kBadWord] != 0) {
      for (void* p : {static_cast<void*>(d_lvl), static_cast<void*>(keys), static_cast<void*>(ord), sort_scr,
                      static_cast<void*>(dsx), static_cast<void*>(d_cnt), static_cast<void*>(lists[0]),
                      static_cast<void*>(lists[1])})
        PDMK_CUDA(cudaFreeAsync(p, st_));
      throw BadInput("positions must lie in [0, L) and charges be finite");
    }
    for (int l = 1; l <= kEager; ++l) {
      if (long(cnt[l - 1]) * 8 > list_cap || cnt[l] > list_cap)
        throw std::runtime_error("tree build: refinement list overflow");
      if (cnt[l] == 0) break;
      maxref = l;
    }
    for (int l = kEager + 1; maxref == l - 1 && l <= MAX_LEVEL; ++l) {
      const long ncand = long(cnt[l - 1]) * 8;
      if (ncand > list_cap) throw std::runtime_error("tree build: refinement list overflow");
      refine(l, grid_for(ncand));
      PDMK_CUDA(cudaMemcpyAsync(cnt + l, d_lvl + l, 4, cudaMemcpyDeviceToHost, st_));
      PDMK_CUDA(cudaStreamSynchronize(st_));
      if (cnt[l] > list_cap) throw std::runtime_error("tree build: refinement list overflow");
      if (cnt[l] > 0) maxref = l;
    }
    PDMK_CUDA(cudaFreeAsync(d_lvl, st_));
  }
  // 2:1 balance, deepest refined level first
  for (int k = maxref; k >= 2; --k) {
    const long cells = 1L << (3 * k);
    const int fan = cells * 26 <= kBalanceFanThreads ? 26 : 1;
    k_balance_level<<<grid_for(cells * fan), TPB, 0, st_>>>(B, k, fan);
    PDMK_LAUNCH_CHECK();
  }
  // ranks of refined cells
  std::vector<int> refined(maxref + 1, 0);
  for (int l = 0; l <= maxref; ++l) {
    B.wprefix[l] = static_cast<int*>(alloc(size_t(nwords[l]) * 4));
    k_word_popc<<<grid_for(nwords[l]), TPB, 0, st_>>>(B.bm[l], nwords[l], B.wprefix[l]);
    PDMK_LAUNCH_CHECK();
    void* scr;
    PDMK_CUDA(cudaMallocAsync(&scr, scan_scratch_bytes(nwords[l]), st_));
    exclusive_scan(B.wprefix[l], B.wprefix[l], nwords[l], scr, st_);
    PDMK_CUDA(cudaFreeAsync(scr, st_));
    k_level_total<<<1, 1, 0, st_>>>(B.bm[l], B.wprefix[l], nwords[l], d_cnt + l);
    PDMK_LAUNCH_CHECK();
  }
  PDMK_CUDA(cudaMemcpyAsync(refined.data(), d_cnt, sizeof(int) * (maxref + 1), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  // levels: 0..maxref+1
  const int nlev = maxref + 2;
  D.max_depth = nlev;
  h_level_start_.assign(nlev + 1, 0);
  h_level_start_[0] = 0;
  h_level_start_[1] = 1;
  for (int l = 1; l < nlev; ++l) h_level_start_[l + 1] = h_level_start_[l] + 8 * refined[l - 1];
  const int n_nodes = h_level_start_[nlev];
  D.n_nodes = n_nodes;
  for (int l = 0; l <= nlev && l < MAX_LEVELS + 2; ++l) D.level_start[l] = h_level_start_[l];
  int* d_level_start = static_cast<int*>(alloc(sizeof(int) * (nlev + 1)));
  put_small(d_level_start, h_level_start_.data(), sizeof(int) * (nlev + 1), st_);
  D.boxsize[0] = L_;
  for (int l = 1; l < MAX_LEVELS + 2; ++l) D.boxsize[l] = 0.5 * D.boxsize[l - 1];
  double* d_boxsize = static_cast<double*>(alloc(sizeof(double) * (MAX_LEVELS + 2)));
  put_small(d_boxsize, D.boxsize, sizeof(double) * (MAX_LEVELS + 2), st_);

  NodeArrays na;
  na.prefix = static_cast<uint64_t*>(alloc(sizeof(uint64_t) * n_nodes));
  na.level = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  na.parent = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  na.child0 = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  {
    uint64_t p0 = 0;
    int l0 = 0, par0 = -1, c0 = 1;
    put_small(na.prefix, &p0, 8, st_);
    put_small(na.level, &l0, 4, st_);
    put_small(na.parent, &par0, 4, st_);
    put_small(na.child0, &c0, 4, st_);
  }
  for (int l = 1; l < nlev; ++l) {
    k_enum_nodes<<<grid_for(nwords[l - 1]), TPB, 0, st_>>>(B, l, maxref, d_level_start, na);
    PDMK_LAUNCH_CHECK();
  }
  for (int l = 0; l < MAX_LEVELS; ++l) {
    D.bm[l] = l <= maxref ? B.bm[l] : nullptr;
    D.wprefix[l] = l <= maxref ? B.wprefix[l] : nullptr;
  }
  D.maxref = maxref;
  D.level_start_d = d_level_start;
  {
    const void* ptrs[2 * MAX_LEVELS];
    for (int l = 0; l < MAX_LEVELS; ++l) {
      ptrs[l] = D.bm[l];
      ptrs[MAX_LEVELS + l] = D.wprefix[l];
    }
    void** d_ptrs = static_cast<void**>(alloc(sizeof(ptrs)));
    put_small(d_ptrs, ptrs, sizeof(ptrs), st_);
    D.bm_d = reinterpret_cast<const uint32_t* const*>(d_ptrs);
    D.wprefix_d = reinterpret_cast<const int* const*>(d_ptrs + MAX_LEVELS);
  }
  D.node_prefix = na.prefix;
  D.node_level = na.level;
  D.node_parent = na.parent;
  D.node_child0 = na.child0;

  // neighbour lists for levels >= 2 (levels 0-1 keep -1)
  D.col27 = static_cast<int*>(alloc(sizeof(int) * 27 * size_t(n_nodes)));
  D.coarse8 = static_cast<int*>(alloc(sizeof(int) * 8 * size_t(n_nodes)));
  PDMK_CUDA(cudaMemsetAsync(D.col27, 0xff, sizeof(int) * 27 * size_t(n_nodes), st_));
  PDMK_CUDA(cudaMemsetAsync(D.coarse8, 0xff, sizeof(int) * 8 * size_t(n_nodes), st_));
  {
    int lo_node = h_level_start_[2];
    k_neighbors<<<grid_for(n_nodes - lo_node), TPB, 0, st_>>>(B, d_level_start, n_nodes, lo_node, L_, d_boxsize,
                                                             na.prefix, na.level, na.parent, na.child0, D.col27,
                                                             D.coarse8);
    PDMK_LAUNCH_CHECK();
  }

  // sorted ranges, leaves in depth-first order, slotted layout
  long *node_lo, *node_hi;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&node_lo), sizeof(long) * 2 * size_t(n_nodes), st_));
  node_hi = node_lo + n_nodes;
  k_node_ranges<<<grid_for(n_nodes), TPB, 0, st_>>>(keys, n, n_nodes, na.prefix, na.level, node_lo, node_hi);
  PDMK_LAUNCH_CHECK();
  uint64_t* lkey;
  int* lid;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&lkey), sizeof(uint64_t) * n_nodes + 16, st_));
  lid = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  PDMK_CUDA(cudaMemsetAsync(d_cnt, 0, 4, st_));
  k_collect_leaves<<<grid_for(n_nodes), TPB, 0, st_>>>(n_nodes, na.prefix, na.level, na.child0, lkey, lid, d_cnt);
  PDMK_LAUNCH_CHECK();
  // leaves = nodes less refined cells (the root and every refined cell of
  // levels 1..maxref is exactly one non-leaf node), known without a read-back
  int nl = n_nodes;
  for (int l = 0; l <= maxref; ++l) nl -= refined[l];
  {
    void* scr;
    PDMK_CUDA(cudaMallocAsync(&scr, radix_sort_scratch_bytes(std::max(nl, 64)), st_));
    radix_sort_pairs(lkey, lid, nl, 8, scr, st_);
    PDMK_CUDA(cudaFreeAsync(scr, st_));
  }
  int* cnt = static_cast<int*>(alloc(sizeof(int) * nl));
  int* cap = static_cast<int*>(alloc(sizeof(int) * nl));
  long* src_lo;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&src_lo), sizeof(long) * nl + 16, st_));
  k_leaf_caps<<<grid_for(nl), TPB, 0, st_>>>(nl, lid, node_lo, node_hi, opt_.leaf_slack, cnt, cap, src_lo);
  PDMK_LAUNCH_CHECK();
  D.node_begin = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  D.node_end = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  D.leaf_count = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  D.node_count = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  D.orig_slot = static_cast<int*>(alloc(sizeof(int) * std::max<long>(n, 1)));
  // persistent per-leaf arrays kept for repacking
  leaf_dev_.lid = lid;
  leaf_dev_.cnt = cnt;
  leaf_dev_.cap = cap;
  leaf_dev_.n = nl;
  leaf_dev_.dfs_of_node = static_cast<int*>(alloc(sizeof(int) * n_nodes));
  leaf_dev_.begin = static_cast<int*>(alloc(sizeof(int) * nl));
  leaf_dev_.cnt_prefix = static_cast<int*>(alloc(sizeof(int) * nl));
  k_leaf_dfs_index<<<grid_for(nl), TPB, 0, st_>>>(nl, lid, leaf_dev_.dfs_of_node);
  PDMK_LAUNCH_CHECK();
  layout_slots(dsx, dsy, dsz, dsq, ord, src_lo, opt_.leaf_slack);
  PDMK_CUDA(cudaFreeAsync(src_lo, st_));
  PDMK_CUDA(cudaFreeAsync(lkey, st_));
  PDMK_CUDA(cudaFreeAsync(node_lo, st_));
  PDMK_CUDA(cudaFreeAsync(dsx, st_));
  PDMK_CUDA(cudaFreeAsync(sort_scr, st_));
  PDMK_CUDA(cudaFreeAsync(ord, st_));
  PDMK_CUDA(cudaFreeAsync(keys, st_));
  PDMK_CUDA(cudaFreeAsync(lists[0], st_));
  PDMK_CUDA(cudaFreeAsync(lists[1], st_));
  PDMK_CUDA(cudaFreeAsync(d_cnt, st_));
  // the refinement bitmaps are no longer needed; they stay in allocs_ (small)
  // overflow pool
  D.pool_cap = opt_.pool_capacity;
  D.px = static_cast<double*>(alloc(sizeof(double) * 4 * size_t(D.pool_cap)));
  D.py = D.px + D.pool_cap;
  D.pz = D.py + D.pool_cap;
  D.pq = D.pz + D.pool_cap;
  D.p_orig = static_cast<int*>(alloc(sizeof(int) * 2 * size_t(D.pool_cap)));
  D.p_leaf = D.p_orig + D.pool_cap;
  D.pool_n = static_cast<int*>(alloc(64));
  D.err = D.pool_n + 1;
  D.work = reinterpret_cast<unsigned long long*>(D.pool_n + 4);
  PDMK_CUDA(cudaMemsetAsync(D.pool_n, 0, 64, st_));
  // no synchronisation: the inputs were consumed before the refinement
  // loop's first read-back, and everything after is stream-ordered
}

// Lay the particles of each DFS leaf j (dense source rows [src_lo[j],
// src_lo[j] + cnt[j])) into slots with `slack` free slots after each leaf.
void DmkTree::layout_slots(const double* dsx, const double* dsy, const double* dsz, const double* dsq,
                           const int* dorig, const long* src_lo, int leaf_slack) {
  DevTree& D = dev_;
  const int nl = leaf_dev_.n;
  int* begin = leaf_dev_.begin;
  // cap = cnt + slack, begin = exclusive scan of cap, cnt_prefix = scan of cnt
  {
    void* scr;
    PDMK_CUDA(cudaMallocAsync(&scr, scan_scratch_bytes(nl), st_));
    exclusive_scan(leaf_dev_.cap, begin, nl, scr, st_);
    exclusive_scan(leaf_dev_.cnt, leaf_dev_.cnt_prefix, nl, scr, st_);
    PDMK_CUDA(cudaFreeAsync(scr, st_));
  }
  // every particle sits in exactly one leaf and cap = cnt + slack, so the
  // slots total N + nl * slack without a look at the device
  const long n_slots_l = N_ + long(nl) * leaf_slack;
  if (n_slots_l > std::numeric_limits<int>::max()) throw std::runtime_error("tree build: too many slots");
  const int n_slots = int(n_slots_l);
  // captured graphs hold the tree description by value: rebuild them later
  for (auto& gx : mc_graph_)
    if (gx) {
      PDMK_CUDA(cudaGraphExecDestroy(gx));
      gx = nullptr;
    }
  if (n_slots > slot_capacity_) {
    // slot arrays live outside allocs_ so they can be regrown
    if (slot_block_) cudaFreeAsync(slot_block_, st_);
    // a multiple of 32 slots: the mixed pass reads the four slot arrays as
    // one 2-D tensor (TMA row strides must be multiples of 16 bytes)
    slot_capacity_ = (n_slots + n_slots / 8 + 64 + 31) & ~31;
    PDMK_CUDA(cudaMallocAsync(&slot_block_, size_t(slot_capacity_) * (4 * sizeof(double) + sizeof(int)), st_));
  }
  double* base = static_cast<double*>(slot_block_);
  D.sx = base;
  D.sy = base + slot_capacity_;
  D.sz = base + 2L * slot_capacity_;
  D.sq = base + 3L * slot_capacity_;
  D.s_orig = reinterpret_cast<int*>(base + 4L * slot_capacity_);
  D.n_slots = n_slots;
  k_fill_slots<<<grid_for(n_slots), TPB, 0, st_>>>(n_slots, nl, begin, leaf_dev_.cnt, src_lo, leaf_dev_.lid,
                                                  D.node_prefix, D.node_level, L_, dsx, dsy, dsz, dsq, dorig, D.sx,
                                                  D.sy, D.sz, D.sq, D.s_orig, D.orig_slot);
  PDMK_LAUNCH_CHECK();
  k_node_slots<<<grid_for(D.n_nodes), TPB, 0, st_>>>(D.n_nodes, D.node_child0, leaf_dev_.dfs_of_node, begin,
                                                    leaf_dev_.cap, leaf_dev_.cnt, leaf_dev_.cnt_prefix, D.node_begin,
                                                    D.node_end, D.leaf_count, D.node_count);
  PDMK_LAUNCH_CHECK();
}

void DmkTree::repack(int leaf_slack) {
  DevTree& D = dev_;
  int pool_used = 0;
  PDMK_CUDA(cudaMemcpyAsync(&pool_used, D.pool_n, 4, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  const int nl = leaf_dev_.n;
  int* old_cnt = static_cast<int*>(nullptr);
  int *cnt2, *dense_begin, *fill;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&old_cnt), sizeof(int) * 4 * size_t(nl) + 64, st_));
  cnt2 = old_cnt + nl;
  dense_begin = cnt2 + nl;
  fill = dense_begin + nl;
  k_leaf_counts_from_nodes<<<grid_for(nl), TPB, 0, st_>>>(nl, leaf_dev_.lid, D.leaf_count, old_cnt);
  PDMK_LAUNCH_CHECK();
  PDMK_CUDA(cudaMemcpyAsync(cnt2, old_cnt, sizeof(int) * nl, cudaMemcpyDeviceToDevice, st_));
  if (pool_used > 0) {
    k_repack_counts<<<grid_for(pool_used), TPB, 0, st_>>>(pool_used, D.p_leaf, D.p_orig, leaf_dev_.dfs_of_node, cnt2);
    PDMK_LAUNCH_CHECK();
  }
  {
    void* scr;
    PDMK_CUDA(cudaMallocAsync(&scr, scan_scratch_bytes(nl), st_));
    exclusive_scan(cnt2, dense_begin, nl, scr, st_);
    PDMK_CUDA(cudaFreeAsync(scr, st_));
  }
  const long n = N_;
  double* dense;
  int* dorig;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dense), sizeof(double) * 4 * size_t(n) + 64, st_));
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&dorig), sizeof(int) * size_t(n) + 64, st_));
  k_repack_gather_slots<<<unsigned(std::max(nl, 1)), 128, 0, st_>>>(nl, leaf_dev_.lid, D.node_begin, D.leaf_count,
                                                                   dense_begin, D.sx, D.sy, D.sz, D.sq, D.s_orig,
                                                                   dense, dense + n, dense + 2 * n, dense + 3 * n, dorig);
  PDMK_LAUNCH_CHECK();
  if (pool_used > 0) {
    PDMK_CUDA(cudaMemsetAsync(fill, 0, sizeof(int) * nl, st_));
    k_repack_gather_pool<<<1, 1, 0, st_>>>(pool_used, D.p_leaf, D.p_orig, D.px, D.py, D.pz, D.pq,
                                          leaf_dev_.dfs_of_node, dense_begin, old_cnt, fill, dense, dense + n,
                                          dense + 2 * n, dense + 3 * n, dorig);
    PDMK_LAUNCH_CHECK();
  }
  PDMK_CUDA(cudaMemcpyAsync(leaf_dev_.cnt, cnt2, sizeof(int) * nl, cudaMemcpyDeviceToDevice, st_));
  long* src_lo;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&src_lo), sizeof(long) * size_t(nl) + 16, st_));
  k_caps_from_counts<<<grid_for(nl), TPB, 0, st_>>>(nl, cnt2, leaf_slack, leaf_dev_.cap, src_lo, dense_begin);
  PDMK_LAUNCH_CHECK();
  layout_slots(dense, dense + n, dense + 2 * n, dense + 3 * n, dorig, src_lo, leaf_slack);
  PDMK_CUDA(cudaMemsetAsync(D.pool_n, 0, 4, st_));
  PDMK_CUDA(cudaFreeAsync(src_lo, st_));
  PDMK_CUDA(cudaFreeAsync(dense, st_));
  PDMK_CUDA(cudaFreeAsync(dorig, st_));
  PDMK_CUDA(cudaFreeAsync(old_cnt, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
}

// ---------------------------------------------------------------------------
namespace {

// Window table W (window_matrix, include/kernels.hpp:60-86) and the level-2
// difference table D2 (difference_matrix, include/kernels.hpp:88-114; every
// other level is D2 scaled by 4^-(l-2), since k sigma_l is level-free).
//
// An entry depends on its mode only through m = ix^2 + iy^2 + iz^2 (in units
// of dk), and the transform arguments |k| sigma = sqrt(m) dk sigma do not
// depend on L: dk sigma is pi / (2c) for the window (dk = 2 pi / L, sigma_2 =
// L / 4c) and 2 pi / 3c, pi / 3c for the two difference terms (dk = 8 pi / 3L,
// sigma_2, sigma_3 = L / 8c). So the psi_0 transforms, the costly part, are
// evaluated once per digits setting and m; a table is those values over
// k^2 = kx^2 + ky^2 + kz^2 of its L. Whole tables are also kept per
// (digits, L) in pinned host memory (each tree's copy to the device is then
// asynchronous and never reads freed memory); past kMaxCached pairs (a run
// over many box sizes) they go to the caller's pageable `own` vector, whose
// copies are staged before cudaMemcpyAsync returns. Both routes give the same
// values.
struct KernelTables {
  const double* W = nullptr;
  const double* D2 = nullptr;
};

struct ModeTransforms {
  std::vector<double> w;  // F(sqrt(m) pi / 2c), m = 0 .. 3 nw^2
  std::vector<double> d;  // F(sqrt(m) pi / 3c) - F(sqrt(m) 2 pi / 3c), m = 0 .. 3 nd^2
};

KernelTables kernel_tables(const ProlateSetup& s, double L, std::vector<double>& own) {
  constexpr size_t kMaxCached = 32;
  constexpr double pi = 3.14159265358979323846;
  static std::mutex mu;
  static std::map<int, ModeTransforms> transforms;
  static std::map<std::pair<int, uint64_t>, KernelTables> cache;
  uint64_t lbits;
  std::memcpy(&lbits, &L, 8);
  std::lock_guard<std::mutex> g(mu);
  auto key = std::make_pair(s.digits, lbits);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  const int nw = s.n_window, dw = 2 * nw + 1, nd = s.n_diff, dd = 2 * nd + 1;
  auto ft = transforms.find(s.digits);
  if (ft == transforms.end()) {
    ModeTransforms t;
    t.w.resize(3 * nw * nw + 1);
    t.d.resize(3 * nd * nd + 1);
    for (size_t m = 1; m < t.w.size(); ++m) t.w[m] = s.fourier(std::sqrt(double(m)) * (pi / (2 * s.c)));
    for (size_t m = 1; m < t.d.size(); ++m) {
      const double r = std::sqrt(double(m));
      t.d[m] = s.fourier(r * (pi / (3 * s.c))) - s.fourier(r * (2 * pi / (3 * s.c)));
    }
    ft = transforms.emplace(s.digits, std::move(t)).first;
  }
  const ModeTransforms& F = ft->second;
  const size_t hw = size_t(dw) * dw * (nw + 1), hd = size_t(dd) * dd * (nd + 1);
  double* W;
  const bool cached = cache.size() < kMaxCached;
  if (cached) {
    PDMK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&W), sizeof(double) * (hw + hd)));
  } else {
    own.resize(hw + hd);
    W = own.data();
  }
  double* D2 = W + hw;
  {
    const double dk = 2 * pi / L;
    for (int k = 0; k < nw + 1; ++k)
      for (int j = 0; j < dw; ++j)
        for (int i = 0; i < dw; ++i) {
          const int m = (i - nw) * (i - nw) + (j - nw) * (j - nw) + (k - nw) * (k - nw);
          const double kx = (i - nw) * dk, ky = (j - nw) * dk, kz = (k - nw) * dk;
          const double k2 = kx * kx + ky * ky + kz * kz;
          const double v = m != 0 ? F.w[m] / k2 : 0.0;
          W[(k * dw + j) * dw + i] = (k == nw) ? v : 2 * v;
        }
  }
  {
    const double dk = (2 * pi / 3) / (0.25 * L), sl = 0.25 * L / s.c, slp1 = 0.5 * sl;
    for (int k = 0; k < nd + 1; ++k)
      for (int j = 0; j < dd; ++j)
        for (int i = 0; i < dd; ++i) {
          const int m = (i - nd) * (i - nd) + (j - nd) * (j - nd) + (k - nd) * (k - nd);
          const double kx = (i - nd) * dk, ky = (j - nd) * dk, kz = (k - nd) * dk;
          const double k2 = kx * kx + ky * ky + kz * kz;
          const double v = m != 0 ? F.d[m] / k2 : s.diff0 * (slp1 * slp1 - sl * sl);
          D2[(k * dd + j) * dd + i] = (k == nd) ? v : 2 * v;
        }
  }
  KernelTables t{W, D2};
  if (cached) cache.emplace(key, t);
  return t;
}

}  // namespace

void DmkTree::build_setup() {
  DevTree& D = dev_;
  const ProlateSetup& s = ps_;
  D.n_window = s.n_window;
  D.n_diff = s.n_diff;
  D.dw = 2 * s.n_window + 1;
  D.dd = 2 * s.n_diff + 1;
  D.Hw = D.dw * D.dw * (s.n_window + 1);
  D.H = D.dd * D.dd * (s.n_diff + 1);
  D.n_poly = int(s.poly.size());
  for (int i = 0; i < MAX_POLY; ++i) D.poly[i] = i < D.n_poly ? s.poly[i] : 0.0;
  const double pi = 3.14159265358979323846;
  // form_wavenumbers (src/tree.cpp:46-68)
  D.delta_k[0] = D.delta_k[1] = 2 * pi / L_;
  for (int l = 2; l < MAX_LEVELS + 2; ++l) D.delta_k[l] = (2.0 * pi / 3.0) / D.boxsize[l];
  for (int l = 0; l < MAX_LEVELS + 2; ++l) D.dscale[l] = l >= 2 ? std::ldexp(1.0, -2 * (l - 2)) : 0.0;
  D.pw_lo = 2;
  D.pw_hi = D.max_depth - 2;  // may be < pw_lo: no difference levels
  D.pw_base = D.level_start[D.pw_lo];
  // window and difference tables, shared by every tree of this (digits, L)
  std::vector<double> own;
  const KernelTables kt = kernel_tables(s, L_, own);
  D.W = static_cast<double*>(alloc(sizeof(double) * D.Hw));
  D.D2 = static_cast<double*>(alloc(sizeof(double) * D.H));
  PDMK_CUDA(cudaMemcpyAsync(D.W, kt.W, sizeof(double) * D.Hw, cudaMemcpyHostToDevice, st_));
  PDMK_CUDA(cudaMemcpyAsync(D.D2, kt.D2, sizeof(double) * D.H, cudaMemcpyHostToDevice, st_));
  // expansions (src/tree.cpp:414-443)
  D.out_root = static_cast<double2*>(alloc(sizeof(double2) * D.Hw));
  PDMK_CUDA(cudaMemsetAsync(D.out_root, 0, sizeof(double2) * D.Hw, st_));
  long n_pw = 0;
  if (D.pw_hi >= D.pw_lo) n_pw = long(D.level_start[D.pw_hi + 1]) - D.level_start[D.pw_lo];
  D.out = static_cast<double2*>(alloc(sizeof(double2) * size_t(std::max<long>(n_pw, 1)) * D.H));
  D.inc = static_cast<double2*>(alloc(sizeof(double2) * size_t(std::max<long>(n_pw, 1)) * D.H));
  PDMK_CUDA(cudaMemsetAsync(D.out, 0, sizeof(double2) * size_t(std::max<long>(n_pw, 1)) * D.H, st_));
  PDMK_CUDA(cudaMemsetAsync(D.inc, 0, sizeof(double2) * size_t(std::max<long>(n_pw, 1)) * D.H, st_));
  // scratch for partial sums and the proposal record
  partials_cap_ = partials_needed();
  D.partials = static_cast<double*>(alloc(sizeof(double) * partials_cap_));
  D.counter = static_cast<unsigned int*>(alloc(64));
  PDMK_CUDA(cudaMemsetAsync(D.counter, 0, 64, st_));
  D.prop = static_cast<Proposal*>(alloc(sizeof(Proposal)));
  PDMK_CUDA(cudaMemsetAsync(D.prop, 0, sizeof(Proposal), st_));
  D.recv = static_cast<Receiver*>(alloc(sizeof(Receiver) * MAX_RECV));
  d_one_idx_ = static_cast<int*>(alloc(64));
  d_one_disp_ = static_cast<double*>(alloc(64));
  d_one_u_ = static_cast<double*>(alloc(64));
}

int DmkTree::check_device_error() const {
  int e[2] = {0, 0};
  PDMK_CUDA(cudaMemcpyAsync(e, dev_.pool_n, 8, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  return e[1];
}

// ---------------------------------------------------------------------------
// exports for tests
void DmkTree::export_nodes(int* level, uint64_t* prefix, int* is_leaf, long* count) const {
  const int nn = dev_.n_nodes;
  std::vector<int> c0(nn), cnt(nn);
  PDMK_CUDA(cudaMemcpyAsync(level, dev_.node_level, sizeof(int) * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(prefix, dev_.node_prefix, sizeof(uint64_t) * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(c0.data(), dev_.node_child0, sizeof(int) * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(cnt.data(), dev_.node_count, sizeof(int) * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  for (int i = 0; i < nn; ++i) {
    is_leaf[i] = c0[i] < 0;
    count[i] = cnt[i];
  }
}

void DmkTree::export_neighbors(int* col27, int* coarse8) const {
  const size_t nn = size_t(dev_.n_nodes);
  PDMK_CUDA(cudaMemcpyAsync(col27, dev_.col27, sizeof(int) * 27 * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(coarse8, dev_.coarse8, sizeof(int) * 8 * nn, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
}

void DmkTree::export_sorted_order(long* out) const {
  std::vector<int> so(dev_.n_slots);
  PDMK_CUDA(cudaMemcpyAsync(so.data(), dev_.s_orig, sizeof(int) * dev_.n_slots, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  long k = 0;
  for (int s = 0; s < dev_.n_slots; ++s)
    if (so[s] >= 0) out[k++] = so[s];
}

namespace {
// positions (xyz-interleaved) and charges in the caller's original order,
// from the slots and the overflow pool
__global__ void k_gather_orig(int n, const int* orig_slot, int n_slots, const double* sx, const double* sy,
                              const double* sz, const double* sq, const double* px, const double* py,
                              const double* pz, const double* pq, double* r, double* q) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int s = orig_slot[i];
  if (s < n_slots) {
    r[3 * i] = sx[s];
    r[3 * i + 1] = sy[s];
    r[3 * i + 2] = sz[s];
    q[i] = sq[s];
  } else {
    const int p = s - n_slots;
    r[3 * i] = px[p];
    r[3 * i + 1] = py[p];
    r[3 * i + 2] = pz[p];
    q[i] = pq[p];
  }
}
}  // namespace

namespace {
// out[0] = max count over leaves, out[1] = min count over refined nodes of
// levels >= 3 (refinement above is forced)
__global__ void k_drift(const int* __restrict__ count, const int* __restrict__ child0, const int* __restrict__ level,
                        int n_nodes, int* out) {
  int mx = 0, mn = 0x7fffffff;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n_nodes; i += gridDim.x * blockDim.x) {
    const int c = count[i];
    if (child0[i] < 0) mx = max(mx, c);
    else if (level[i] >= 3) mn = min(mn, c);
  }
  for (int o = 16; o > 0; o >>= 1) {
    mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    mn = min(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(out, mx);
    atomicMin(out + 1, mn);
  }
}
}  // namespace

void DmkTree::drift(int* max_leaf, int* min_refined) const {
  const DevTree& D = dev_;
  int* d_out = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_out), 2 * sizeof(int), st_));
  const int init[2] = {0, int(N_)};
  PDMK_CUDA(cudaMemcpyAsync(d_out, init, sizeof(init), cudaMemcpyHostToDevice, st_));
  const int blocks = std::max(1, std::min(592, (D.n_nodes + 255) / 256));
  k_drift<<<unsigned(blocks), 256, 0, st_>>>(D.node_count, D.node_child0, D.node_level, D.n_nodes, d_out);
  PDMK_LAUNCH_CHECK();
  int out[2];
  PDMK_CUDA(cudaMemcpyAsync(out, d_out, sizeof(out), cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaFreeAsync(d_out, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  *max_leaf = out[0];
  *min_refined = out[1];
}

void DmkTree::gather_device(double* d_r, double* d_q) const {
  const DevTree& D = dev_;
  const int n = int(N_);
  k_gather_orig<<<unsigned((n + 255) / 256), 256, 0, st_>>>(n, D.orig_slot, D.n_slots, D.sx, D.sy, D.sz, D.sq, D.px,
                                                            D.py, D.pz, D.pq, d_r, d_q);
  PDMK_LAUNCH_CHECK();
}

void DmkTree::export_positions(double* r) const {
  const int ns = dev_.n_slots;
  std::vector<double> x(ns), y(ns), z(ns);
  std::vector<int> so(ns);
  PDMK_CUDA(cudaMemcpyAsync(x.data(), dev_.sx, sizeof(double) * ns, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(y.data(), dev_.sy, sizeof(double) * ns, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(z.data(), dev_.sz, sizeof(double) * ns, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaMemcpyAsync(so.data(), dev_.s_orig, sizeof(int) * ns, cudaMemcpyDeviceToHost, st_));
  int pn = 0;
  PDMK_CUDA(cudaMemcpyAsync(&pn, dev_.pool_n, 4, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  for (int s = 0; s < ns; ++s)
    if (so[s] >= 0) {
      r[3 * so[s]] = x[s];
      r[3 * so[s] + 1] = y[s];
      r[3 * so[s] + 2] = z[s];
    }
  if (pn > 0) {
    std::vector<double> px(pn), py(pn), pz(pn);
    std::vector<int> po(pn);
    PDMK_CUDA(cudaMemcpyAsync(px.data(), dev_.px, sizeof(double) * pn, cudaMemcpyDeviceToHost, st_));
    PDMK_CUDA(cudaMemcpyAsync(py.data(), dev_.py, sizeof(double) * pn, cudaMemcpyDeviceToHost, st_));
    PDMK_CUDA(cudaMemcpyAsync(pz.data(), dev_.pz, sizeof(double) * pn, cudaMemcpyDeviceToHost, st_));
    PDMK_CUDA(cudaMemcpyAsync(po.data(), dev_.p_orig, sizeof(int) * pn, cudaMemcpyDeviceToHost, st_));
    PDMK_CUDA(cudaStreamSynchronize(st_));
    for (int p = 0; p < pn; ++p)
      if (po[p] >= 0) {
        r[3 * po[p]] = px[p];
        r[3 * po[p] + 1] = py[p];
        r[3 * po[p] + 2] = pz[p];
      }
  }
}

void DmkTree::export_pw(long node, int which, double* out) const {
  if (node == 0) {
    if (which != 0) throw std::invalid_argument("the root has no incoming expansion");
    PDMK_CUDA(cudaMemcpyAsync(out, dev_.out_root, sizeof(double2) * dev_.Hw, cudaMemcpyDeviceToHost, st_));
  } else {
    long lo = dev_.level_start[dev_.pw_lo];
    long hi = dev_.pw_hi >= dev_.pw_lo ? dev_.level_start[dev_.pw_hi + 1] : lo;
    if (node < lo || node >= hi) throw std::invalid_argument("node carries no expansion");
    const double2* src = (which == 0 ? dev_.out : dev_.inc) + size_t(node - lo) * dev_.H;
    PDMK_CUDA(cudaMemcpyAsync(out, src, sizeof(double2) * dev_.H, cudaMemcpyDeviceToHost, st_));
  }
  PDMK_CUDA(cudaStreamSynchronize(st_));
}

void DmkTree::export_W(double* out) const {
  PDMK_CUDA(cudaMemcpyAsync(out, dev_.W, sizeof(double) * dev_.Hw, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
}

void DmkTree::export_D(int level, double* out) const {
  PDMK_CUDA(cudaMemcpyAsync(out, dev_.D2, sizeof(double) * dev_.H, cudaMemcpyDeviceToHost, st_));
  PDMK_CUDA(cudaStreamSynchronize(st_));
  for (int k = 0; k < dev_.H; ++k) out[k] *= dev_.dscale[level];
}

namespace {
struct Staging {
  std::mutex mu;
  char* buf = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;  // the last copy out of buf
};
Staging g_staging[64];
}  // namespace

void staged_h2d(void* dst, const std::vector<HostPiece>& pieces, cudaStream_t st) {
  size_t total = 0;
  for (const HostPiece& p : pieces) total += p.bytes;
  int dev = 0;
  PDMK_CUDA(cudaGetDevice(&dev));
  if (total < (size_t(4) << 20) || dev < 0 || dev >= 64) {
    char* d = static_cast<char*>(dst);
    for (const HostPiece& p : pieces) {
      PDMK_CUDA(cudaMemcpyAsync(d, p.src, p.bytes, cudaMemcpyHostToDevice, st));
      d += p.bytes;
    }
    return;
  }
  Staging& S = g_staging[dev];
  std::lock_guard<std::mutex> g(S.mu);
  if (S.done) PDMK_CUDA(cudaEventSynchronize(S.done));
  else PDMK_CUDA(cudaEventCreateWithFlags(&S.done, cudaEventDisableTiming));
  if (S.cap < total) {
    if (S.buf) PDMK_CUDA(cudaFreeHost(S.buf));
    S.buf = nullptr;
    S.cap = 0;
    PDMK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&S.buf), total));
    S.cap = total;
  }
  size_t off = 0;
  for (const HostPiece& p : pieces) {
    const char* src = static_cast<const char*>(p.src);
    char* stage = S.buf + off;
    parallel_chunks(long(p.bytes),
                    [&](long b, long e) { std::memcpy(stage + b, src + b, size_t(e - b)); }, 1L << 22);
    off += p.bytes;
  }
  PDMK_CUDA(cudaMemcpyAsync(dst, S.buf, total, cudaMemcpyHostToDevice, st));
  PDMK_CUDA(cudaEventRecord(S.done, st));
}

}  // namespace pdmk
