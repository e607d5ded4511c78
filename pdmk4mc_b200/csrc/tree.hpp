// The device-resident DMK tree behind the C-ABI: particles binned into a
// periodic 2:1-balanced adaptive octree, per-level plane-wave expansions, and
// the kernels that form, evaluate and update them on one B200.
//
// Reference counterpart: struct HPDMKPtTree<Real> (include/tree.hpp:29-132)
// and its methods in src/tree.cpp, src/planewave.cpp, src/energy.cpp and
// src/energy_shift.cpp.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"
#include "pswf.hpp"

namespace pdmk {

constexpr int MAX_POLY = 25;
constexpr int PATH_LEN_MAX = MAX_LEVELS;

// One proposed single-particle move and what the shift kernel found for it.
struct Proposal {
  int i_orig;
  int slot;       // current slot (>= n_slots: overflow pool entry)
  double q;
  double xo[3], xt[3];
  int depth_o, depth_t;  // number of path nodes (leaf level + 1)
  int path_o[PATH_LEN_MAX], path_t[PATH_LEN_MAX];
  double dE;
  double parts[5];  // window, difference, residual(target), residual(origin), self
  int accepted;
  int valid;
  int n_recv;  // expansion vectors an accepted move updates (records in DevTree::recv)
};

// One expansion vector touched by an accepted move, with the contributions of
// the target (+) and origin (-) single-particle expansions and the periodic
// image flags of each source box as seen from the receiving box.
struct Receiver {
  int off;              // (node - first expansion node), selects out/inc row
  signed char is_out;   // 1: outgoing (no conjugate, no shift), 0: incoming
  signed char level;
  signed char has_t, has_o;
  signed char ft[3], fo[3];
  signed char pad[2];
};
constexpr int MAX_RECV = 2 * 28 * MAX_LEVELS;

// Where the captured Metropolis graph reads its proposals: set before each
// launch of the graph, so one instantiated graph serves every batch.
struct MoveCursor {
  const int* idx;
  const double* disp;
  const double* u;
  double* dE;
  int* acc;
  int off;
  int mode;
  double beta;
};

// Everything the kernels need, by value (all pointers are device pointers).
struct DevTree {
  double L;
  int N;
  int n_window, n_diff;
  int dw, dd;  // 2n+1
  int Hw, H;   // half-space sizes d^2 (n+1)
  int max_depth;  // number of levels
  int n_nodes;
  int level_start[MAX_LEVELS + 2];
  double boxsize[MAX_LEVELS + 2];
  double delta_k[MAX_LEVELS + 2];
  double dscale[MAX_LEVELS + 2];  // D_l = D_2 * dscale[l]
  int pw_lo, pw_hi;               // levels carrying expansions: [pw_lo, pw_hi]
  double poly[MAX_POLY];
  int n_poly;
  // particle slots (leaf-major in Morton order, with slack)
  int n_slots;
  double *sx, *sy, *sz, *sq;
  int* s_orig;     // original index or -1
  int* orig_slot;  // [N]; values >= n_slots are pool entries
  // overflow pool for arrivals into full leaves
  int pool_cap;
  double *px, *py, *pz, *pq;
  int *p_orig, *p_leaf;
  int* pool_n;
  // nodes (level-major, Morton order within a level)
  uint64_t* node_prefix;
  int* node_level;
  int* node_parent;
  int* node_child0;  // -1 for leaves
  int* node_begin;   // slot range of the subtree
  int* node_end;
  int* leaf_count;  // particles present in a leaf (compact from node_begin)
  int* node_count;  // particles in the subtree (maintained by moves)
  int* col27;       // [n_nodes][27], same-level neighbours, -1 absent or self
  int* coarse8;     // [n_nodes][8], coarse-grain leaf neighbours, -1 pad
  // refinement bitmaps per level and exclusive word-popcount prefixes: the
  // node id of any cell follows from these without walking the tree
  const uint32_t* bm[MAX_LEVELS];
  const int* wprefix[MAX_LEVELS];
  int maxref;  // deepest level with a refined cell
  // device copies of the per-level tables, for indexing by a run-time level
  // (indexing the by-value kernel parameter would copy it to local memory)
  const int* level_start_d;
  const uint32_t* const* bm_d;
  const int* const* wprefix_d;
  int pw_base;  // level_start[pw_lo], the first node carrying expansions
  // expansions: root, then nodes of levels [pw_lo, pw_hi] (contiguous ids)
  double2* out_root;
  double2* out;  // [(node - level_start[pw_lo]) * H + k]
  double2* inc;
  double* W;   // [Hw]
  double* D2;  // [H], the level-2 difference kernel
  // scratch
  double* partials;
  unsigned int* counter;
  Proposal* prop;
  Receiver* recv;  // [MAX_RECV]
  int* err;  // device error word (nonzero: pool overflow etc.)
  unsigned long long* work;  // [0] accepted moves, [1] update bytes (read + write), [2] dE bytes (persistent kernel)
};

// per-level geometry, computed rather than indexed: box side L 2^-l, the
// difference-level mode spacing (2 pi / 3) / bs_l (form_wavenumbers,
// src/tree.cpp:64-68) and the difference-kernel scale 4^-(l-2)
__host__ __device__ inline double level_box(const DevTree& T, int l) { return ldexp(T.L, -l); }
__host__ __device__ inline double level_dk(const DevTree& T, int l) {
  return (2.0 * 3.14159265358979323846 / 3.0) / ldexp(T.L, -l);
}
__host__ __device__ inline double level_dscale(int l) { return ldexp(1.0, -2 * (l - 2)); }

// The residual polynomial with its coefficients in registers (include/pswf.hpp:70-78
// and include/kernels.hpp:50-58): res(r; b) = P(2 r / b - 1) / r, zero outside (0, b).
template <int NP>
struct ResidualPoly {
  double c[NP];
  __device__ explicit ResidualPoly(const DevTree& T) {
#pragma unroll
    for (int i = 0; i < NP; ++i) c[i] = T.poly[i];
  }
  __device__ double operator()(double r, double b) const {
    const double xs = (r / b - 0.5) * 2.0;
    if (fabs(xs) >= 1.0) return 0.0;
    double v = 0;
#pragma unroll
    for (int i = 0; i < NP; ++i) v = fma(v, xs, c[i]);
    return v / r;
  }
  // the same kernel from r^2 with one reciprocal square root in place of a
  // square root and two divisions (inv_b = 1 / b); zero at r = 0 as above
  __device__ double from_r2(double r2, double inv_b) const {
    if (!(r2 > 0.0)) return 0.0;
    const double ri = rsqrt(r2);
    const double xs = (r2 * ri * inv_b - 0.5) * 2.0;
    if (fabs(xs) >= 1.0) return 0.0;
    double v = 0;
#pragma unroll
    for (int i = 0; i < NP; ++i) v = fma(v, xs, c[i]);
    return v * ri;
  }
  // d/dr of the residual kernel, P'(x) (2 / b) / r - P(x) / r^2 with x = 2 r / b - 1
  __device__ double deriv(double r, double b) const {
    const double xs = (r / b - 0.5) * 2.0;
    if (fabs(xs) >= 1.0) return 0.0;
    double v = 0, dv = 0;
#pragma unroll
    for (int i = 0; i < NP; ++i) {
      dv = fma(dv, xs, v);
      v = fma(v, xs, c[i]);
    }
    return (dv * (2.0 / b) - v / r) / r;
  }
};

struct EnergyParts {
  double window = 0, diff = 0, res = 0;
  double total() const { return window + diff + res; }
};


// Run-time split and tile choices of the energy pipeline, picked per digits
// setting, precision and size by the autotuner (tune.cpp) and cached in a
// JSON table that trees read at construction.
struct Tuning {
  int ksplit = 4096;       // particles per split-K chunk of a box in the outgoing pass
  int ksplit_root = 2048;  // particles per chunk of the root pass
  int inc_waves = 4;       // resident waves of blocks (2 per SM) in the incoming pass
  int res_ny_max = 8;      // most target chunks (64 targets each) per leaf in the near field
};

struct TreeOptions {
  int leaf_slack = 0;      // extra particle slots per leaf for moves
  int pool_capacity = 4096;
  int precision = 0;       // 0: FP64 outgoing pass; 1: int8-sliced tensor-core outgoing pass (mixed)
};

class DmkTree {
 public:
  DmkTree(double L, int n_per_leaf, int digits, long n, const double* r, const double* q, bool inputs_on_device,
          const TreeOptions& opt, cudaStream_t stream);
  ~DmkTree();
  DmkTree(const DmkTree&) = delete;
  DmkTree& operator=(const DmkTree&) = delete;

  void form_outgoing_pw();
  void form_incoming_pw();
  EnergyParts eval_energy();
  double eval_window_energy();
  double eval_diff_energy();
  double eval_res_energy();
  // FP64 Ewald energy of the current particles (comparator); parts: real, reciprocal, self
  double ewald_energy(double* parts = nullptr);
  // single move through the drop-in API: host scalars in, host scalar out
  double eval_shift_energy(long i, double dx, double dy, double dz, double* parts = nullptr);
  void update_shift(long i, double dx, double dy, double dz);
  // sequential Metropolis over device-resident proposals; no host sync
  void mc_run_device(int n_moves, const int* d_idx, const double* d_disp, const double* d_u, double beta,
                     double* d_dE, int* d_acc);
  // Metropolis sequence mode: 0 one persistent cooperative launch (default),
  // 1 CUDA graphs of kGraphMoves (shift, update) launch pairs
  void set_mc_mode(int mode) { mc_mode_ = mode; }
  // Metropolis sequences of m moves for each of many trees (same digits, same
  // device) in one launch, one block per tree; arrays hold tree t's moves at
  // [t m, (t + 1) m)
  // potential phi_i = sum_{j != i, images} q_j / r_ij and field -grad phi at
  // original particles d_idx[0..m) into d_phi[m] and d_field[3m] (may be null)
  void potential_batch(int m, const int* d_idx, double* d_phi, double* d_field);
  static void replicas_mc_run(const std::vector<DmkTree*>& trees, int m, const int* d_idx, const double* d_disp,
                              const double* d_u, double beta, double* d_dE, int* d_acc);
  int mc_mode() const { return mc_mode_; }
  // batched energy shifts of many candidates against the current state
  void shift_batch_device(int m, const int* d_idx, const double* d_disp, double* d_dE);
  // the same batch through one fixed static device buffer: no device
  // allocation in the call (host arrays in and out, synchronous)
  void shift_batch_static(int m, const long* h_idx, const double* h_disp, double* h_dE);

  // introspection (tests)
  int max_depth() const { return dev_.max_depth; }
  int n_nodes() const { return dev_.n_nodes; }
  const DevTree& dev() const { return dev_; }
  void export_nodes(int* level, uint64_t* prefix, int* is_leaf, long* count) const;
  void export_neighbors(int* col27, int* coarse8) const;
  void export_sorted_order(long* orig_of_sorted) const;
  void export_positions(double* r_orig_order) const;
  // current positions [3n] and charges [n] in original order into device buffers (stream-ordered)
  void gather_device(double* d_r, double* d_q) const;
  // the largest particle count of a leaf and the smallest of a refined node
  // below level 2 (N when there is none), from the maintained node counts
  void drift(int* max_leaf, int* min_refined) const;
  long n_particles() const { return N_; }
  int n_per_leaf() const { return n_per_leaf_; }
  int digits() const { return digits_; }
  const TreeOptions& options() const { return opt_; }
  double box() const { return L_; }
  void export_pw(long node, int which, double* out) const;
  void export_W(double* out) const;
  void export_D(int level, double* out) const;
  void synchronize() const;
  cudaStream_t stream() const { return st_; }
  int check_device_error() const;
  void repack(int leaf_slack);

 private:
  void build(const double* r, const double* q, bool on_device);
  void build_setup();
  void layout_slots(const double* dsx, const double* dsy, const double* dsz, const double* dsq, const int* dorig,
                    const long* src_lo, int leaf_slack);
  size_t partials_needed() const;
  int res_chunks() const;
  void launch_shift(const int* d_idx, const double* d_disp, const double* d_u, double beta, int move, int mode,
                    double* d_dE, int* d_acc);
  void launch_update();  // accept-and-update and membership commit, one launch
  void ensure_packed();
  void prepare_box_lists();
  void build_box_lists(const std::vector<int>& child0);  // from a host copy of node_child0
  void launch_window_energy();  // enqueue the window energy into d_scalars_[0]
  void launch_res_energy();     // enqueue the near-field energy into d_scalars_[2]
  void run_incoming(bool write_inc);

  double L_;
  int n_per_leaf_;
  int digits_;
  long N_;
  TreeOptions opt_;
  cudaStream_t st_;
  ProlateSetup ps_;
  DevTree dev_{};
  // host copies of the topology
  std::vector<int> h_level_start_;
  std::vector<void*> allocs_;
  void* alloc(size_t bytes);
  // leaves in depth-first order and their slot bookkeeping (device)
  struct LeafArrays {
    int n = 0;
    int* lid = nullptr;          // node id of the j-th leaf
    int* cnt = nullptr;          // particles at layout time
    int* cap = nullptr;          // slots
    int* begin = nullptr;        // first slot
    int* cnt_prefix = nullptr;   // exclusive prefix of cnt
    int* dfs_of_node = nullptr;  // node id -> j (leaves only)
  } leaf_dev_;
  void* slot_block_ = nullptr;
  int slot_capacity_ = 0;
  size_t partials_cap_ = 0;
  // energy bookkeeping
  bool diff_cached_ = false;
  bool moved_ = false;  // moves ran since the last pack: the overflow pool may hold particles
  bool box_lists_ready_ = false;
  int n_nonleaf_ = 0, n_leaves_ = 0;
  int* d_nonleaf_ = nullptr;  // non-leaf nodes of the expansion levels
  int* d_leaves_ = nullptr;   // leaves at levels >= 2
  int n_cubes_ = 0;
  int* d_cubes_ = nullptr;    // boxes two levels above the expansion levels with a non-leaf grandchild
  double* d_Cl_ = nullptr;
  double* d_Sl_ = nullptr;
  double* d_scalars_ = nullptr;
  // optional CUDA-event timing per kernel class (0 shift, 1 update pair, 2 commit, 3 NUDFT)
 public:
  void set_timing(bool on) { timing_ = on; }
  void get_timing(double* out, bool reset);
  void get_work(double* out);
  void reset_work();
  void time_begin(int cls);
  void time_end(int cls);

 private:
  bool timing_ = false;
  std::vector<cudaEvent_t> ev_pool_;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_open_;
  double t_ms_[4] = {0, 0, 0, 0};
  long t_cnt_[4] = {0, 0, 0, 0};
  cudaEvent_t ev_cur_[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t take_event();
  int shift_grid_ = 0;
  // captured Metropolis batches (plain, and with per-update timing events)
  static constexpr int kGraphMoves = 128;
  static constexpr int kMcChunk = 1 << 16;  // moves per persistent launch
  int mc_mode_ = 0;
  int mc_grid_ = 0;
  double* mc_partials_ = nullptr;
  unsigned int* mc_sync_ = nullptr;
  void mc_run_persistent(int n_moves, const int* d_idx, const double* d_disp, const double* d_u, double beta,
                         double* d_dE, int* d_acc);
  static constexpr int kTimedEvery = 8;
  long timed_batches_ = 0;
  cudaGraphExec_t mc_graph_[2] = {nullptr, nullptr};
  std::vector<cudaEvent_t> graph_ev_;  // [2 * kGraphMoves] start/end of each update
  MoveCursor* d_cursor_ = nullptr;
  bool capturing_ = false;
  bool use_cursor_ = false;
  void ensure_move_resources();
  void ensure_shift_config();
  void build_mc_graph(int timed);
  void launch_shift_cursor(int move);
  cudaStream_t aux_ = nullptr;  // second stream for the root plane-wave pass
  // mixed precision: [0] max |q| (fixed-point scale), [1] error word (as int) of the tensor-core pass
  double* d_mix_ = nullptr;
  bool qmax_ready_ = false;
  Tuning tune_;
 public:
  int precision() const { return opt_.precision; }
  const Tuning& tuning() const { return tune_; }
  // clamps to the supported ranges (the mixed pass's exact int32 sums bound
  // a split-K chunk to 16384 particles)
  void set_tuning(const Tuning& t);
  // times one phase of the energy pipeline (0 outgoing, 1 incoming, 2 near
  // field) `reps` times on the tree's stream; returns the median milliseconds
  double time_phase(int phase, int reps);
  // error word of the mixed pass (nonzero: a pipeline wait gave up); synchronises
  int check_mixed_error();

 private:
  cudaEvent_t ev_fork_ = nullptr, ev_join_ = nullptr;
  double2* ptab_ = nullptr;  // phase tables of the last proposal, both paths
  long ptab_per_ = 0;
  // host-side copy of the last proposal arguments (for update_shift)
  long last_i_ = -1;
  double last_d_[3] = {0, 0, 0};
  bool last_valid_ = false;
  // arguments of the single-move API in device memory
  int* d_one_idx_ = nullptr;
  double* d_one_disp_ = nullptr;
  double* d_one_u_ = nullptr;
};

}  // namespace pdmk
