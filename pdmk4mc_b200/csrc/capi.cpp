// The C-ABI boundary: plain pointers and sizes in, status codes out. Every
// exception of the C++ layer is caught here (the reference throws
// std::runtime_error / std::invalid_argument, src/tree.cpp:21-27,
// include/utils.hpp:47, src/upward_pass.cpp:13).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/hpdmk.h"
#include "hostpar.hpp"
#include "tree.hpp"

namespace pdmk {
bool read_particle_info(const std::string& filename, std::vector<double>& xyzq);
Tuning lookup_tuning(int digits, int precision, long n);
void autotune_tree(DmkTree& t, const char* path, int reps, int* out, double* times);
Tuning lookup_tuning_file(const std::string& path, int digits, int precision, long n);
}

namespace {

thread_local int g_last_error = HPDMK_OK;
thread_local std::string g_last_message;

struct Handle {
  std::unique_ptr<pdmk::DmkTree> tree;
  cudaStream_t stream = nullptr;
  bool own_stream = true;
  long n = 0;
  double L = 0;
  int device = 0;
  double rebuild_factor = 0;  // rebuild policy: 0 off, else the leaf drift factor
  int rebuilds = 0;           // rebuilds the policy made
  int base_max = 0, base_min = 0;  // the drift of the tree when the policy was set or last rebuilt
  // staging buffers for the host-array batched calls
  int* d_i = nullptr;
  double* d_d = nullptr;
  double* d_u = nullptr;
  double* d_dE = nullptr;
  int* d_acc = nullptr;
  int cap = 0;
  ~Handle() {
    tree.reset();
    if (d_i) cudaFree(d_i);
    if (d_d) cudaFree(d_d);
    if (d_u) cudaFree(d_u);
    if (d_dE) cudaFree(d_dE);
    if (d_acc) cudaFree(d_acc);
    if (stream && own_stream) cudaStreamDestroy(stream);
  }
  void ensure(int m) {
    if (m <= cap) return;
    if (d_i) cudaFree(d_i);
    if (d_d) cudaFree(d_d);
    if (d_u) cudaFree(d_u);
    if (d_dE) cudaFree(d_dE);
    if (d_acc) cudaFree(d_acc);
    d_i = nullptr;
    d_d = d_u = d_dE = nullptr;
    d_acc = nullptr;
    cap = 0;
    PDMK_CUDA(cudaMalloc(&d_i, sizeof(int) * m));
    PDMK_CUDA(cudaMalloc(&d_d, sizeof(double) * 3 * m));
    PDMK_CUDA(cudaMalloc(&d_u, sizeof(double) * m));
    PDMK_CUDA(cudaMalloc(&d_dE, sizeof(double) * m));
    PDMK_CUDA(cudaMalloc(&d_acc, sizeof(int) * m));
    cap = m;
  }
};

int fail(int code, const std::string& msg) {
  g_last_error = code;
  g_last_message = msg;
  return code;
}

int ok() {
  g_last_error = HPDMK_OK;
  g_last_message.clear();
  return HPDMK_OK;
}

template <class F>
int guarded(F&& f) {
  try {
    return f();
  } catch (const std::bad_alloc& e) {
    return fail(HPDMK_ERR_OUT_OF_MEMORY, e.what());
  } catch (const pdmk::BadInput& e) {
    return fail(HPDMK_ERR_BAD_INPUT, e.what());
  } catch (const pdmk::DeviceError& e) {
    return fail(HPDMK_ERR_DEVICE, e.what());
  } catch (const pdmk::CudaError& e) {
    std::string m = e.what();
    if (m.find("out of memory") != std::string::npos) return fail(HPDMK_ERR_OUT_OF_MEMORY, m);
    return fail(HPDMK_ERR_CUDA, m);
  } catch (const std::invalid_argument& e) {
    return fail(HPDMK_ERR_BAD_PARAMS, e.what());
  } catch (const std::exception& e) {
    return fail(HPDMK_ERR_INTERNAL, e.what());
  }
}

Handle* H(hpdmk_tree t) { return static_cast<Handle*>(t); }

// Makes the tree's device current for one call and restores the caller's
// device afterwards: every tree's stream, buffers and kernel attributes
// belong to the device it was created on.
struct DeviceGuard {
  int prev = -1, want = 0;
  explicit DeviceGuard(int dev) : want(dev) {
    PDMK_CUDA(cudaGetDevice(&prev));
    if (prev != want) PDMK_CUDA(cudaSetDevice(want));
  }
  ~DeviceGuard() {
    if (prev >= 0 && prev != want) cudaSetDevice(prev);
  }
  DeviceGuard(const DeviceGuard&) = delete;
  DeviceGuard& operator=(const DeviceGuard&) = delete;
};

// Re-bins the tree from its particles' current positions on the device: a
// fresh tree of the same parameters, settings and tuning replaces the old
// one (the expansions are not formed here).
void rebuild_structure(Handle* h) {
  const pdmk::DmkTree& old = *h->tree;
  const long n = old.n_particles();
  double* d_r = nullptr;
  PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_r), sizeof(double) * 4 * size_t(n), h->stream));
  double* d_q = d_r + 3 * n;
  old.gather_device(d_r, d_q);
  try {
    auto nt = std::make_unique<pdmk::DmkTree>(old.box(), old.n_per_leaf(), old.digits(), n, d_r, d_q, true,
                                              old.options(), h->stream);
    nt->set_mc_mode(old.mc_mode());  // the caller's settings carry over
    nt->set_tuning(old.tuning());
    h->tree = std::move(nt);
  } catch (...) {
    cudaFreeAsync(d_r, h->stream);
    throw;
  }
  PDMK_CUDA(cudaFreeAsync(d_r, h->stream));
}

// The drift of a tree as built is the policy's baseline: leaves at the level
// cap may hold more than n_per_leaf particles and nodes refined for the 2:1
// balance fewer, and neither is drift.
void record_baseline(Handle* h) { h->tree->drift(&h->base_max, &h->base_min); }

// device error word: bit 0 overflow pool exhausted, bit 1 grid barrier wait gave up
int device_fail(int e) {
  if (e & 2) return fail(HPDMK_ERR_DEVICE, "persistent Metropolis kernel: a grid barrier wait gave up");
  return fail(HPDMK_ERR_DEVICE, "overflow pool exhausted");
}

int check_params(const HPDMKParams& p) {
  if (!(p.L > 0) || !std::isfinite(p.L)) return fail(HPDMK_ERR_BAD_PARAMS, "L must be positive and finite");
  if (p.n_per_leaf < 1) return fail(HPDMK_ERR_BAD_PARAMS, "n_per_leaf must be >= 1");
  if (p.digits != 3 && p.digits != 6 && p.digits != 9 && p.digits != 12)
    return fail(HPDMK_ERR_BAD_PARAMS, "double only supports 3, 6, 9 and 12 digits accuracy");
  if (p.init != DIRECT && p.init != PROXY) return fail(HPDMK_ERR_BAD_PARAMS, "init must be DIRECT or PROXY");
  if (p.init == PROXY && p.digits > 3)
    return fail(HPDMK_ERR_BAD_PARAMS, "PROXY initialisation supports 3 digits only; use DIRECT");
  return HPDMK_OK;
}

int check_inputs(double L, int n, const double* r, const double* q) {
  if (n < 1 || !r || !q) return fail(HPDMK_ERR_BAD_INPUT, "need n >= 1 particles with positions and charges");
  // branch-free scans over pieces of the arrays, on a few threads
  std::atomic<int> bad_r{0}, bad_q{0};
  pdmk::parallel_chunks(3L * n, [&](long b, long e) {
    int bad = 0;
    for (long k = b; k < e; ++k) bad |= !(r[k] >= 0.0 && r[k] < L);
    if (bad) bad_r = 1;
  });
  pdmk::parallel_chunks(long(n), [&](long b, long e) {
    int bad = 0;
    for (long k = b; k < e; ++k) bad |= !std::isfinite(q[k]);
    if (bad) bad_q = 1;
  });
  if (bad_r) return fail(HPDMK_ERR_BAD_INPUT, "positions must lie in [0, L)");
  if (bad_q) return fail(HPDMK_ERR_BAD_INPUT, "charges must be finite");
  return HPDMK_OK;
}

int check_move(const Handle* h, long i, double dx, double dy, double dz) {
  if (i < 0 || i >= h->n) return fail(HPDMK_ERR_BAD_INPUT, "particle index out of range");
  const double lim = 64.0 * h->L;
  if (!(std::fabs(dx) < lim && std::fabs(dy) < lim && std::fabs(dz) < lim))
    return fail(HPDMK_ERR_BAD_INPUT, "displacement must be finite and below 64 L");
  return HPDMK_OK;
}

hpdmk_tree init_impl(HPDMKParams params, const HPDMKExtParams* ext, int n, const double* r, const double* q,
                     bool on_device = false) {
  if (check_params(params) != HPDMK_OK) return nullptr;
  if (on_device) {
    if (n < 1 || !r || !q) {
      fail(HPDMK_ERR_BAD_INPUT, "need n >= 1 particles with positions and charges");
      return nullptr;
    }
  } else if (check_inputs(params.L, n, r, q) != HPDMK_OK) {
    return nullptr;
  }
  Handle* h = nullptr;
  int st = guarded([&]() {
    // the guard outlives the handle under construction, so a failed build
    // releases its device memory with its own device current
    DeviceGuard dg(ext ? ext->device : 0);
    auto hh = std::make_unique<Handle>();
    pdmk::TreeOptions opt;
    opt.leaf_slack = ext ? ext->leaf_slack : 8;
    opt.pool_capacity = ext && ext->pool_capacity > 0 ? ext->pool_capacity : 4096;
    if (opt.leaf_slack < 0) return fail(HPDMK_ERR_BAD_PARAMS, "leaf_slack must be >= 0");
    if (ext && ext->precision != HPDMK_PRECISION_FP64 && ext->precision != HPDMK_PRECISION_MIXED)
      return fail(HPDMK_ERR_BAD_PARAMS, "unknown precision mode");
    opt.precision = ext ? ext->precision : HPDMK_PRECISION_FP64;
    hh->device = ext ? ext->device : 0;
    if (ext && ext->stream) {
      hh->stream = static_cast<cudaStream_t>(ext->stream);
      hh->own_stream = false;
    } else {
      PDMK_CUDA(cudaStreamCreateWithFlags(&hh->stream, cudaStreamNonBlocking));
    }
    hh->n = n;
    hh->L = params.L;
    hh->tree = std::make_unique<pdmk::DmkTree>(params.L, params.n_per_leaf, params.digits, n, r, q, on_device, opt,
                                               hh->stream);
    hh->tree->set_tuning(pdmk::lookup_tuning(params.digits, opt.precision, n));
    h = hh.release();
    return ok();
  });
  return st == HPDMK_OK ? h : nullptr;
}

}  // namespace

extern "C" {

void hpdmk_tree_create(MPI_Comm, HPDMKParams params, int n_src, const double* r_src, const double* charge) {
  hpdmk_tree t = init_impl(params, nullptr, n_src, r_src, charge);
  if (t) delete H(t);
}

hpdmk_tree hpdmk_tree_init(MPI_Comm, HPDMKParams params, int n_src, const double* r_src, const double* charge) {
  return init_impl(params, nullptr, n_src, r_src, charge);
}

hpdmk_tree hpdmk_tree_init_ext(MPI_Comm, HPDMKParams params, const HPDMKExtParams* ext, int n_src,
                               const double* r_src, const double* charge) {
  return init_impl(params, ext, n_src, r_src, charge);
}

hpdmk_tree hpdmk_tree_init_device(MPI_Comm, HPDMKParams params, const HPDMKExtParams* ext, int n_src,
                                  const double* d_r_src, const double* d_charge) {
  return init_impl(params, ext, n_src, d_r_src, d_charge, true);
}

void hpdmk_tree_destroy(hpdmk_tree tree) {
  if (!tree) return;
  try {
    DeviceGuard dg(H(tree)->device);
    delete H(tree);
  } catch (...) {
    delete H(tree);  // the device could not be made current: release what can be released
  }
}

int hpdmk_form_outgoing_pw(hpdmk_tree t) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    Handle* h = H(t);
    DeviceGuard dg(h->device);
    if (h->rebuild_factor > 1.0) {
      int mx = 0, mn = 0;
      h->tree->drift(&mx, &mn);
      const double npl = double(h->tree->n_per_leaf());
      if (mx > std::max(h->rebuild_factor * npl, double(h->base_max)) ||
          mn < std::min(npl / h->rebuild_factor, double(h->base_min))) {
        rebuild_structure(h);
        ++h->rebuilds;
        record_baseline(h);
      }
    }
    h->tree->form_outgoing_pw();
    return ok();
  });
}

int hpdmk_form_incoming_pw(hpdmk_tree t) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->form_incoming_pw();
    return ok();
  });
}

int hpdmk_eval_energy(hpdmk_tree t, double* energy, double* window, double* difference, double* residual) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    pdmk::EnergyParts p = H(t)->tree->eval_energy();
    if (energy) *energy = p.total();
    if (window) *window = p.window;
    if (difference) *difference = p.diff;
    if (residual) *residual = p.res;
    return ok();
  });
}

int hpdmk_energy(hpdmk_tree t, double* energy) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    auto* tr = H(t)->tree.get();
    tr->form_outgoing_pw();
    tr->form_incoming_pw();
    pdmk::EnergyParts p = tr->eval_energy();
    if (energy) *energy = p.total();
    return ok();
  });
}

int hpdmk_eval_shift_energy(hpdmk_tree t, long i, double dx, double dy, double dz, double* dE) {
  if (!t || !dE) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  if (check_move(H(t), i, dx, dy, dz) != HPDMK_OK) return g_last_error;
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    *dE = H(t)->tree->eval_shift_energy(i, dx, dy, dz, nullptr);
    return ok();
  });
}

int hpdmk_debug_shift_parts(hpdmk_tree t, long i, double dx, double dy, double dz, double* parts) {
  if (!t || !parts) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  if (check_move(H(t), i, dx, dy, dz) != HPDMK_OK) return g_last_error;
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->eval_shift_energy(i, dx, dy, dz, parts);
    return ok();
  });
}

int hpdmk_update_shift(hpdmk_tree t, long i, double dx, double dy, double dz) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  if (check_move(H(t), i, dx, dy, dz) != HPDMK_OK) return g_last_error;
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->update_shift(i, dx, dy, dz);
    if (int e = H(t)->tree->check_device_error()) return device_fail(e);
    return ok();
  });
}

int hpdmk_eval_shift_energy_batch_static(hpdmk_tree t, int m, const long* i, const double* d, double* dE) {
  if (!t || m < 0 || (m > 0 && (!i || !d || !dE))) return fail(HPDMK_ERR_BAD_INPUT, "bad batch arguments");
  if (m > HPDMK_STATIC_MAX_MOVES)
    return fail(HPDMK_ERR_BAD_INPUT, "hpdmk_eval_shift_energy_batch_static: m = " + std::to_string(m) +
                                         " exceeds the static buffer limit of " +
                                         std::to_string(HPDMK_STATIC_MAX_MOVES) + " candidates per call");
  Handle* h = H(t);
  for (int c = 0; c < m; ++c)
    if (check_move(h, i[c], d[3 * c], d[3 * c + 1], d[3 * c + 2]) != HPDMK_OK) return g_last_error;
  if (m == 0) return ok();
  return guarded([&]() {
    // the static array's address is per device: the tree's device is current
    DeviceGuard dg(h->device);
    h->tree->shift_batch_static(m, i, d, dE);
    return ok();
  });
}

int hpdmk_eval_shift_energy_batch(hpdmk_tree t, int m, const long* i, const double* d, double* dE) {
  if (!t || m < 0 || (m > 0 && (!i || !d || !dE))) return fail(HPDMK_ERR_BAD_INPUT, "bad batch arguments");
  Handle* h = H(t);
  for (int c = 0; c < m; ++c)
    if (check_move(h, i[c], d[3 * c], d[3 * c + 1], d[3 * c + 2]) != HPDMK_OK) return g_last_error;
  if (m == 0) return ok();
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    h->ensure(m);
    std::vector<int> ii(i, i + m);
    PDMK_CUDA(cudaMemcpyAsync(h->d_i, ii.data(), sizeof(int) * m, cudaMemcpyHostToDevice, h->stream));
    PDMK_CUDA(cudaMemcpyAsync(h->d_d, d, sizeof(double) * 3 * m, cudaMemcpyHostToDevice, h->stream));
    h->tree->shift_batch_device(m, h->d_i, h->d_d, h->d_dE);
    PDMK_CUDA(cudaMemcpyAsync(dE, h->d_dE, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
    PDMK_CUDA(cudaStreamSynchronize(h->stream));
    return ok();
  });
}

int hpdmk_eval_shift_energy_batch_device(hpdmk_tree t, int m, const int* d_i, const double* d_d, double* d_dE) {
  if (!t || m < 0 || (m > 0 && (!d_i || !d_d || !d_dE))) return fail(HPDMK_ERR_BAD_INPUT, "bad batch arguments");
  if (m == 0) return ok();
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->shift_batch_device(m, d_i, d_d, d_dE);
    return ok();
  });
}

int hpdmk_mc_run(hpdmk_tree t, int n, const long* i, const double* d, const double* u, double beta, double* dE,
                 int* accepted) {
  if (!t || n < 0 || (n > 0 && (!i || !d || !u))) return fail(HPDMK_ERR_BAD_INPUT, "bad move arguments");
  Handle* h = H(t);
  for (int c = 0; c < n; ++c)
    if (check_move(h, i[c], d[3 * c], d[3 * c + 1], d[3 * c + 2]) != HPDMK_OK) return g_last_error;
  if (n == 0) return ok();
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    h->ensure(n);
    std::vector<int> ii(i, i + n);
    PDMK_CUDA(cudaMemcpyAsync(h->d_i, ii.data(), sizeof(int) * n, cudaMemcpyHostToDevice, h->stream));
    PDMK_CUDA(cudaMemcpyAsync(h->d_d, d, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, h->stream));
    PDMK_CUDA(cudaMemcpyAsync(h->d_u, u, sizeof(double) * n, cudaMemcpyHostToDevice, h->stream));
    h->tree->reset_work();
    h->tree->mc_run_device(n, h->d_i, h->d_d, h->d_u, beta, h->d_dE, h->d_acc);
    if (dE) PDMK_CUDA(cudaMemcpyAsync(dE, h->d_dE, sizeof(double) * n, cudaMemcpyDeviceToHost, h->stream));
    if (accepted) PDMK_CUDA(cudaMemcpyAsync(accepted, h->d_acc, sizeof(int) * n, cudaMemcpyDeviceToHost, h->stream));
    PDMK_CUDA(cudaStreamSynchronize(h->stream));
    if (int e = h->tree->check_device_error()) return device_fail(e);
    return ok();
  });
}

int hpdmk_mc_run_device(hpdmk_tree t, int n, const int* d_i, const double* d_d, const double* d_u, double beta,
                        double* d_dE, int* d_accepted) {
  if (!t || n < 0 || (n > 0 && (!d_i || !d_d || !d_u))) return fail(HPDMK_ERR_BAD_INPUT, "bad move arguments");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->reset_work();
    H(t)->tree->mc_run_device(n, d_i, d_d, d_u, beta, d_dE, d_accepted);
    return ok();
  });
}

int hpdmk_get_positions(hpdmk_tree t, double* r) {
  if (!t || !r) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->export_positions(r);
    return ok();
  });
}

int hpdmk_tree_info(hpdmk_tree t, long* info) {
  if (!t || !info) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  const auto& D = H(t)->tree->dev();
  info[0] = D.max_depth;
  info[1] = D.n_nodes;
  info[2] = D.N;
  info[3] = D.Hw;
  info[4] = D.H;
  return ok();
}

int hpdmk_synchronize(hpdmk_tree t) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->synchronize();
    return ok();
  });
}

int hpdmk_get_stream(hpdmk_tree t, void** stream) {
  if (!t || !stream) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  *stream = static_cast<void*>(H(t)->stream);
  return ok();
}

int hpdmk_set_mc_mode(hpdmk_tree t, int mode) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  if (mode != HPDMK_MC_PERSISTENT && mode != HPDMK_MC_GRAPH) return fail(HPDMK_ERR_BAD_PARAMS, "unknown mc mode");
  H(t)->tree->set_mc_mode(mode);
  return ok();
}

int hpdmk_set_timing(hpdmk_tree t, int enable) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  H(t)->tree->set_timing(enable != 0);
  return ok();
}

int hpdmk_get_timing(hpdmk_tree t, double* out, int reset) {
  if (!t || !out) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->get_timing(out, reset != 0);
    return ok();
  });
}

int hpdmk_eval_potential(hpdmk_tree t, int m, const long* i, double* phi, double* field) {
  if (!t || m < 0 || (m > 0 && (!i || !phi))) return fail(HPDMK_ERR_BAD_INPUT, "bad potential arguments");
  Handle* h = H(t);
  for (int c = 0; c < m; ++c)
    if (i[c] < 0 || i[c] >= h->n) return fail(HPDMK_ERR_BAD_INPUT, "particle index out of range");
  if (m == 0) return ok();
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    h->ensure(m);
    std::vector<int> ii(i, i + m);
    double* d_field = nullptr;
    if (field) PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&d_field), sizeof(double) * 3 * m, h->stream));
    PDMK_CUDA(cudaMemcpyAsync(h->d_i, ii.data(), sizeof(int) * m, cudaMemcpyHostToDevice, h->stream));
    h->tree->potential_batch(m, h->d_i, h->d_dE, d_field);
    PDMK_CUDA(cudaMemcpyAsync(phi, h->d_dE, sizeof(double) * m, cudaMemcpyDeviceToHost, h->stream));
    if (field) {
      PDMK_CUDA(cudaMemcpyAsync(field, d_field, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, h->stream));
      PDMK_CUDA(cudaFreeAsync(d_field, h->stream));
    }
    PDMK_CUDA(cudaStreamSynchronize(h->stream));
    return ok();
  });
}

int hpdmk_replicas_mc_run(int n_trees, const hpdmk_tree* trees, int m, const long* i, const double* d,
                          const double* u, double beta, double* dE, int* accepted) {
  if (n_trees < 1 || !trees || m < 0 || (m > 0 && (!i || !d || !u)))
    return fail(HPDMK_ERR_BAD_INPUT, "bad replica arguments");
  std::vector<pdmk::DmkTree*> ts;
  for (int t = 0; t < n_trees; ++t) {
    if (!trees[t]) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
    Handle* h = H(trees[t]);
    if (h->device != H(trees[0])->device) return fail(HPDMK_ERR_BAD_INPUT, "replicas must share one device");
    for (int c = 0; c < m; ++c) {
      const size_t k = size_t(t) * m + c;
      if (check_move(h, i[k], d[3 * k], d[3 * k + 1], d[3 * k + 2]) != HPDMK_OK) return g_last_error;
    }
    ts.push_back(h->tree.get());
  }
  if (m == 0) return ok();
  Handle* h0 = H(trees[0]);
  return guarded([&]() {
    DeviceGuard dg(h0->device);
    const size_t tot = size_t(n_trees) * m;
    std::vector<int> ii(i, i + tot);
    char* buf = nullptr;
    const size_t bytes = tot * (4 + 24 + 8 + 8 + 4) + 64;
    PDMK_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&buf), bytes, h0->stream));
    double* d_d = reinterpret_cast<double*>(buf);
    double* d_u = d_d + 3 * tot;
    double* d_dE = d_u + tot;
    int* d_i = reinterpret_cast<int*>(d_dE + tot);
    int* d_acc = d_i + tot;
    PDMK_CUDA(cudaMemcpyAsync(d_i, ii.data(), sizeof(int) * tot, cudaMemcpyHostToDevice, h0->stream));
    PDMK_CUDA(cudaMemcpyAsync(d_d, d, sizeof(double) * 3 * tot, cudaMemcpyHostToDevice, h0->stream));
    PDMK_CUDA(cudaMemcpyAsync(d_u, u, sizeof(double) * tot, cudaMemcpyHostToDevice, h0->stream));
    for (auto* t : ts) t->reset_work();
    pdmk::DmkTree::replicas_mc_run(ts, m, d_i, d_d, d_u, beta, d_dE, d_acc);
    if (dE) PDMK_CUDA(cudaMemcpyAsync(dE, d_dE, sizeof(double) * tot, cudaMemcpyDeviceToHost, h0->stream));
    if (accepted) PDMK_CUDA(cudaMemcpyAsync(accepted, d_acc, sizeof(int) * tot, cudaMemcpyDeviceToHost, h0->stream));
    PDMK_CUDA(cudaFreeAsync(buf, h0->stream));
    PDMK_CUDA(cudaStreamSynchronize(h0->stream));
    for (int t = 0; t < n_trees; ++t)
      if (int e = ts[t]->check_device_error()) return device_fail(e);
    return ok();
  });
}

int hpdmk_replicas_energy(int n_trees, const hpdmk_tree* trees, double* energy) {
  if (n_trees < 1 || !trees || !energy) return fail(HPDMK_ERR_BAD_INPUT, "bad replica arguments");
  for (int t = 0; t < n_trees; ++t)
    if (!trees[t]) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  // each tree runs on its own stream; host threads keep several trees' work
  // in flight, since every tree's pipeline waits on the device a few times
  const int nth = std::max(1, std::min(n_trees, 16));
  std::atomic<int> next{0};
  std::vector<int> codes(n_trees, HPDMK_OK);
  std::vector<std::string> msgs(n_trees);
  std::vector<std::thread> pool;
  for (int w = 0; w < nth; ++w)
    pool.emplace_back([&]() {
      for (int t = next++; t < n_trees; t = next++) {
        Handle* h = H(trees[t]);
        codes[t] = guarded([&]() {
          PDMK_CUDA(cudaSetDevice(h->device));
          h->tree->form_outgoing_pw();
          h->tree->form_incoming_pw();
          energy[t] = h->tree->eval_energy().total();
          return ok();
        });
        if (codes[t] != HPDMK_OK) msgs[t] = g_last_message;
      }
    });
  for (auto& th : pool) th.join();
  for (int t = 0; t < n_trees; ++t)
    if (codes[t] != HPDMK_OK) return fail(codes[t], "replica " + std::to_string(t) + ": " + msgs[t]);
  return ok();
}

int hpdmk_tree_rebuild(hpdmk_tree t) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  Handle* h = H(t);
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    rebuild_structure(h);
    if (h->rebuild_factor > 1.0) record_baseline(h);
    h->tree->form_outgoing_pw();
    h->tree->form_incoming_pw();
    return ok();
  });
}

int hpdmk_set_rebuild_policy(hpdmk_tree t, double leaf_factor) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  if (!(leaf_factor == 0.0 || (leaf_factor > 1.0 && std::isfinite(leaf_factor))))
    return fail(HPDMK_ERR_BAD_INPUT, "leaf_factor must be 0 (off) or a finite number above 1");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->rebuild_factor = leaf_factor;
    if (leaf_factor > 1.0) record_baseline(H(t));
    return ok();
  });
}

int hpdmk_tree_drift(hpdmk_tree t, int* max_leaf, int* min_refined, int* rebuilds) {
  if (!t || !max_leaf || !min_refined) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->drift(max_leaf, min_refined);
    if (rebuilds) *rebuilds = H(t)->rebuilds;
    return ok();
  });
}

int hpdmk_ewald_energy(hpdmk_tree t, double* energy, double* parts) {
  if (!t || !energy) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    *energy = H(t)->tree->ewald_energy(parts);
    return ok();
  });
}

int hpdmk_autotune(hpdmk_tree t, const char* path, int reps, int* chosen, double* times) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    pdmk::autotune_tree(*H(t)->tree, path, reps, chosen, times);
    return ok();
  });
}

int hpdmk_get_tuning(hpdmk_tree t, int* out) {
  if (!t || !out) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  const pdmk::Tuning& u = H(t)->tree->tuning();
  out[0] = u.ksplit;
  out[1] = u.ksplit_root;
  out[2] = u.inc_waves;
  out[3] = u.res_ny_max;
  return ok();
}

int hpdmk_set_tuning(hpdmk_tree t, const int* in) {
  if (!t || !in) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  pdmk::Tuning u;
  u.ksplit = in[0];
  u.ksplit_root = in[1];
  u.inc_waves = in[2];
  u.res_ny_max = in[3];
  H(t)->tree->set_tuning(u);
  return ok();
}

int hpdmk_debug_tuning_lookup(const char* path, int digits, int precision, long n, int* out) {
  if (!path || !out) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    const pdmk::Tuning u = pdmk::lookup_tuning_file(path, digits, precision, n);
    out[0] = u.ksplit;
    out[1] = u.ksplit_root;
    out[2] = u.inc_waves;
    out[3] = u.res_ny_max;
    return ok();
  });
}

int hpdmk_get_launch_count(long long* out) {
  if (!out) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  *out = pdmk::g_launch_count.load();
  return ok();
}

int hpdmk_get_update_bytes(hpdmk_tree t, double* out) {
  if (!t || !out) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->get_work(out);
    return ok();
  });
}

int hpdmk_read_particle_info(const char* filename, long* n, double* r, double* q, long capacity) {
  if (!filename || !n) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    std::vector<double> xyzq;
    if (!pdmk::read_particle_info(filename, xyzq))
      return fail(HPDMK_ERR_BAD_INPUT, std::string("cannot open particle file ") + filename);
    const long m = long(xyzq.size() / 4);
    *n = m;
    if (!r && !q) return ok();  // size query
    if (!r || !q) return fail(HPDMK_ERR_BAD_INPUT, "need both r and q, or neither for a size query");
    if (capacity < m)
      return fail(HPDMK_ERR_BAD_INPUT, "particle file holds " + std::to_string(m) + " particles, capacity is " +
                                           std::to_string(capacity));
    for (long i = 0; i < m; ++i) {
      r[3 * i] = xyzq[4 * i];
      r[3 * i + 1] = xyzq[4 * i + 1];
      r[3 * i + 2] = xyzq[4 * i + 2];
      q[i] = xyzq[4 * i + 3];
    }
    return ok();
  });
}

int hpdmk_last_error(void) { return g_last_error; }
const char* hpdmk_last_error_message(void) { return g_last_message.c_str(); }

int hpdmk_debug_nodes(hpdmk_tree t, int* level, unsigned long long* prefix, int* is_leaf, long* count) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->export_nodes(level, reinterpret_cast<uint64_t*>(prefix), is_leaf, count);
    return ok();
  });
}

int hpdmk_debug_neighbors(hpdmk_tree t, int* col27, int* coarse8) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->export_neighbors(col27, coarse8);
    return ok();
  });
}

int hpdmk_debug_sorted_order(hpdmk_tree t, long* o) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->export_sorted_order(o);
    return ok();
  });
}

int hpdmk_debug_pw(hpdmk_tree t, long node, int which, double* out) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    H(t)->tree->export_pw(node, which, out);
    return ok();
  });
}

int hpdmk_debug_kernels(hpdmk_tree t, int level, double* out) {
  if (!t) return fail(HPDMK_ERR_BAD_INPUT, "null tree");
  return guarded([&]() {
    DeviceGuard dg(H(t)->device);
    if (level == 0) H(t)->tree->export_W(out);
    else H(t)->tree->export_D(level, out);
    return ok();
  });
}

int hpdmk_debug_prolate(int digits, double* out, int nx, const double* x, double* psi) {
  if (!out || (nx > 0 && (!x || !psi))) return fail(HPDMK_ERR_BAD_INPUT, "null argument");
  return guarded([&]() {
    pdmk::ProlateSetup s = pdmk::make_prolate_setup(digits);
    out[0] = s.c;
    out[1] = s.lambda;
    out[2] = s.C0 / s.psi0_0;
    out[3] = s.diff0;
    out[4] = s.n_window;
    out[5] = s.n_diff;
    for (int k = 0; k < nx; ++k) psi[k] = s.psi0(x[k]) / s.psi0_0;
    return ok();
  });
}

}  // extern "C"
