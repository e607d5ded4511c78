// C-ABI shim over the reference's own math sources, compiled in place from the
// reference tree (src/pswf.cpp plus the header-only templates in include/).
// It exists only so the oracle's golden-vector script and tests can evaluate
// the reference's PSWF functions, constant tables, k-space kernel matrices,
// shift phases, half-plane NUDFTs, vector reductions and wrap helpers on the
// same inputs as the oracle restatement. Test infrastructure only.
#include <hpdmk.h>
#include <utils.hpp>
#include <kernels.hpp>
#include <shiftmat.hpp>
#include <nudft.hpp>
#include <vecops.hpp>
#include <pswf.hpp>
#include <complex>
#include <cstring>
#include <random>

// LAPACK/BLAS are absent here; these are reached only from the reference's
// unused polynomial fitting (approximate_*_poly), which the shim never calls.
extern "C" void dgemm_(char*, char*, int*, int*, int*, double*, double*, int*, double*, int*, double*,
                       double*, int*) {}
extern "C" void dgesdd_(char*, int*, int*, double*, int*, double*, double*, int*, double*, int*, double*,
                        int*, int*, int*) {}

using cd = std::complex<double>;

extern "C" {
double ref_prolate0_eval(double c, double x) { return hpdmk::prolate0_eval(c, x); }
double ref_prolate0_int_eval(double c, double r) { return hpdmk::prolate0_int_eval(c, r); }
double ref_prolate0_intx2_eval(double c, double r) { return hpdmk::prolate0_intx2_eval(c, r); }
double ref_prolate0_lambda(double c) { return hpdmk::prolate0_lambda(c); }

// get_prolate_params (include/utils.hpp:20-52); coefs are returned in the
// reference's Horner order (highest degree first), at most 25 of them.
int ref_get_prolate_params(int digits, double* c, double* lambda, double* C0, int* n_diff, double* coefs) {
  std::vector<double> v;
  hpdmk::get_prolate_params(digits, *c, *lambda, *C0, *n_diff, v);
  for (size_t i = 0; i < v.size(); ++i) coefs[i] = v[i];
  return static_cast<int>(v.size());
}

// diff0 as formed in form_wavenumbers (src/tree.cpp:41-42)
double ref_diff0(double c, double C0) { return -2.0 * M_PI * hpdmk::prolate0_intx2_eval(c, 1.0) / C0 * c * c; }

void ref_window_matrix(double lambda, double C0, double c, double sigma, double dk, int n_k, double* out) {
  auto w = hpdmk::window_matrix<double>(lambda, C0, c, sigma, dk, n_k);
  std::memcpy(out, &w[0], sizeof(double) * w.Dim());
}

void ref_difference_matrix(double lambda, double C0, double c, double diff0, double sigma_l, double sigma_lp1,
                           double dk, int n_k, double* out) {
  auto d = hpdmk::difference_matrix<double>(lambda, C0, c, diff0, sigma_l, sigma_lp1, dk, n_k);
  std::memcpy(out, &d[0], sizeof(double) * d.Dim());
}

// one shift-phase vector of ShiftMatrix (include/shiftmat.hpp:16-38), all d^3 entries
void ref_shift_vec(int n_k, double dk, double L, int px, int py, int pz, double* out) {
  hpdmk::ShiftMatrix<double> sm(n_k, dk, L);
  auto& v = sm.select_shift_vec(px, py, pz);
  std::memcpy(out, &v[0], sizeof(cd) * v.Dim());
}

void ref_nudft3d1_halfplane(int M, const double* x, const double* y, const double* z, const double* c,
                            int iflag, int N1, int N2, int N3, double* f) {
  hpdmk::nudft3d1_halfplane<double>(M, x, y, z, reinterpret_cast<const cd*>(c), iflag, N1, N2, N3,
                                    reinterpret_cast<cd*>(f));
}

void ref_nudft3d1_single_halfplane(double x, double y, double z, double q, int iflag, int N1, int N2, int N3,
                                   double* f) {
  std::vector<cd> xc(N1), yc(N2), zc(N3);
  hpdmk::nudft3d1_single_halfplane<double>(x, y, z, cd(q, 0), iflag, N1, N2, N3, xc.data(), yc.data(), zc.data(),
                                           reinterpret_cast<cd*>(f));
}

double ref_vec_doudot(int M, const double* A, const double* B) {
  return hpdmk::vec_doudot<double>(M, reinterpret_cast<const cd*>(A), B);
}
double ref_vec_tridot_nn(int M, const double* A, const double* B, const double* C) {
  return hpdmk::vec_tridot<double, false, false>(M, reinterpret_cast<const cd*>(A), reinterpret_cast<const cd*>(B), C);
}
double ref_vec_shift_window(int M, const double* t, const double* o, const double* g, const double* W) {
  return hpdmk::vec_shift_window<double>(M, reinterpret_cast<const cd*>(t), reinterpret_cast<const cd*>(o),
                                         reinterpret_cast<const cd*>(g), W);
}
double ref_vec_shift_diff_origin(int M, const double* o, const double* inc, const double* D) {
  return hpdmk::vec_shift_diff_origin<double>(M, reinterpret_cast<const cd*>(o), reinterpret_cast<const cd*>(inc), D);
}
// vec_addsub / vec_muladdsub (include/vecops.hpp:49-114), selected by flags
void ref_vec_addsub(int M, double* A, const double* B, int add, int conj_b) {
  auto a = reinterpret_cast<cd*>(A);
  auto b = reinterpret_cast<const cd*>(B);
  if (add && conj_b) hpdmk::vec_addsub<double, true, true>(M, a, b);
  else if (add) hpdmk::vec_addsub<double, true, false>(M, a, b);
  else if (conj_b) hpdmk::vec_addsub<double, false, true>(M, a, b);
  else hpdmk::vec_addsub<double, false, false>(M, a, b);
}
void ref_vec_muladdsub(int M, double* A, const double* B, const double* C, int add, int conj_b) {
  auto a = reinterpret_cast<cd*>(A);
  auto b = reinterpret_cast<const cd*>(B);
  auto c = reinterpret_cast<const cd*>(C);
  if (add && conj_b) hpdmk::vec_muladdsub<double, true, true>(M, a, b, c);
  else if (add) hpdmk::vec_muladdsub<double, true, false>(M, a, b, c);
  else if (conj_b) hpdmk::vec_muladdsub<double, false, true>(M, a, b, c);
  else hpdmk::vec_muladdsub<double, false, false>(M, a, b, c);
}

double ref_my_mod(double x, double L) { return hpdmk::my_mod(x, L); }
int ref_periodic_shift(double xi, double xj, double L, double bi, double bj) {
  return hpdmk::periodic_shift<double>(xi, xj, L, bi, bj);
}

// residual_kernel (include/kernels.hpp:50-58) with the digits' PolyFun
double ref_residual_kernel(double r, int digits, double cutoff) {
  double c, lambda, C0;
  int n_diff;
  std::vector<double> v;
  hpdmk::get_prolate_params(digits, c, lambda, C0, n_diff, v);
  hpdmk::PolyFun<double> p(v);
  return hpdmk::residual_kernel<double>(r, p, cutoff);
}

// random_init (include/utils.hpp:122-129): default-seeded std::mt19937 stream
void ref_random_init(long n, double lo, double hi, double* out) {
  sctl::Vector<double> v(n);
  hpdmk::random_init(v, lo, hi);
  for (long i = 0; i < n; ++i) out[i] = v[i];
}
}
