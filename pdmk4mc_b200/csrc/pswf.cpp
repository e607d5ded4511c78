// psi_0^c as an even Legendre series. Its coefficients are the eigenvector of
// the smallest eigenvalue of the prolate differential operator
//   -(1 - x^2) psi'' + 2 x psi' + c^2 x^2 psi
// in the normalised Legendre basis, where it is symmetric tridiagonal over
// the even orders (x^2 P_k = a_k P_{k+2} + b_k P_k + c_k P_{k-2}). The
// smallest eigenvalue is found by Sturm-sequence bisection and its
// eigenvector by inverse iteration. Integrals use Gauss-Legendre rules.
#include "pswf.hpp"

#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <stdexcept>

namespace pdmk {
namespace {

constexpr double kPi = 3.14159265358979323846;

// The reference's accuracy table (include/utils.hpp:20-52): bandwidth c, the
// difference-kernel half-width n_diff, and the residual polynomial in
// ascending powers of x_scaled = 2 r / b - 1. These numbers define the
// method's kernels, so they are kept identical.
struct TableRow {
  int digits;
  double c;
  int n_diff;
  std::vector<double> ascending;
};

const std::vector<TableRow>& table() {
  static const std::vector<TableRow> t = {
      {3, 7.2462000846862793, 6,
       {1.627823522210361e-01, -4.553645597616490e-01, 4.171687104204163e-01, -7.073638602709915e-02,
        -8.957845614474928e-02, 2.617986644718201e-02, 9.633427876507601e-03}},
      {6, 13.739999771118164, 12,
       {5.482525801351582e-02, -2.616592110444692e-01, 4.862652666337138e-01, -3.894296348642919e-01,
        1.638587821812791e-02, 1.870328434198821e-01, -8.714171086568978e-02, -3.927020727017803e-02,
        3.728187607052319e-02, 3.153734425831139e-03, -8.651313377285847e-03, 1.725110090795567e-04,
        1.034762385284044e-03}},
      {9, 20.736000061035156, 19,
       {1.835718730962269e-02, -1.258015846164503e-01, 3.609487248584408e-01, -5.314579651112283e-01,
        3.447559412892380e-01, 9.664692318551721e-02, -3.124274531849053e-01, 1.322460720579388e-01,
        9.773007866584822e-02, -1.021958831082768e-01, -3.812847450976566e-03, 3.858117355875043e-02,
        -8.728545924521301e-03, -9.401196355382909e-03, 4.024549377076924e-03, 1.512806105865091e-03,
        -9.576734877247042e-04, -1.303457547418901e-04, 1.100385844683190e-04}},
      {12, 27.870000839233398, 26,
       {6.262472576363448e-03, -5.605742936112479e-02, 2.185890864792949e-01, -4.717350304955679e-01,
        5.669680214206270e-01, -2.511606878849214e-01, -2.744523658778361e-01, 4.582527599363415e-01,
        -1.397724810121539e-01, -2.131762135835757e-01, 1.995489373508990e-01, 1.793390341864239e-02,
        -1.035055132403432e-01, 3.035606831075176e-02, 3.153931762550532e-02, -2.033178627450288e-02,
        -5.406682731236552e-03, 7.543645573618463e-03, 1.437788047407851e-05, -1.928370882351732e-03,
        2.891658777328665e-04, 3.332996162099811e-04, -8.397699195938912e-05, -3.015837377517983e-05,
        9.640642701924662e-06}},
  };
  return t;
}

// number of eigenvalues of the symmetric tridiagonal (d, e) below x
int sturm_count(const std::vector<double>& d, const std::vector<double>& e, double x) {
  int cnt = 0;
  double q = 1.0;
  for (size_t i = 0; i < d.size(); ++i) {
    double off = i == 0 ? 0.0 : e[i - 1] * e[i - 1] / q;
    q = d[i] - x - off;
    if (q == 0.0) q = -1e-300;
    if (q < 0) ++cnt;
  }
  return cnt;
}

std::vector<double> legendre_coefficients(double c) {
  const int m = int(2 * c) + 60;  // even orders 0..2(m-1); the tail decays super-exponentially
  std::vector<double> d(m), e(m - 1);
  for (int j = 0; j < m; ++j) {
    double k = 2.0 * j;
    double b = ((k + 1) * (k + 1) / (2 * k + 3) + k * k / (2 * k - 1)) / (2 * k + 1);
    d[j] = k * (k + 1) + c * c * b;
    if (j + 1 < m) {
      double kp = k + 2;
      e[j] = c * c * kp * (kp - 1) / ((2 * kp - 1) * std::sqrt((2 * kp - 3) * (2 * kp + 1)));
    }
  }
  // Gershgorin interval, then bisection for the smallest eigenvalue
  double lo = 1e300, hi = -1e300;
  for (int j = 0; j < m; ++j) {
    double r = (j > 0 ? std::fabs(e[j - 1]) : 0) + (j + 1 < m ? std::fabs(e[j]) : 0);
    lo = std::min(lo, d[j] - r);
    hi = std::max(hi, d[j] + r);
  }
  for (int it = 0; it < 200; ++it) {
    double mid = 0.5 * (lo + hi);
    if (mid == lo || mid == hi) break;
    if (sturm_count(d, e, mid) >= 1) hi = mid;
    else lo = mid;
  }
  const double mu = lo - 1e-12 * std::max(1.0, std::fabs(lo));
  // inverse iteration: solve (A - mu I) v = v_prev by tridiagonal elimination
  std::vector<double> v(m, 1.0), cp(m), dp(m);
  for (int it = 0; it < 4; ++it) {
    double den = d[0] - mu;
    cp[0] = (m > 1 ? e[0] : 0) / den;
    dp[0] = v[0] / den;
    for (int i = 1; i < m; ++i) {
      den = (d[i] - mu) - e[i - 1] * cp[i - 1];
      cp[i] = (i + 1 < m ? e[i] : 0) / den;
      dp[i] = (v[i] - e[i - 1] * dp[i - 1]) / den;
    }
    v[m - 1] = dp[m - 1];
    for (int i = m - 2; i >= 0; --i) v[i] = dp[i] - cp[i] * v[i + 1];
    double nrm = 0;
    for (double x : v) nrm += x * x;
    nrm = std::sqrt(nrm);
    for (double& x : v) x /= nrm;
  }
  std::vector<double> coef(2 * m, 0.0);
  for (int j = 0; j < m; ++j) coef[2 * j] = v[j] * std::sqrt(2.0 * j + 0.5);
  return coef;
}

double legendre_series(const std::vector<double>& a, double x) {
  double p0 = 1.0, p1 = x, s = a[0] + (a.size() > 1 ? a[1] * x : 0.0);
  for (size_t k = 1; k + 1 < a.size(); ++k) {
    double p2 = ((2.0 * k + 1.0) * x * p1 - double(k) * p0) / double(k + 1);
    s += a[k + 1] * p2;
    p0 = p1;
    p1 = p2;
  }
  return s;
}

// n-point Gauss-Legendre rule on [-1, 1] (Newton iteration on P_n)
void gauss_legendre(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0);
  w.assign(n, 0);
  for (int i = 0; i < (n + 1) / 2; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5));
    double pp = 1;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1.0, p1 = z;
      for (int k = 1; k < n; ++k) {
        double p2 = ((2.0 * k + 1.0) * z * p1 - k * p0) / (k + 1.0);
        p0 = p1;
        p1 = p2;
      }
      pp = n * (z * p1 - p0) / (z * z - 1.0);
      double dz = p1 / pp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = -z;
    x[n - 1 - i] = z;
    w[i] = w[n - 1 - i] = 2.0 / ((1.0 - z * z) * pp * pp);
  }
}

}  // namespace

double ProlateSetup::psi0(double x) const {
  if (std::fabs(x) > 1.0) return 0.0;
  return legendre_series(legendre, x);
}

namespace {
ProlateSetup compute_prolate_setup(int digits);
}

// one set-up per digits setting per process
ProlateSetup make_prolate_setup(int digits) {
  static std::mutex mu;
  static std::map<int, ProlateSetup> cache;
  std::lock_guard<std::mutex> g(mu);
  auto it = cache.find(digits);
  if (it != cache.end()) return it->second;
  ProlateSetup s = compute_prolate_setup(digits);
  cache[digits] = s;
  return s;
}

namespace {
ProlateSetup compute_prolate_setup(int digits) {
  const TableRow* row = nullptr;
  for (const auto& r : table())
    if (r.digits == digits) row = &r;
  if (!row) throw std::invalid_argument("double only supports 3, 6, 9 and 12 digits accuracy");
  ProlateSetup s;
  s.digits = digits;
  s.c = row->c;
  s.n_diff = row->n_diff;
  s.n_window = int(std::floor(2 * s.c / kPi));
  s.poly.assign(row->ascending.rbegin(), row->ascending.rend());
  s.legendre = legendre_coefficients(s.c);
  if (legendre_series(s.legendre, 0.0) < 0)
    for (double& a : s.legendre) a = -a;
  std::vector<double> gx, gw;
  gauss_legendre(200, gx, gw);
  double lam = 0, c0 = 0, x2 = 0;
  for (int i = 0; i < 200; ++i) {
    lam += gw[i] * s.psi0(gx[i]) * std::cos(s.c * gx[i] * 0.5);
    double xs = 0.5 * (gx[i] + 1.0);
    double p = s.psi0(xs);
    c0 += gw[i] * 0.5 * p;
    x2 += gw[i] * 0.5 * p * xs * xs;
  }
  s.lambda = lam / s.psi0(0.5);
  s.C0 = c0;
  s.psi0_0 = s.psi0(0.0);
  s.diff0 = -2.0 * kPi * x2 / c0 * s.c * s.c;
  return s;
}
}  // namespace

}  // namespace pdmk
