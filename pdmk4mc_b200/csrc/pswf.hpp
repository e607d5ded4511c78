// Host-side FP64 set-up of the DMK kernels: the zeroth prolate spheroidal
// wave function psi_0^c and the constants derived from it.
//
// Reference counterparts: get_prolate_params (include/utils.hpp:20-52),
// prolate0_eval / prolate0_int_eval / prolate0_intx2_eval / prolate0_lambda
// (src/pswf.cpp:1118-1218), form_wavenumbers (src/tree.cpp:17-81).
#pragma once
#include <vector>

namespace pdmk {

struct ProlateSetup {
  int digits = 0;
  double c = 0;        // PSWF bandwidth
  int n_diff = 0;      // difference-kernel modes per axis half-width
  int n_window = 0;    // window modes per axis half-width, floor(2c/pi)
  double lambda = 0;   // eigenvalue of psi_0 under the Fourier operator
  double C0 = 0;       // int_0^1 psi_0
  double psi0_0 = 0;   // psi_0(0)
  double diff0 = 0;    // -2 pi int_0^1 x^2 psi_0 / C0 * c^2
  std::vector<double> poly;      // residual polynomial, Horner order (highest first)
  std::vector<double> legendre;  // Legendre-series coefficients of psi_0 on [-1, 1]

  // psi_0(x); zero for |x| > 1 (the reference's evaluator returns zero there
  // for every tabulated c, src/pswf.cpp:976-982)
  double psi0(double x) const;
  // the Fourier transform factor 2 pi lambda psi_0(x) / C0
  double fourier(double x) const { return 2.0 * 3.14159265358979323846 * lambda * psi0(x) / C0; }
};

// throws std::invalid_argument for digits other than 3, 6, 9, 12
ProlateSetup make_prolate_setup(int digits);

}  // namespace pdmk
