// Stand-in for <finufft.h>: finufft 2.4.1 is an unvendored dependency of the
// reference. The oracle's reference build never calls nufft3d1, so only the
// two entry points it names are declared (and left undefined).
#pragma once
#include <complex>
int finufft3d1(long M, double* x, double* y, double* z, std::complex<double>* c, int iflag, double eps,
               long n1, long n2, long n3, std::complex<double>* f, void* opts);
int finufftf3d1(long M, float* x, float* y, float* z, std::complex<float>* c, int iflag, float eps,
                long n1, long n2, long n3, std::complex<float>* f, void* opts);
