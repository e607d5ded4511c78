// ORACLE — test infrastructure only. A CPU restatement of the reference's
// periodic DMK energy path (tree build, DIRECT plane-wave upward pass,
// incoming plane waves, window/difference/residual energies, single-particle
// energy shift and accept-and-update) plus an FP64 Ewald sum. Only tests/,
// __graft_entry__.smoke() and bench.py's CPU-baseline leg may load it; the
// product library never links or calls it.
#pragma once
#include <cstdint>

extern "C" {
// Set-up constants are computed by oracle/pswf.py (a numpy restatement of
// the reference's src/pswf.cpp); leg[] are the Legendre-series coefficients
// of psi_0^c on [-1,1] (all orders, odd ones zero).
void* or_create(double L, int n_per_leaf, int digits, long n, const double* r, const double* q,
                int n_leg, const double* leg, double c, double lambda, double C0, double diff0,
                int n_poly, const double* poly_horner, int n_window, int n_diff);
void or_destroy(void* h);
// info[0]=max_depth (number of levels) info[1]=n_nodes info[2]=n_particles
// info[3]=H_window info[4]=H_diff info[5]=n_window info[6]=n_diff
void or_info(void* h, long* info);
void or_form_outgoing(void* h, int nthreads);
void or_form_incoming(void* h, int nthreads);
void or_energy(void* h, int nthreads, double* parts /*window,diff,res*/);
void or_energy_direct(void* h, int nthreads, double* parts);
double or_shift(void* h, long i_orig, double dx, double dy, double dz, double* parts /*w,d,rt,ro,self or null*/);
void or_update(void* h, long i_orig, double dx, double dy, double dz, int nthreads);
// tree export: per node (level-major, Morton within a level)
void or_tree_nodes(void* h, int* level, uint64_t* prefix, int* is_leaf, long* count);
void or_tree_neighbors(void* h, int* colleague27 /*[n_nodes][27], -1 absent/self*/, int* coarse8 /*[n_nodes][8] -1 pad*/);
void or_sorted_order(void* h, long* orig_of_sorted);
void or_positions(void* h, double* r_orig_order /*[3n]*/);
void or_get_pw(void* h, long node, int which /*0 out,1 inc*/, double* out);
void or_get_W(void* h, double* out);
void or_get_D(void* h, int level, double* out);
void or_leaf_path(void* h, double x, double y, double z, long* path, int* depth);
// FP64 Ewald (restating the reference's src/ewald.cpp with an O(N^2)
// minimum-image-free real-space loop over 27 images).
double or_ewald_energy(double L, double s, double alpha, long n, const double* r, const double* q, int nthreads);
double or_ewald_potential(double L, double s, double alpha, long n, const double* r, const double* q,
                          double x, double y, double z, long exclude, int nthreads);
// reference test-data stream: default-seeded std::mt19937 through
// std::uniform_real_distribution<double>(lo, hi) (include/utils.hpp:122-129)
void* or_ewald_create(double L, double s, double alpha, long n, const double* r, const double* q, int nthreads);
void or_ewald_destroy(void* h);
double or_ewald_move(void* h, long i, double dx, double dy, double dz, int apply);
void or_random_init(long n, double lo, double hi, double* out);
void or_nudft_halfplane(long M, const double* x, const double* y, const double* z, const double* c, int N, double* f);
void or_nudft_single(double x, double y, double z, double q, int N, double* f);
void or_shift_phases(int n, double dk, double L, int px, int py, int pz, double* out);
double or_res_kernel(int n_poly, const double* poly, double r, double cutoff);
double or_my_mod(double x, double L);
int or_periodic_shift(double xi, double xj, double L, double bi, double bj);
void or_reference_trials(long ntrials, double L, long n, double* d, long* idx);
}
