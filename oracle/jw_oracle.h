/*
 * jw_oracle -- CPU restatement of the JIMWLK Langevin hot path in FP64.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the CUDA library is compared
 * against (tests/, __graft_entry__.smoke(), bench.py's CPU baseline leg); the
 * product library never links, loads or calls it.  It is itself pinned against
 * the reference's own code compiled here (oracle/_ref/libref_<N>.so, see
 * oracle/ref_harness.cpp) and against the committed golden vectors in
 * tests/golden/.
 *
 * Layout of every field argument: the reference's site-major interleaved
 * complex layout (field.h:73, 170-173): element k (row-major 3x3 index
 * 3*row+col for t = 9) of site (x, y) at complex offset (x*N + y)*t + k,
 * i.e. doubles [2*((x*N+y)*t+k)] (real) and [+1] (imag).
 *
 * Each function cites the reference file:line it restates.
 */
#ifndef JW_ORACLE_H
#define JW_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* enum values identical to config.h:38-42 */
enum { JWO_POSITION_EVOLUTION = 0, JWO_MOMENTUM_EVOLUTION = 1 };
enum { JWO_SQRT_COUPLING = 0, JWO_NOISE_COUPLING = 1, JWO_HATTA_COUPLING = 2 };
/* fixed coupling: plain generate_gaussian + the NOISE kernel factor 1 (see jwo_evolve_momentum) */
enum { JWO_FIXED_COUPLING = 3 };
enum { JWO_LINEAR_KERNEL = 0, JWO_SIN_KERNEL = 1 };

/* ---- noise stream (the engine's definition; the reference's RNG is clock-seeded) ---- */
void jwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
/* 16 unit normals per site for Langevin step `step` of the event with `seed`:
 * z[(x*N+y)*16 + j]; the reference's draw order n0,m0,n1,m1,... (field.h:2170-2173). */
void jwo_langevin_normals(uint64_t seed, uint64_t step, int N, double* z);
/* 8 unit normals per site for MV slice `slice`: z[(x*N+y)*8 + a] (field.h:703-705). */
void jwo_mv_normals(uint64_t seed, int slice, int N, double* z);

/* ---- 2-D unitary FFT of t interleaved components (mpi_fftw_class.h:191-315) ---- */
void jwo_execute2D(double* f, int N, int t, int dir);

/* ---- per-site functions (field.h) ---- */
void jwo_generate_gaussian(const double* z16, double* xi_x, double* xi_y, int N, int with_coupling);
void jwo_set_mv_model(const double* z8, double sigma, double* f, int N);
void jwo_solve_poisson(double* f, int N, double mass, double g);
void jwo_mul_exp(double* V, const double* f, int N);
void jwo_prepare_A_local(double* A, const double* xi_x, const double* xi_y, int N, int coupling, int kernel);
void jwo_uxiulocal(double* ux, double* uy, const double* V, const double* xi_x, const double* xi_y, int N);
void jwo_update_uf(double* V, const double* B, const double* A, int N, double step);
/* su3_matrix::exponentiate: m <- Q diag(exp(i*sign*w)) Q^dagger; returns eigensolver status. */
int jwo_su3_exponentiate(double* m, double sign);
int jwo_zheevh3(const double* A, double* Q, double* w);
void jwo_set_unit(double* V, int N);

/* ---- measurement (field.h:1375-1536) ---- */
void jwo_trace(const double* Vk, double* corr, int N);
void jwo_average_and_symmetrize(double* corr, int N);
void jwo_reduce(const double* corr, double* sum, double* err, int N);

/* ---- driver-level compositions (main_optimized.cpp) ---- */
/* main_optimized.cpp:88, 178-191.  mu_cfg/mass_cfg are the config values
 * (config.h:61-62); g = 1; mu_MV = mu_cfg / N; sigma = g*mu_MV/sqrt(nslices);
 * Poisson mass = mass_cfg * g^2 * mu_MV. */
void jwo_initial_condition(double* V, int N, double mu_cfg, double mass_cfg, int nslices, uint64_t seed);
/* main_optimized.cpp:243-269, 304: `steps` momentum-space steps starting at
 * global step index step0.  coupling = SQRT or NOISE as in the reference (NOISE
 * takes generate_gaussian_with_noise_coupling_constant); FIXED takes plain
 * generate_gaussian with the NOISE kernel factor 1. */
void jwo_evolve_momentum(double* V, int N, int steps, uint64_t step0, double step, int coupling,
                         int kernel, uint64_t seed);
/* main_optimized.cpp:321-334: FFT(V), trace, symmetrise, reduce into sum/err. */
void jwo_measure(const double* V, int N, double* corr, double* sum, double* err);

/* ---- position-space evolution (field.h:2368-2519, positions.h:105-150) ----
 * A(x) = sum_y k(x-y) xi(y), B(x) = sum_y k(x-y) V(y) xi(y) V(y)^dagger, the
 * direct O(V^2) sum in the reference's order.  rr = rr_hatta (main_optimized.cpp:229);
 * for coupling HATTA the reference leaves the coupling uninitialised, and the
 * oracle evaluates the running (SQRT) coupling at min(r^2, rr), its evident intent. */
void jwo_prepare_A_and_B(double* A, double* B, const double* xi_x, const double* xi_y, const double* V, int N,
                         int rr, int coupling, int kernel);
/* The position-space kernel value at displacement (dx, dy) in 0..N-1 (the
 * reference's k_x, k_y before multiplying xi; 0 at the origin). */
void jwo_position_kernel(int dx, int dy, int N, int rr, int coupling, int kernel, double* kx, double* ky);
/* Correlated noise (main_optimized.cpp:145-157): corr(x) =
 * IFFT_unitary(sqrt_alpha(phat2)/N) (field.h:1633-1651); the complex-symmetric
 * Cholesky factor L (L L^T = Sigma, Sigma_ij = corr(|dx|, |dy|), NON-periodic,
 * gmatrix::decompose matrix.h:151-200), lower triangle, row-major V x V
 * complex; multiplyByCholesky (field.h:1653-1689) xi' = L xi per component. */
void jwo_correlations(int N, double* corr);
void jwo_cholesky(const double* corr, int N, double* L);
void jwo_multiply_by_cholesky(const double* L, double* xi, int N);
/* POSITION branch of main_optimized.cpp:243-304: plain generate_gaussian,
 * Cholesky (coupling NOISE, L given), prepare_A_and_B, update_uf. */
void jwo_evolve_position(double* V, int N, int steps, uint64_t step0, double step, int coupling, int kernel,
                         int rr, const double* L, uint64_t seed);
/* gfield::reduce_hatta (field.h:1538-1567): only element (xr, yr). */
void jwo_reduce_hatta(const double* corr, double* sum, double* err, int N, int xr, int yr);

/* ---- dipole in position space (defined by this project; the reference stops at C(k)) ----
 * S(r) = (N^2/3) * sum_k C_sym(k) exp(+2 pi i k.r / N), real part, for every
 * displacement r on the lattice (S_xy[(dx*N+dy)], dx, dy in 0..N-1); then the
 * angular average over bins b = floor(|r_min| + 0.5), |r_min| the minimum-image
 * length, for b < nbins = N/2 + 1: S_b = mean over displacements in bin b.
 * Q_s = sqrt(2)/r_s where S(r_s) = exp(-1/2), by linear interpolation between the
 * first pair of bins that brackets exp(-1/2) (0 if none). */
void jwo_dipole_position(const double* corr_sym, int N, double* S_xy);
int jwo_dipole_radial(const double* S_xy, int N, double* S_b, double* r_b, int* count_b);
double jwo_saturation_scale(const double* S_b, const double* r_b, int nbins);

#ifdef __cplusplus
}
#endif

#endif
