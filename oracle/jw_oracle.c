/*
 * jw_oracle.c -- CPU restatement (FP64, plain C) of the reference's JIMWLK
 * Langevin hot path.  TEST INFRASTRUCTURE ONLY: the checker for the CUDA
 * library, never part of it.  See jw_oracle.h for layouts; every function
 * names the reference file:line it restates.
 *
 * Build: oracle/Makefile (gcc -O2 -ffp-contract=off), into oracle/build/.
 */
#include "jw_oracle.h"

#include <complex.h>
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef double _Complex cplx;

#define RE(p, i) ((p)[2 * (i)])
#define IM(p, i) ((p)[2 * (i) + 1])

static inline cplx ld(const double* p, long i) { return CMPLX(p[2 * i], p[2 * i + 1]); }
static inline void st(double* p, long i, cplx v) {
    p[2 * i] = creal(v);
    p[2 * i + 1] = cimag(v);
}
static inline double sqr(double x) { return x * x; }
static inline double abs2(cplx z) { return sqr(creal(z)) + sqr(cimag(z)); }

/* ======================= noise stream ======================= */

/* Philox-4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with a
 * Weyl-sequence key schedule. */
void jwo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Box-Muller on two 32-bit words: u = (r + 1/2) 2^-32 in (0,1),
 * z0 = sqrt(-2 ln u0) cos(2 pi u1), z1 = sqrt(-2 ln u0) sin(2 pi u1). */
static void box_muller(uint32_t r0, uint32_t r1, double* z0, double* z1) {
    const double two_pi = 6.283185307179586;
    double u0 = ((double)r0 + 0.5) * 2.3283064365386963e-10;
    double u1 = ((double)r1 + 0.5) * 2.3283064365386963e-10;
    double rad = sqrt(-2.0 * log(u0));
    double a = two_pi * u1;
    *z0 = rad * cos(a);
    *z1 = rad * sin(a);
}

#define JW_TAG_LANGEVIN 0x4A570000u
#define JW_TAG_MV 0x4D560000u

void jwo_langevin_normals(uint64_t seed, uint64_t step, int N, double* z) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (long s = 0; s < (long)N * N; ++s) {
        for (uint32_t c = 0; c < 4; ++c) {
            uint32_t ctr[4] = {(uint32_t)s, (uint32_t)step, JW_TAG_LANGEVIN | c, (uint32_t)(step >> 32)};
            uint32_t r[4];
            jwo_philox4x32_10(ctr, key, r);
            double* o = z + s * 16 + 4 * c;
            box_muller(r[0], r[1], &o[0], &o[1]);
            box_muller(r[2], r[3], &o[2], &o[3]);
        }
    }
}

void jwo_mv_normals(uint64_t seed, int slice, int N, double* z) {
    uint32_t key[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (long s = 0; s < (long)N * N; ++s) {
        for (uint32_t c = 0; c < 2; ++c) {
            uint32_t ctr[4] = {(uint32_t)s, (uint32_t)slice, JW_TAG_MV | c, 0u};
            uint32_t r[4];
            jwo_philox4x32_10(ctr, key, r);
            double* o = z + s * 8 + 4 * c;
            box_muller(r[0], r[1], &o[0], &o[1]);
            box_muller(r[2], r[3], &o[2], &o[3]);
        }
    }
}

/* ======================= FFT ======================= */

/* In-place DFT of n complex values at stride `stride` (complex units):
 * y_k = sum_j x_j exp(sign 2 pi i j k / n), sign = -1 forward (FFTW_FORWARD)
 * and +1 backward.  Radix-2 decimation in time for powers of two, direct sum
 * otherwise; twiddles from libm cos/sin of 2 pi k / n. */
static void dft_line(double* x, long stride, int n, int sign, double* buf, const double* tw) {
    for (int j = 0; j < n; ++j) {
        buf[2 * j] = x[2 * j * stride];
        buf[2 * j + 1] = x[2 * j * stride + 1];
    }
    if ((n & (n - 1)) == 0) {
        for (int i = 1, j = 0; i < n; ++i) {
            int bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double t0 = buf[2 * i], t1 = buf[2 * i + 1];
                buf[2 * i] = buf[2 * j]; buf[2 * i + 1] = buf[2 * j + 1];
                buf[2 * j] = t0; buf[2 * j + 1] = t1;
            }
        }
        for (int len = 2; len <= n; len <<= 1) {
            int half = len >> 1, step = n / len;
            for (int s = 0; s < n; s += len) {
                for (int k = 0; k < half; ++k) {
                    double wr = tw[2 * k * step], wi = sign * tw[2 * k * step + 1];
                    double* a = buf + 2 * (s + k);
                    double* b = buf + 2 * (s + k + half);
                    double br = b[0] * wr - b[1] * wi, bi = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - br; b[1] = a[1] - bi;
                    a[0] = a[0] + br; a[1] = a[1] + bi;
                }
            }
        }
        for (int j = 0; j < n; ++j) {
            x[2 * j * stride] = buf[2 * j];
            x[2 * j * stride + 1] = buf[2 * j + 1];
        }
    } else {
        for (int k = 0; k < n; ++k) {
            double sr = 0.0, si = 0.0;
            for (int j = 0; j < n; ++j) {
                long m = ((long)j * k) % n;
                double wr = tw[2 * m], wi = sign * tw[2 * m + 1];
                sr += buf[2 * j] * wr - buf[2 * j + 1] * wi;
                si += buf[2 * j] * wi + buf[2 * j + 1] * wr;
            }
            x[2 * k * stride] = sr;
            x[2 * k * stride + 1] = si;
        }
    }
}

/* fftw2D::execute2D (mpi_fftw_class.h:191-315): the 2-D DFT of each of the t
 * interleaved components, dir = 1 -> FFTW_FORWARD, dir = 0 -> FFTW_BACKWARD,
 * then every value times 1/sqrt(N*N) (:197, :306-310). */
void jwo_execute2D(double* f, int N, int t, int dir) {
    int sign = dir ? -1 : +1;
    double* tw = (double*)malloc(sizeof(double) * 2 * (size_t)N);
    double* buf = (double*)malloc(sizeof(double) * 2 * (size_t)N);
    for (int k = 0; k < N; ++k) {
        double a = 2.0 * M_PI * (double)k / (double)N;
        tw[2 * k] = cos(a);
        tw[2 * k + 1] = sin(a);
    }
    for (int c = 0; c < t; ++c) {
        for (int x = 0; x < N; ++x) dft_line(f + 2 * ((long)x * N * t + c), t, N, sign, buf, tw);
        for (int y = 0; y < N; ++y) dft_line(f + 2 * ((long)y * t + c), (long)N * t, N, sign, buf, tw);
    }
    double scale = 1.0 / sqrt((double)((long)N * N));
    for (long i = 0; i < 2L * t * N * N; ++i) f[i] = f[i] * scale;
    free(tw);
    free(buf);
}

/* ======================= Gell-Mann embedding ======================= */

/* sum_a n_a lambda_a into a 3x3 (row-major 0..8), in the reference's order of
 * accumulation (field.h:2176-2231, identical for setMVModel :716-746).  The
 * second, fifth and seventh matrices enter as +i at (row<col) and -i at
 * (row>col), as the reference writes them. */
static void embed_lambda(const double n[8], cplx m[9]) {
    const double s3 = sqrt(3.0);
    for (int k = 0; k < 9; ++k) m[k] = 0.0;
    m[1] += n[0]; m[3] += n[0];
    m[1] += CMPLX(0.0, n[1]); m[3] -= CMPLX(0.0, n[1]);
    m[0] += n[2]; m[4] -= n[2];
    m[2] += n[3]; m[6] += n[3];
    m[2] += CMPLX(0.0, n[4]); m[6] -= CMPLX(0.0, n[4]);
    m[5] += n[5]; m[7] += n[5];
    m[5] += CMPLX(0.0, n[6]); m[7] -= CMPLX(0.0, n[6]);
    m[0] += n[7] / s3; m[4] += n[7] / s3; m[8] += -2.0 * n[7] / s3;
}

/* generate_gaussian (field.h:2116-2243); with_coupling: the variant
 * generate_gaussian_with_noise_coupling_constant (field.h:2245-2365), which
 * scales every Gaussian at site i by sqrt(4pi/9 / log((w + (phat2(i) N^2/36)^5)^0.2)),
 * phat2 evaluated at the momentum index equal to the SITE index i (:2273). */
void jwo_generate_gaussian(const double* z16, double* xi_x, double* xi_y, int N, int with_coupling) {
    const double tmp = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    const double tmp2 = 4.0 * M_PI / (11.0 - 2.0 * 3.0 / 3.0);
    for (long i = 0; i < (long)N * N; ++i) {
        double n[8], m[8];
        double f = 1.0;
        if (with_coupling) {
            int ix = (int)(i / N), iy = (int)(i % N);
            double sx = sin(M_PI * ix / (1.0 * N)), sy = sin(M_PI * iy / (1.0 * N));
            double phat2 = 4.0 * pow(sx, 2.0) + 4.0 * pow(sy, 2.0);
            f = sqrt(tmp2 / log(pow(tmp + pow((phat2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
        }
        for (int k = 0; k < 8; ++k) {
            n[k] = (z16[i * 16 + 2 * k] * 1.0 + 0.0) * f;
            m[k] = (z16[i * 16 + 2 * k + 1] * 1.0 + 0.0) * f;
        }
        cplx a[9], b[9];
        embed_lambda(n, a);
        embed_lambda(m, b);
        for (int k = 0; k < 9; ++k) {
            st(xi_x, i * 9 + k, a[k]);
            st(xi_y, i * 9 + k, b[k]);
        }
    }
}

/* lfield::setMVModel (field.h:683-757): n_a = sigma z_a, sigma = g mu/sqrt(Ny). */
void jwo_set_mv_model(const double* z8, double sigma, double* f, int N) {
    for (long i = 0; i < (long)N * N; ++i) {
        double n[8];
        for (int k = 0; k < 8; ++k) n[k] = z8[i * 8 + k] * sigma + 0.0;
        cplx a[9];
        embed_lambda(n, a);
        for (int k = 0; k < 9; ++k) st(f, i * 9 + k, a[k]);
    }
}

/* momenta::set (momenta.h:90-124) for one momentum index (ig, jg). */
static double phat2_of(int ig, int jg, int N) {
    double sx = sin(M_PI * ig / (1.0 * N)), sy = sin(M_PI * jg / (1.0 * N));
    return 4.0 * pow(sx, 2.0) + 4.0 * pow(sy, 2.0);
}
static double pbar_of(int ig, int N) { return sin(2.0 * M_PI * ig / (1.0 * N)); }

/* lfield::solvePoisson (field.h:867-877): f(k) *= -g / (-phat2(k) + mass^2). */
void jwo_solve_poisson(double* f, int N, double mass, double g) {
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
            long i = (long)x * N + y;
            double fac = -1.0 * g / (-phat2_of(x, y, N) + mass * mass);
            for (int k = 0; k < 9; ++k) st(f, i * 9 + k, ld(f, i * 9 + k) * CMPLX(fac, 0.0));
        }
}

/* ======================= SU(3) algebra ======================= */

/* su3_matrix::operator* (su3_matrix.h:155-168): naive 27-term product. */
static void mul3(const cplx* a, const cplx* b, cplx* c) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cplx s = 0.0;
            for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
            c[i * 3 + j] = s;
        }
}
static void dagger3(const cplx* a, cplx* d) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) d[i * 3 + j] = conj(a[j * 3 + i]);
}

/* Eigenvalues of a Hermitian 3x3 by Cardano's formula, reading only the
 * diagonal real parts and the upper triangle -- the published algorithm of
 * J. Kopp, "Efficient numerical diagonalization of hermitian 3x3 matrices",
 * Int. J. Mod. Phys. C 19 (2008) 523 (arXiv:physics/0610206), routine
 * ZHEEVC3, as the reference vendors it (zheevh3-C-1.1/zheevc3.cpp:33-86). */
static void eig_cardano(const cplx A[3][3], double w[3]) {
    cplx de = A[0][1] * A[1][2];
    double dd = abs2(A[0][1]), ee = abs2(A[1][2]), ff = abs2(A[0][2]);
    double a = creal(A[0][0]), b = creal(A[1][1]), c = creal(A[2][2]);
    double m = a + b + c;
    double c1 = (a * b + a * c + b * c) - (dd + ee + ff);
    double c0 = c * dd + a * ee + b * ff - a * b * c
              - 2.0 * (creal(A[0][2]) * creal(de) + cimag(A[0][2]) * cimag(de));
    double p = sqr(m) - 3.0 * c1;
    double q = m * (p - (3.0 / 2.0) * c1) - (27.0 / 2.0) * c0;
    double sqrt_p = sqrt(fabs(p));
    double phi = 27.0 * (0.25 * sqr(c1) * (p - c1) + c0 * (q + 27.0 / 4.0 * c0));
    phi = (1.0 / 3.0) * atan2(sqrt(fabs(phi)), q);
    double cc = sqrt_p * cos(phi);
    double s = (1.0 / 1.73205080756887729352744634151) * sqrt_p * sin(phi);
    w[1] = (1.0 / 3.0) * (m - cc);
    w[2] = w[1] + s;
    w[0] = w[1] + cc;
    w[1] -= s;
}

/* Householder reduction of a Hermitian 3x3 to real tridiagonal form,
 * A = Q T Q^H (Kopp, ZHETRD3; zheevh3-C-1.1/zhetrd3.cpp:30-). */
static void tridiag_householder(const cplx A[3][3], cplx Q[3][3], double d[3], double e[3]) {
    cplx u[3], q[3], omega, f;
    double K, h, g;
    for (int i = 0; i < 3; ++i) {
        Q[i][i] = 1.0;
        for (int j = 0; j < i; ++j) Q[i][j] = Q[j][i] = 0.0;
    }
    h = abs2(A[0][1]) + abs2(A[0][2]);
    g = (creal(A[0][1]) > 0) ? -sqrt(h) : sqrt(h);
    e[0] = g;
    f = g * A[0][1];
    u[1] = conj(A[0][1]) - g;
    u[2] = conj(A[0][2]);
    omega = h - f;
    if (creal(omega) > 0.0) {
        omega = 0.5 * (1.0 + conj(omega) / omega) / creal(omega);
        K = 0.0;
        for (int i = 1; i < 3; ++i) {
            f = conj(A[1][i]) * u[1] + A[i][2] * u[2];
            q[i] = omega * f;
            K += creal(conj(u[i]) * f);
        }
        K *= 0.5 * abs2(omega);
        for (int i = 1; i < 3; ++i) q[i] = q[i] - K * u[i];
        d[0] = creal(A[0][0]);
        d[1] = creal(A[1][1]) - 2.0 * creal(q[1] * conj(u[1]));
        d[2] = creal(A[2][2]) - 2.0 * creal(q[2] * conj(u[2]));
        for (int j = 1; j < 3; ++j) {
            f = omega * conj(u[j]);
            for (int i = 1; i < 3; ++i) Q[i][j] = Q[i][j] - f * u[i];
        }
        f = A[1][2] - q[1] * conj(u[2]) - u[1] * conj(q[2]);
    } else {
        for (int i = 0; i < 3; ++i) d[i] = creal(A[i][i]);
        f = A[1][2];
    }
    e[1] = cabs(f);
    if (e[1] != 0.0) {
        f = conj(f) / e[1];
        for (int i = 1; i < 3; ++i) Q[i][2] = Q[i][2] * f;
    }
}

/* QL iteration with implicit shifts on the tridiagonal form, at most 30
 * sweeps per eigenvalue (Kopp, ZHEEVQ3; zheevh3-C-1.1/zheevq3.cpp:31-).
 * Returns -1 when an eigenvalue has not converged. */
static int eig_ql(const cplx A[3][3], cplx Q[3][3], double w[3]) {
    double e[3], g, r, p, f, b, s, c;
    int m;
    tridiag_householder(A, Q, w, e);
    for (int l = 0; l < 2; ++l) {
        int nIter = 0;
        for (;;) {
            for (m = l; m <= 1; ++m) {
                g = fabs(w[m]) + fabs(w[m + 1]);
                if (fabs(e[m]) + g == g) break;
            }
            if (m == l) break;
            if (nIter++ >= 30) return -1;
            g = (w[l + 1] - w[l]) / (e[l] + e[l]);
            r = sqrt(sqr(g) + 1.0);
            if (g > 0) g = w[m] - w[l] + e[l] / (g + r);
            else g = w[m] - w[l] + e[l] / (g - r);
            s = c = 1.0;
            p = 0.0;
            for (int i = m - 1; i >= l; --i) {
                f = s * e[i];
                b = c * e[i];
                if (fabs(f) > fabs(g)) {
                    c = g / f;
                    r = sqrt(sqr(c) + 1.0);
                    e[i + 1] = f * r;
                    c *= (s = 1.0 / r);
                } else {
                    s = f / g;
                    r = sqrt(sqr(s) + 1.0);
                    e[i + 1] = g * r;
                    s *= (c = 1.0 / r);
                }
                g = w[i + 1] - p;
                r = (w[i] - g) * s + 2.0 * c * b;
                p = s * r;
                w[i + 1] = g + p;
                g = c * r - b;
                for (int k = 0; k < 3; ++k) {
                    cplx t = Q[k][i + 1];
                    Q[k][i + 1] = s * Q[k][i] + c * t;
                    Q[k][i] = c * Q[k][i] - s * t;
                }
            }
            w[l] -= p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

/* Hybrid eigensolver (Kopp's ZHEEVH3 as templated in su3_matrix.h:256-359):
 * Cardano eigenvalues, eigenvectors from cross products of the columns of
 * A - w I, falling back to the QL route when a cross product is too small
 * relative to 256 eps max|w|^2 (or max|w|^4 when max|w| >= 1). */
static int hybrid_eigh(const cplx A[3][3], cplx Q[3][3], double w[3]) {
    double norm, error, t, u;
    eig_cardano(A, w);
    t = fabs(w[0]);
    if ((u = fabs(w[1])) > t) t = u;
    if ((u = fabs(w[2])) > t) t = u;
    u = (t < 1.0) ? t : sqr(t);
    error = 256.0 * DBL_EPSILON * sqr(u);
    Q[0][1] = A[0][1] * A[1][2] - A[0][2] * creal(A[1][1]);
    Q[1][1] = A[0][2] * conj(A[0][1]) - A[1][2] * creal(A[0][0]);
    Q[2][1] = abs2(A[0][1]);
    Q[0][0] = Q[0][1] + A[0][2] * w[0];
    Q[1][0] = Q[1][1] + A[1][2] * w[0];
    Q[2][0] = (creal(A[0][0]) - w[0]) * (creal(A[1][1]) - w[0]) - Q[2][1];
    norm = abs2(Q[0][0]) + abs2(Q[1][0]) + sqr(creal(Q[2][0]));
    if (norm <= error) return eig_ql(A, Q, w);
    norm = sqrt(1.0 / norm);
    for (int j = 0; j < 3; ++j) Q[j][0] = Q[j][0] * norm;
    Q[0][1] = Q[0][1] + A[0][2] * w[1];
    Q[1][1] = Q[1][1] + A[1][2] * w[1];
    Q[2][1] = (creal(A[0][0]) - w[1]) * (creal(A[1][1]) - w[1]) - creal(Q[2][1]);
    norm = abs2(Q[0][1]) + abs2(Q[1][1]) + sqr(creal(Q[2][1]));
    if (norm <= error) return eig_ql(A, Q, w);
    norm = sqrt(1.0 / norm);
    for (int j = 0; j < 3; ++j) Q[j][1] = Q[j][1] * norm;
    Q[0][2] = conj(Q[1][0] * Q[2][1] - Q[2][0] * Q[1][1]);
    Q[1][2] = conj(Q[2][0] * Q[0][1] - Q[0][0] * Q[2][1]);
    Q[2][2] = conj(Q[0][0] * Q[1][1] - Q[1][0] * Q[0][1]);
    return 0;
}

int jwo_zheevh3(const double* Ain, double* Qout, double* w) {
    cplx A[3][3], Q[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = ld(Ain, i * 3 + j);
    int st_ = hybrid_eigh(A, Q, w);
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) st(Qout, i * 3 + j, Q[i][j]);
    return st_;
}

/* su3_matrix::exponentiate (su3_matrix.h:173-253):
 * m <- sum_k Q[:,k] exp(i sign w_k) Q[:,k]^H. */
static int su3_exp(cplx m[9], double sign) {
    cplx A[3][3], Q[3][3], eig[3];
    double w[3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) A[i][j] = m[i * 3 + j];
    int status = hybrid_eigh(A, Q, w);
    for (int k = 0; k < 3; ++k) eig[k] = CMPLX(cos(sign * w[k]), sin(sign * w[k]));
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            cplx s = 0.0;
            for (int k = 0; k < 3; ++k) s += Q[i][k] * eig[k] * conj(Q[j][k]);
            m[i * 3 + j] = s;
        }
    return status;
}

int jwo_su3_exponentiate(double* m, double sign) {
    cplx a[9];
    for (int k = 0; k < 9; ++k) a[k] = ld(m, k);
    int s = su3_exp(a, sign);
    for (int k = 0; k < 9; ++k) st(m, k, a[k]);
    return s;
}

void jwo_set_unit(double* V, int N) {
    memset(V, 0, sizeof(double) * 18 * (size_t)N * N);
    for (long i = 0; i < (long)N * N; ++i) {
        V[18 * i + 0] = 1.0;
        V[18 * i + 8] = 1.0;
        V[18 * i + 16] = 1.0;
    }
}

/* lfield::operator*= (field.h:337-365): V(x) <- V(x) exp(+i f(x)). */
void jwo_mul_exp(double* V, const double* f, int N) {
    for (long i = 0; i < (long)N * N; ++i) {
        cplx a[9], b[9], c[9];
        for (int k = 0; k < 9; ++k) { a[k] = ld(V, i * 9 + k); b[k] = ld(f, i * 9 + k); }
        su3_exp(b, 1.0);
        mul3(a, b, c);
        for (int k = 0; k < 9; ++k) st(V, i * 9 + k, c[k]);
    }
}

/* prepare_A_local (field.h:1998-2075):
 * A(k) = K_x(k) xi_x(k) + K_y(k) xi_y(k), K_i = -2 pi i sqrt(alpha) q_i / q^2,
 * q from the wrapped index (k >= N/2 -> k - N); zero mode (|p|^2 <= 1e-8) -> 0.
 * LINEAR: q = p = 2 pi k / N.  SIN: q_i = pbar_i = sin(2 pi k_i / N) (unwrapped
 * index), q^2 = phat2.  alpha = 1 (NOISE) or the running coupling (SQRT);
 * HATTA leaves the coupling undefined in the reference and is rejected here. */
void jwo_prepare_A_local(double* A, const double* xi_x, const double* xi_y, int N, int coupling, int kernel) {
    for (int ix = 0; ix < N; ++ix)
        for (int iy = 0; iy < N; ++iy) {
            long i = (long)ix * N + iy;
            int xx = ix, yy = iy;
            if (xx >= N / 2) xx = xx - N;
            if (yy >= N / 2) yy = yy - N;
            double px = 2.0 * M_PI * xx / (1.0 * N), py = 2.0 * M_PI * yy / (1.0 * N);
            cplx E[9];
            for (int k = 0; k < 9; ++k) E[k] = 0.0;
            if (fabs(px * px + py * py) > 10e-9) {
                double cc = 1.0;
                cplx AA = 0.0, BB = 0.0;
                if (kernel == JWO_LINEAR_KERNEL) {
                    if (coupling == JWO_SQRT_COUPLING)
                        cc = 4.0 * M_PI / ((11.0 - 2.0 * 3.0 / 3.0) *
                             log(pow(pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2) +
                                     pow(((px * px + py * py) * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
                    AA = CMPLX(0.0, -2.0 * M_PI * sqrt(cc) * px / (px * px + py * py));
                    BB = CMPLX(0.0, -2.0 * M_PI * sqrt(cc) * py / (px * px + py * py));
                } else {
                    double ph2 = phat2_of(ix, iy, N);
                    if (coupling == JWO_SQRT_COUPLING)
                        cc = 4.0 * M_PI / ((11.0 - 2.0 * 3.0 / 3.0) *
                             log(pow(pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2) +
                                     pow((ph2 * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2)));
                    AA = CMPLX(0.0, -2.0 * M_PI * sqrt(cc) * pbar_of(ix, N) / ph2);
                    BB = CMPLX(0.0, -2.0 * M_PI * sqrt(cc) * pbar_of(iy, N) / ph2);
                }
                for (int k = 0; k < 9; ++k) E[k] = AA * ld(xi_x, i * 9 + k) + BB * ld(xi_y, i * 9 + k);
            }
            for (int k = 0; k < 9; ++k) st(A, i * 9 + k, E[k]);
        }
}

/* uxiulocal (field.h:1892-1933): ux = V xi_x V^dagger, uy = V xi_y V^dagger,
 * evaluated as (V xi) V^dagger. */
void jwo_uxiulocal(double* ux, double* uy, const double* V, const double* xi_x, const double* xi_y, int N) {
    for (long i = 0; i < (long)N * N; ++i) {
        cplx a[9], b[9], c[9], d[9], t[9], e[9], f[9];
        for (int k = 0; k < 9; ++k) { a[k] = ld(V, i * 9 + k); b[k] = ld(xi_x, i * 9 + k); c[k] = ld(xi_y, i * 9 + k); }
        dagger3(a, d);
        mul3(a, b, t); mul3(t, d, e);
        mul3(a, c, t); mul3(t, d, f);
        for (int k = 0; k < 9; ++k) { st(ux, i * 9 + k, e[k]); st(uy, i * 9 + k, f[k]); }
    }
}

/* update_uf (field.h:1966-1996): V <- exp(+i sqrt(eps) B) V exp(-i sqrt(eps) A),
 * as exponentiate(-1) of -sqrt(eps) B and of +sqrt(eps) A, product (eB V) eA. */
void jwo_update_uf(double* V, const double* B, const double* A, int N, double step) {
    double se = sqrt(step);
    for (long i = 0; i < (long)N * N; ++i) {
        cplx a[9], b[9], c[9], t[9], e[9];
        for (int k = 0; k < 9; ++k) {
            a[k] = ld(V, i * 9 + k);
            b[k] = -se * ld(B, i * 9 + k);
            c[k] = se * ld(A, i * 9 + k);
        }
        su3_exp(b, -1.0);
        su3_exp(c, -1.0);
        mul3(b, a, t);
        mul3(t, c, e);
        for (int k = 0; k < 9; ++k) st(V, i * 9 + k, e[k]);
    }
}

/* ======================= measurement ======================= */

/* lfield::trace (field.h:1375-1432): C(k) = tr(A A^dagger) with A = Vk/(N*N). */
void jwo_trace(const double* Vk, double* corr, int N) {
    const double v = 1.0 * N * N;
    for (long i = 0; i < (long)N * N; ++i) {
        cplx a[9], b[9], c[9];
        for (int k = 0; k < 9; ++k) a[k] = ld(Vk, i * 9 + k) / v;
        for (int r = 0; r < 3; ++r)
            for (int s = 0; s < 3; ++s) b[r * 3 + s] = conj(ld(Vk, i * 9 + s * 3 + r) / v);
        mul3(a, b, c);
        st(corr, i, c[0] + c[4] + c[8]);
    }
}

/* gfield::average_and_symmetrize (field.h:1460-1492): symmetrise kx <-> ky,
 * then average over (+-kx, +-ky). */
void jwo_average_and_symmetrize(double* corr, int N) {
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)N * N);
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j)
            st(tmp, (long)i * N + j, 0.5 * (ld(corr, (long)i * N + j) + ld(corr, (long)j * N + i)));
    for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
            int a = abs(i - N) % N, b = abs(j - N) % N;
            st(corr, (long)i * N + j,
               0.25 * (ld(tmp, (long)i * N + j) + ld(tmp, (long)a * N + j) +
                       ld(tmp, (long)i * N + b) + ld(tmp, (long)a * N + b)));
        }
    free(tmp);
}

/* gfield::reduce (field.h:1521-1536): sum += C, err += C^2 (complex square). */
void jwo_reduce(const double* corr, double* sum, double* err, int N) {
    for (long i = 0; i < (long)N * N; ++i) {
        cplx c = ld(corr, i);
        st(sum, i, ld(sum, i) + c);
        cplx sq = (cimag(c) == 0.0 && creal(c) > 0.0) ? CMPLX(pow(creal(c), 2.0), 0.0) : c * c;
        st(err, i, ld(err, i) + sq);
    }
}

/* ======================= driver compositions ======================= */

void jwo_initial_condition(double* V, int N, double mu_cfg, double mass_cfg, int nslices, uint64_t seed) {
    const long vol = (long)N * N;
    const double g = 1.0;
    const double mu = mu_cfg / N;
    const double sigma = g * mu / sqrt((double)nslices);
    double* z = (double*)malloc(sizeof(double) * 8 * vol);
    double* f = (double*)malloc(sizeof(double) * 18 * vol);
    jwo_set_unit(V, N);
    for (int s = 0; s < nslices; ++s) {
        jwo_mv_normals(seed, s, N, z);
        jwo_set_mv_model(z, sigma, f, N);
        jwo_execute2D(f, N, 9, 1);
        jwo_solve_poisson(f, N, mass_cfg * pow(g, 2.0) * mu, g);
        jwo_execute2D(f, N, 9, 0);
        jwo_mul_exp(V, f, N);
    }
    free(z);
    free(f);
}

void jwo_evolve_momentum(double* V, int N, int steps, uint64_t step0, double step, int coupling,
                         int kernel, uint64_t seed) {
    const long vol = (long)N * N;
    double* z = (double*)malloc(sizeof(double) * 16 * vol);
    double* xx = (double*)malloc(sizeof(double) * 18 * vol);
    double* xy = (double*)malloc(sizeof(double) * 18 * vol);
    double* A = (double*)malloc(sizeof(double) * 18 * vol);
    double* B = (double*)malloc(sizeof(double) * 18 * vol);
    double* ux = (double*)malloc(sizeof(double) * 18 * vol);
    double* uy = (double*)malloc(sizeof(double) * 18 * vol);
    const int kc = (coupling == JWO_FIXED_COUPLING) ? JWO_NOISE_COUPLING : coupling;
    for (int s = 0; s < steps; ++s) {
        jwo_langevin_normals(seed, step0 + (uint64_t)s, N, z);
        jwo_generate_gaussian(z, xx, xy, N, coupling == JWO_NOISE_COUPLING);
        jwo_execute2D(xx, N, 9, 1);
        jwo_execute2D(xy, N, 9, 1);
        jwo_prepare_A_local(A, xx, xy, N, kc, kernel);
        jwo_execute2D(A, N, 9, 0);
        jwo_execute2D(xx, N, 9, 0);
        jwo_execute2D(xy, N, 9, 0);
        jwo_uxiulocal(ux, uy, V, xx, xy, N);
        jwo_execute2D(ux, N, 9, 1);
        jwo_execute2D(uy, N, 9, 1);
        jwo_prepare_A_local(B, ux, uy, N, kc, kernel);
        jwo_execute2D(B, N, 9, 0);
        jwo_update_uf(V, B, A, N, step);
    }
    free(z); free(xx); free(xy); free(A); free(B); free(ux); free(uy);
}

void jwo_measure(const double* V, int N, double* corr, double* sum, double* err) {
    const long vol = (long)N * N;
    double* c = (double*)malloc(sizeof(double) * 18 * vol);
    memcpy(c, V, sizeof(double) * 18 * vol);
    jwo_execute2D(c, N, 9, 1);
    jwo_trace(c, corr, N);
    jwo_average_and_symmetrize(corr, N);
    jwo_reduce(corr, sum, err, N);
    free(c);
}

/* ======================= position-space evolution ======================= */

void jwo_position_kernel(int dxi, int dyi, int N, int rr, int coupling, int kernel, double* kx, double* ky) {
    double dx, dy, rrr;
    if (kernel == JWO_SIN_KERNEL) {
        /* positions::set (positions.h:130-141) at ii = dxi*N + dyi */
        dx = 0.5 * N * sin(2.0 * M_PI * dxi / (1.0 * N)) / M_PI;
        dy = 0.5 * N * sin(2.0 * M_PI * dyi / (1.0 * N)) / M_PI;
        double sx = N * sin(M_PI * dxi / (1.0 * N)) / M_PI, sy = N * sin(M_PI * dyi / (1.0 * N)) / M_PI;
        rrr = pow(sx, 2.0) + pow(sy, 2.0);
    } else {
        dx = dxi;
        if (dx >= N / 2) dx = dx - N;
        if (dx < -N / 2) dx = dx + N;
        dy = dyi;
        if (dy >= N / 2) dy = dy - N;
        if (dy < -N / 2) dy = dy + N;
        rrr = 1.0 * (dx * dx + dy * dy);
    }
    double rrrmin = rrr;
    if (coupling == JWO_HATTA_COUPLING) rrrmin = (rrr <= rr) ? rrr : rr;
    const double lambda = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    double sc = 1.0;
    if (coupling == JWO_SQRT_COUPLING || coupling == JWO_HATTA_COUPLING)
        sc = sqrt(4.0 * M_PI / ((11.0 - 2.0 * 3.0 / 3.0) *
                                log(pow(lambda + 1.26 / pow(6.0 * 6.0 * rrrmin / N / N, 1.0 / 0.2), 0.2))));
    *kx = 0.0;
    *ky = 0.0;
    if (rrr > 10e-9) {
        *kx = sc * dx / rrr;
        *ky = sc * dy / rrr;
    }
}

/* prepare_A_and_B_local (field.h:2368-2519): for output site x the sum over
 * all y in (xx, yy) order, re and im accumulated separately. */
void jwo_prepare_A_and_B(double* A, double* B, const double* xi_x, const double* xi_y, const double* V, int N,
                         int rr, int coupling, int kernel) {
    for (int xg = 0; xg < N; ++xg)
        for (int yg = 0; yg < N; ++yg) {
            double sAr[9] = {0}, sAi[9] = {0}, sBr[9] = {0}, sBi[9] = {0};
            for (int xx = 0; xx < N; ++xx)
                for (int yy = 0; yy < N; ++yy) {
                    long i = (long)xx * N + yy;
                    int dxi = xg >= xx ? xg - xx : xg - xx + N;
                    int dyi = yg >= yy ? yg - yy : yg - yy + N;
                    double kx, ky;
                    jwo_position_kernel(dxi, dyi, N, rr, coupling, kernel, &kx, &ky);
                    cplx Ak = CMPLX(kx, 0.0), Bk = CMPLX(ky, 0.0);
                    cplx E[9], G[9], H[9], T[9], K[9];
                    for (int k = 0; k < 9; ++k) {
                        E[k] = Ak * ld(xi_x, i * 9 + k) + Bk * ld(xi_y, i * 9 + k);
                        G[k] = ld(V, i * 9 + k);
                    }
                    dagger3(G, H);
                    mul3(G, E, T);
                    mul3(T, H, K);
                    for (int k = 0; k < 9; ++k) {
                        sAr[k] += creal(E[k]); sAi[k] += cimag(E[k]);
                        sBr[k] += creal(K[k]); sBi[k] += cimag(K[k]);
                    }
                }
            long o = (long)xg * N + yg;
            for (int k = 0; k < 9; ++k) {
                st(A, o * 9 + k, CMPLX(sAr[k], sAi[k]));
                st(B, o * 9 + k, CMPLX(sBr[k], sBi[k]));
            }
        }
}

/* lfield::setCorrelationsForCouplingConstant (field.h:1633-1651), then the
 * backward unitary transform (main_optimized.cpp:149). */
void jwo_correlations(int N, double* corr) {
    const double w = pow(15.0 * 15.0 / 6.0 / 6.0, 1.0 / 0.2);
    const double f = 4.0 * M_PI / (11.0 - 2.0 * 3.0 / 3.0);
    for (int xx = 0; xx < N; ++xx)
        for (int yy = 0; yy < N; ++yy) {
            long i = (long)xx * N + yy;
            double sc = f / log(pow(w + pow((phat2_of(xx, yy, N) * N * N) / 6.0 / 6.0, 1.0 / 0.2), 0.2));
            st(corr, i, CMPLX(sc / sqrt((double)(N * N)), 0.0));
        }
    jwo_execute2D(corr, N, 1, 0);
}

/* gmatrix::decompose (matrix.h:151-200): row-oriented complex-symmetric
 * Cholesky, L_ii = sqrt(corr[0] - sum_k L_ik^2), L_ij = (corr[|dx| N + |dy|] -
 * sum_k L_ik L_jk) / L_jj.  pow(z, 2) with an int exponent is z*z (then times
 * 1) in libstdc++; complex sqrt and division as C99 csqrt and __divdc3. */
void jwo_cholesky(const double* corr, int N, double* L) {
    const long n = (long)N * N;
    memset(L, 0, sizeof(double) * 2 * (size_t)n * n);
    for (long i = 0; i < n; ++i)
        for (long j = 0; j <= i; ++j) {
            if (j == i) {
                cplx sum = 0;
                for (long k = 0; k < i; ++k) {
                    cplx z = ld(L, i * n + k);
                    sum += CMPLX(1.0, 0.0) * (z * z);
                }
                st(L, i * n + i, csqrt(ld(corr, 0) - sum));
            } else {
                cplx sum = 0;
                for (long k = 0; k < j; ++k) sum += ld(L, i * n + k) * ld(L, j * n + k);
                long xi = i / N, yi = i - xi * N, xj = j / N, yj = j - xj * N;
                long ii = labs(xi - xj) * N + labs(yi - yj);
                st(L, i * n + j, (ld(corr, ii) - sum) / ld(L, j * n + j));
            }
        }
}

/* gfield::multiplyByCholesky (field.h:1653-1689): per component, over all j. */
void jwo_multiply_by_cholesky(const double* L, double* xi, int N) {
    const long n = (long)N * N;
    double* tmp = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (int tt = 0; tt < 9; ++tt) {
        for (long a = 0; a < n; ++a) {
            cplx s = 0;
            for (long b = 0; b < n; ++b) s += ld(L, a * n + b) * ld(xi, b * 9 + tt);
            st(tmp, a, s);
        }
        for (long a = 0; a < n; ++a) st(xi, a * 9 + tt, ld(tmp, a));
    }
    free(tmp);
}

void jwo_evolve_position(double* V, int N, int steps, uint64_t step0, double step, int coupling, int kernel,
                         int rr, const double* L, uint64_t seed) {
    const long vol = (long)N * N;
    double* z = (double*)malloc(sizeof(double) * 16 * vol);
    double* xx = (double*)malloc(sizeof(double) * 18 * vol);
    double* xy = (double*)malloc(sizeof(double) * 18 * vol);
    double* A = (double*)malloc(sizeof(double) * 18 * vol);
    double* B = (double*)malloc(sizeof(double) * 18 * vol);
    for (int s = 0; s < steps; ++s) {
        jwo_langevin_normals(seed, step0 + (uint64_t)s, N, z);
        jwo_generate_gaussian(z, xx, xy, N, 0);
        if (coupling == JWO_NOISE_COUPLING && L) {
            jwo_multiply_by_cholesky(L, xx, N);
            jwo_multiply_by_cholesky(L, xy, N);
        }
        jwo_prepare_A_and_B(A, B, xx, xy, V, N, rr, coupling, kernel);
        jwo_update_uf(V, B, A, N, step);
    }
    free(z); free(xx); free(xy); free(A); free(B);
}

void jwo_reduce_hatta(const double* corr, double* sum, double* err, int N, int xr, int yr) {
    long i = (long)xr * N + yr;
    cplx c = ld(corr, i);
    st(sum, i, ld(sum, i) + c);
    cplx sq = (cimag(c) == 0.0 && creal(c) > 0.0) ? CMPLX(pow(creal(c), 2.0), 0.0) : c * c;
    st(err, i, ld(err, i) + sq);
}

/* ======================= position-space dipole ======================= */

void jwo_dipole_position(const double* corr_sym, int N, double* S_xy) {
    const long vol = (long)N * N;
    double* c = (double*)malloc(sizeof(double) * 2 * vol);
    memcpy(c, corr_sym, sizeof(double) * 2 * vol);
    /* unitary backward transform times N: sum_k C(k) e^{+i...} = N * IFFT_unitary */
    jwo_execute2D(c, N, 1, 0);
    for (long i = 0; i < vol; ++i) S_xy[i] = ((double)N * N / 3.0) * ((double)N * c[2 * i]);
    free(c);
}

static int min_image(int d, int N) { return (d > N / 2) ? d - N : d; }

int jwo_dipole_radial(const double* S_xy, int N, double* S_b, double* r_b, int* count_b) {
    int nb = N / 2 + 1;
    for (int b = 0; b < nb; ++b) { S_b[b] = 0.0; r_b[b] = 0.0; count_b[b] = 0; }
    for (int x = 0; x < N; ++x)
        for (int y = 0; y < N; ++y) {
            int dx = min_image(x, N), dy = min_image(y, N);
            double r = sqrt((double)(dx * dx + dy * dy));
            int b = (int)floor(r + 0.5);
            if (b >= nb) continue;
            S_b[b] += S_xy[(long)x * N + y];
            r_b[b] += r;
            count_b[b] += 1;
        }
    for (int b = 0; b < nb; ++b)
        if (count_b[b]) { S_b[b] /= count_b[b]; r_b[b] /= count_b[b]; }
    return nb;
}

double jwo_saturation_scale(const double* S_b, const double* r_b, int nbins) {
    const double target = exp(-0.5);
    for (int b = 0; b + 1 < nbins; ++b) {
        if (S_b[b] >= target && S_b[b + 1] < target) {
            double t = (S_b[b] - target) / (S_b[b] - S_b[b + 1]);
            double rs = r_b[b] + t * (r_b[b + 1] - r_b[b]);
            return rs > 0.0 ? sqrt(2.0) / rs : 0.0;
        }
    }
    return 0.0;
}
