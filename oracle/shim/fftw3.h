/*
 * FFTW3-API shim (oracle test infrastructure only).
 *
 * The reference solver calls FFTW3 + FFTW3-MPI (mpi_fftw_class.h:56-352).
 * Neither library is present here, so the oracle compiles the reference's own
 * headers against this project-written replacement.  It provides exactly the
 * API surface mpi_fftw_class.h uses and computes the unnormalised discrete
 * Fourier transform with FFTW's conventions (FFTW docs, "What FFTW Really
 * Computes"):
 *     Y[k0,k1] = sum_{j0,j1} X[j0,j1] * exp(sign * 2*pi*i * (j0*k0/n0 + j1*k1/n1))
 * with sign = FFTW_FORWARD = -1 or FFTW_BACKWARD = +1, row-major n0 x n1, and
 * `howmany` interleaved transforms (element (j0,j1) of transform k at offset
 * (j0*n1 + j1)*howmany + k), which is FFTW's "many" layout with unit
 * inner stride between the transforms.
 *
 * Algorithm: iterative radix-2 Cooley-Tukey (decimation in time, bit-reversed
 * input order) for power-of-two lengths, and the direct O(n^2) sum otherwise.
 * Twiddles exp(sign*2*pi*i*k/n) are tabulated once per length with libm
 * cos/sin of 2*pi*k/n.  Rows are transformed first, then columns; with OpenMP
 * the lines are distributed over threads.  This is NOT FFTW: results agree
 * with FFTW to rounding (both are O(eps log n) accurate), not bit for bit.
 */
#ifndef JW_ORACLE_FFTW3_SHIM_H
#define JW_ORACLE_FFTW3_SHIM_H

#include <math.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef double fftw_complex[2];

struct jw_shim_plan {
    ptrdiff_t n0, n1, howmany;
    int sign;
    double* data; /* array the plan was created for (fftw_execute) */
};
typedef struct jw_shim_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_ESTIMATE (1U << 6)
#define FFTW_MEASURE (0U)

static inline int fftw_init_threads(void) { return 1; }
static inline void fftw_plan_with_nthreads(int n) { (void)n; }
static inline void fftw_cleanup_threads(void) {}
static inline fftw_complex* fftw_alloc_complex(size_t n) {
    return (fftw_complex*)calloc(n ? n : 1, sizeof(fftw_complex));
}
static inline void fftw_free(void* p) { free(p); }
static inline void fftw_destroy_plan(fftw_plan p) { free(p); }

/* ---- 1-D line transform on a contiguous buffer of n complex values ---- */
static inline int jw_shim_is_pow2(ptrdiff_t n) { return n > 0 && (n & (n - 1)) == 0; }

/* tw[2k], tw[2k+1] = cos, sign*sin of 2*pi*k/n, k < n */
static inline double* jw_shim_twiddles(ptrdiff_t n, int sign) {
    double* tw = (double*)malloc(sizeof(double) * 2 * (size_t)n);
    for (ptrdiff_t k = 0; k < n; ++k) {
        double a = 2.0 * M_PI * (double)k / (double)n;
        tw[2 * k] = cos(a);
        tw[2 * k + 1] = (double)sign * sin(a);
    }
    return tw;
}

static inline void jw_shim_line(double* x, ptrdiff_t n, const double* tw, double* scratch) {
    if (n <= 1) return;
    if (jw_shim_is_pow2(n)) {
        /* bit-reversal permutation */
        for (ptrdiff_t i = 1, j = 0; i < n; ++i) {
            ptrdiff_t bit = n >> 1;
            for (; j & bit; bit >>= 1) j ^= bit;
            j ^= bit;
            if (i < j) {
                double tr = x[2 * i], ti = x[2 * i + 1];
                x[2 * i] = x[2 * j]; x[2 * i + 1] = x[2 * j + 1];
                x[2 * j] = tr; x[2 * j + 1] = ti;
            }
        }
        for (ptrdiff_t len = 2; len <= n; len <<= 1) {
            ptrdiff_t half = len >> 1, step = n / len;
            for (ptrdiff_t s = 0; s < n; s += len) {
                for (ptrdiff_t k = 0; k < half; ++k) {
                    double wr = tw[2 * k * step], wi = tw[2 * k * step + 1];
                    double* a = x + 2 * (s + k);
                    double* b = x + 2 * (s + k + half);
                    double br = b[0] * wr - b[1] * wi;
                    double bi = b[0] * wi + b[1] * wr;
                    b[0] = a[0] - br; b[1] = a[1] - bi;
                    a[0] = a[0] + br; a[1] = a[1] + bi;
                }
            }
        }
    } else {
        for (ptrdiff_t k = 0; k < n; ++k) {
            double sr = 0.0, si = 0.0;
            for (ptrdiff_t j = 0; j < n; ++j) {
                ptrdiff_t m = (j * k) % n;
                double wr = tw[2 * m], wi = tw[2 * m + 1];
                sr += x[2 * j] * wr - x[2 * j + 1] * wi;
                si += x[2 * j] * wi + x[2 * j + 1] * wr;
            }
            scratch[2 * k] = sr; scratch[2 * k + 1] = si;
        }
        memcpy(x, scratch, sizeof(double) * 2 * (size_t)n);
    }
}

/* In-place 2-D transform of `howmany` interleaved n0 x n1 arrays. */
static inline void jw_shim_execute(const struct jw_shim_plan* p, double* d) {
    const ptrdiff_t n0 = p->n0, n1 = p->n1, h = p->howmany;
    double* tw1 = jw_shim_twiddles(n1, p->sign);
    double* tw0 = (n0 == n1) ? tw1 : jw_shim_twiddles(n0, p->sign);
    const ptrdiff_t nmax = n0 > n1 ? n0 : n1;
    /* rows: transform k, row j0, along j1 (stride h) */
#ifdef _OPENMP
#pragma omp parallel
#endif
    {
        double* buf = (double*)malloc(sizeof(double) * 4 * (size_t)nmax);
        double* scr = buf + 2 * nmax;
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (ptrdiff_t j0 = 0; j0 < n0; ++j0) {
            for (ptrdiff_t k = 0; k < h; ++k) {
                double* base = d + 2 * (j0 * n1 * h + k);
                for (ptrdiff_t j1 = 0; j1 < n1; ++j1) {
                    buf[2 * j1] = base[2 * j1 * h];
                    buf[2 * j1 + 1] = base[2 * j1 * h + 1];
                }
                jw_shim_line(buf, n1, tw1, scr);
                for (ptrdiff_t j1 = 0; j1 < n1; ++j1) {
                    base[2 * j1 * h] = buf[2 * j1];
                    base[2 * j1 * h + 1] = buf[2 * j1 + 1];
                }
            }
        }
        /* columns: transform k, column j1, along j0 (stride n1*h) */
#ifdef _OPENMP
#pragma omp for collapse(2) schedule(static)
#endif
        for (ptrdiff_t j1 = 0; j1 < n1; ++j1) {
            for (ptrdiff_t k = 0; k < h; ++k) {
                double* base = d + 2 * (j1 * h + k);
                for (ptrdiff_t j0 = 0; j0 < n0; ++j0) {
                    buf[2 * j0] = base[2 * j0 * n1 * h];
                    buf[2 * j0 + 1] = base[2 * j0 * n1 * h + 1];
                }
                jw_shim_line(buf, n0, tw0, scr);
                for (ptrdiff_t j0 = 0; j0 < n0; ++j0) {
                    base[2 * j0 * n1 * h] = buf[2 * j0];
                    base[2 * j0 * n1 * h + 1] = buf[2 * j0 + 1];
                }
            }
        }
        free(buf);
    }
    if (tw0 != tw1) free(tw0);
    free(tw1);
}

static inline void fftw_execute(const fftw_plan p) { jw_shim_execute(p, p->data); }

#endif
