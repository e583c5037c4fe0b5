/*
 * FFTW3-MPI API shim (oracle test infrastructure only): the single-rank
 * counterpart of the calls in mpi_fftw_class.h:134-189 and :231-295.  With one
 * rank the local slab is the whole array (local_n0 = n0, local_0_start = 0)
 * and a distributed plan is an ordinary in-place 2-D plan; the transform
 * itself is the one in fftw3.h.
 */
#ifndef JW_ORACLE_FFTW3_MPI_SHIM_H
#define JW_ORACLE_FFTW3_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "fftw3.h"
#include "mpi.h"

#define FFTW_MPI_DEFAULT_BLOCK ((ptrdiff_t)0)

static inline void fftw_mpi_init(void) {}

static inline ptrdiff_t fftw_mpi_local_size_2d(ptrdiff_t n0, ptrdiff_t n1, MPI_Comm c,
                                               ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
    (void)c;
    *local_n0 = n0;
    *local_0_start = 0;
    return n0 * n1;
}

static inline ptrdiff_t fftw_mpi_local_size_many(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                                 ptrdiff_t block0, MPI_Comm c,
                                                 ptrdiff_t* local_n0, ptrdiff_t* local_0_start) {
    (void)block0; (void)c;
    if (rnk != 2) { fprintf(stderr, "fftw shim: only rank-2 transforms\n"); abort(); }
    *local_n0 = n[0];
    *local_0_start = 0;
    return n[0] * n[1] * howmany;
}

static inline fftw_plan jw_shim_make_plan(ptrdiff_t n0, ptrdiff_t n1, ptrdiff_t howmany,
                                          fftw_complex* in, fftw_complex* out, int sign) {
    if (in != out) { fprintf(stderr, "fftw shim: only in-place plans\n"); abort(); }
    fftw_plan p = (fftw_plan)malloc(sizeof(struct jw_shim_plan));
    p->n0 = n0; p->n1 = n1; p->howmany = howmany; p->sign = sign;
    p->data = (double*)in;
    return p;
}

static inline fftw_plan fftw_mpi_plan_dft_2d(ptrdiff_t n0, ptrdiff_t n1, fftw_complex* in,
                                             fftw_complex* out, MPI_Comm c, int sign,
                                             unsigned flags) {
    (void)c; (void)flags;
    return jw_shim_make_plan(n0, n1, 1, in, out, sign);
}

static inline fftw_plan fftw_mpi_plan_many_dft(int rnk, const ptrdiff_t* n, ptrdiff_t howmany,
                                               ptrdiff_t block, ptrdiff_t tblock,
                                               fftw_complex* in, fftw_complex* out,
                                               MPI_Comm c, int sign, unsigned flags) {
    (void)block; (void)tblock; (void)c; (void)flags;
    if (rnk != 2) { fprintf(stderr, "fftw shim: only rank-2 transforms\n"); abort(); }
    return jw_shim_make_plan(n[0], n[1], howmany, in, out, sign);
}

static inline void fftw_mpi_execute_dft(const fftw_plan p, fftw_complex* in, fftw_complex* out) {
    if (in != out) memcpy(out, in, sizeof(fftw_complex) * (size_t)(p->n0 * p->n1 * p->howmany));
    jw_shim_execute(p, (double*)out);
}

#endif
