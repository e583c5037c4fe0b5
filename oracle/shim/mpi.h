/*
 * Single-rank MPI shim (oracle test infrastructure only).
 *
 * The reference solver is written against MPI (mpi_class.h:63-85, mpi_init.cpp,
 * field.h:535-591).  This container has no MPI, so the oracle compiles the
 * reference's own headers against this header instead.  Every call behaves as
 * MPI would on a communicator of size 1:
 *   - MPI_Init_thread / MPI_Finalize: no-ops, provided = requested level;
 *   - MPI_Comm_size = 1, MPI_Comm_rank = 0;
 *   - MPI_Allgather: one contribution, i.e. a copy of sendbuf into recvbuf;
 *   - MPI_Barrier, MPI_Comm_split: no-ops (split returns the same comm);
 *   - MPI_Send / MPI_Recv: never reached on one rank (the halo exchange in
 *     field.h:593-681 is dead code); they abort loudly if called.
 * Nothing here is used by the product library.
 */
#ifndef JW_ORACLE_MPI_SHIM_H
#define JW_ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD ((MPI_Comm)0)
#define MPI_DOUBLE ((MPI_Datatype)8)
#define MPI_INT ((MPI_Datatype)4)
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

static inline int MPI_Init_thread(int* argc, char*** argv, int required, int* provided) {
    (void)argc; (void)argv;
    if (provided) *provided = required;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm c, int* size) { (void)c; *size = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_rank(MPI_Comm c, int* rank) { (void)c; *rank = 0; return MPI_SUCCESS; }
static inline int MPI_Barrier(MPI_Comm c) { (void)c; return MPI_SUCCESS; }
static inline int MPI_Comm_split(MPI_Comm c, int color, int key, MPI_Comm* out) {
    (void)color; (void)key; *out = c; return MPI_SUCCESS;
}
/* The datatype handle is the element size in bytes. */
static inline int MPI_Allgather(const void* sendbuf, int sendcount, MPI_Datatype st,
                                void* recvbuf, int recvcount, MPI_Datatype rt, MPI_Comm c) {
    (void)recvcount; (void)rt; (void)c;
    memmove(recvbuf, sendbuf, (size_t)sendcount * (size_t)st);
    return MPI_SUCCESS;
}
static inline int MPI_Send(const void* b, int n, MPI_Datatype t, int dest, int tag, MPI_Comm c) {
    (void)b; (void)n; (void)t; (void)dest; (void)tag; (void)c;
    fprintf(stderr, "mpi shim: MPI_Send is not available on a single rank\n");
    abort();
}
static inline int MPI_Recv(void* b, int n, MPI_Datatype t, int src, int tag, MPI_Comm c, MPI_Status* s) {
    (void)b; (void)n; (void)t; (void)src; (void)tag; (void)c; (void)s;
    fprintf(stderr, "mpi shim: MPI_Recv is not available on a single rank\n");
    abort();
}

#endif
