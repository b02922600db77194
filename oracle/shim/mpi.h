/*
 * Single-rank MPI stand-in — TEST INFRASTRUCTURE ONLY.
 *
 * Lets the reference's own translation units (src/mpi_manager.cpp,
 * src/array2d.cpp, src/diagnostics.cpp, src/integrals.cpp,
 * src/verification.cpp) compile and run as one MPI rank, which is the
 * configuration the B200 path replaces: MPI_Cart_shift returns
 * MPI_PROC_NULL for every neighbour, so the halo exchange is a no-op and the
 * ghost cells stay zero; reductions over one rank copy the input.
 * Project-written; not derived from any MPI implementation.
 */
#ifndef MPD_ORACLE_MPI_SHIM_H
#define MPD_ORACLE_MPI_SHIM_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int source, tag, error; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_PROC_NULL (-2)
#define MPI_DOUBLE 1
#define MPI_INT 2
#define MPI_CHAR 3
#define MPI_MAX 1
#define MPI_SUM 2
#define MPI_MIN 3
#define MPI_STATUS_IGNORE ((MPI_Status *)0)
#define MPI_STATUSES_IGNORE ((MPI_Status *)0)

static inline size_t mpd_shim_type_size(MPI_Datatype t) {
    return t == MPI_DOUBLE ? sizeof(double) : t == MPI_INT ? sizeof(int) : 1;
}

static inline int MPI_Init(int *, char ***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Comm_rank(MPI_Comm, int *rank) { *rank = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int *size) { *size = 1; return 0; }
static inline int MPI_Comm_free(MPI_Comm *comm) { *comm = MPI_COMM_NULL; return 0; }
static inline int MPI_Dims_create(int, int ndims, int *dims) {
    for (int i = 0; i < ndims; ++i)
        if (dims[i] <= 0) dims[i] = 1;
    return 0;
}
static inline int MPI_Cart_create(MPI_Comm, int, const int *, const int *, int, MPI_Comm *c) {
    *c = 0;
    return 0;
}
static inline int MPI_Cart_coords(MPI_Comm, int, int ndims, int *coords) {
    for (int i = 0; i < ndims; ++i) coords[i] = 0;
    return 0;
}
static inline int MPI_Cart_shift(MPI_Comm, int, int, int *src, int *dst) {
    *src = MPI_PROC_NULL;
    *dst = MPI_PROC_NULL;
    return 0;
}
static inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) {
    *r = 0;
    return 0;
}
static inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *r) {
    *r = 0;
    return 0;
}
static inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }
static inline int MPI_Allreduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    memcpy(out, in, (size_t)n * mpd_shim_type_size(t));
    return 0;
}
static inline int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    memcpy(out, in, (size_t)n * mpd_shim_type_size(t));
    return 0;
}
static inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
static inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) { return 0; }
static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}
static inline int MPI_Abort(MPI_Comm, int code) {
    fprintf(stderr, "MPI_Abort(%d) in single-rank oracle build\n", code);
    exit(code);
}

#endif
