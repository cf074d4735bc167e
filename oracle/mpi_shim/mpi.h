/*
 * Single-rank MPI shim for building the reference solver on one CPU process.
 *
 * Test infrastructure only (part of the oracle build, never linked into the
 * product library).  It implements the subset of the MPI-3 C API that the
 * reference sources use (names and signatures from the MPI standard) with
 * the semantics of a communicator of size 1:
 *   - every collective degenerates to a copy of the caller's send buffer into
 *     its receive buffer (nothing when the send buffer is MPI_IN_PLACE);
 *   - MPI_Exscan leaves the receive buffer untouched, as the standard leaves
 *     it undefined on rank 0;
 *   - point-to-point calls are never reached with zero neighbours and abort
 *     loudly if they are;
 *   - MPI_Wtime returns a monotonic wall clock.
 * A datatype encodes a small type id in bits 8.. and its byte size in bits 0..7
 * so that distinct types compare unequal while sizes stay recoverable.
 */
#ifndef CFDG_ORACLE_MPI_SHIM_H
#define CFDG_ORACLE_MPI_SHIM_H

#include <stddef.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#ifdef __cplusplus
extern "C++" {
#endif

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef int MPI_Info;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_SUCCESS 0
#define MPI_COMM_NULL 0
#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_INFO_NULL 0
#define MPI_REQUEST_NULL 0
#define MPI_UNDEFINED (-32766)
#define MPI_IDENT 0
#define MPI_CONGRUENT 1
#define MPI_SIMILAR 2
#define MPI_UNEQUAL 3
#define MPI_COMM_TYPE_SHARED 1
#define MPI_THREAD_SINGLE 0
#define MPI_THREAD_FUNNELED 1
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_IN_PLACE ((void*)-1)

#define CFDG_SHIM_TYPE(id, size) (((id) << 8) | (size))
#define MPI_BYTE          CFDG_SHIM_TYPE(1, 1)
#define MPI_CHAR          CFDG_SHIM_TYPE(2, 1)
#define MPI_INT           CFDG_SHIM_TYPE(3, 4)
#define MPI_INT32_T       CFDG_SHIM_TYPE(4, 4)
#define MPI_INT64_T       CFDG_SHIM_TYPE(5, 8)
#define MPI_UINT64_T      CFDG_SHIM_TYPE(6, 8)
#define MPI_LONG_LONG_INT CFDG_SHIM_TYPE(7, 8)
#define MPI_DOUBLE        CFDG_SHIM_TYPE(8, 8)
#define MPI_UNSIGNED_LONG_LONG CFDG_SHIM_TYPE(9, 8)
#define MPI_LONG_LONG     MPI_LONG_LONG_INT

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_LAND 4
#define MPI_LOR 5

static inline size_t cfdg_shim_size(MPI_Datatype t) { return (size_t)(t & 0xff); }

static inline void cfdg_shim_copy(const void* s, void* r, int count, MPI_Datatype t) {
    if (s == MPI_IN_PLACE || s == r || count <= 0) return;
    memcpy(r, s, (size_t)count * cfdg_shim_size(t));
}

static inline void cfdg_shim_unreachable(const char* what) {
    fprintf(stderr, "mpi shim: %s needs a peer rank; the single-rank shim has none\n", what);
    abort();
}

static inline int MPI_Init(int*, char***) { return MPI_SUCCESS; }
static inline int MPI_Init_thread(int*, char***, int, int* provided) {
    if (provided) *provided = MPI_THREAD_FUNNELED;
    return MPI_SUCCESS;
}
static inline int MPI_Finalize(void) { return MPI_SUCCESS; }
static inline int MPI_Initialized(int* flag) { *flag = 1; return MPI_SUCCESS; }
static inline int MPI_Abort(MPI_Comm, int code) {
    fprintf(stderr, "mpi shim: MPI_Abort(%d)\n", code);
    fflush(stderr);
    abort();
    return code;
}
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return MPI_SUCCESS; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return MPI_SUCCESS; }
static inline int MPI_Comm_dup(MPI_Comm c, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return MPI_SUCCESS; }
static inline int MPI_Comm_compare(MPI_Comm a, MPI_Comm b, int* res) {
    *res = (a == b) ? MPI_IDENT : MPI_CONGRUENT;
    return MPI_SUCCESS;
}
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return MPI_SUCCESS; }
static inline int MPI_Comm_split_type(MPI_Comm c, int, int, MPI_Info, MPI_Comm* out) {
    *out = c;
    return MPI_SUCCESS;
}
static inline int MPI_Barrier(MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return MPI_SUCCESS; }
static inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
    cfdg_shim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
    cfdg_shim_copy(s, r, n, t);
    return MPI_SUCCESS;
}
static inline int MPI_Exscan(const void*, void*, int, MPI_Datatype, MPI_Op, MPI_Comm) {
    return MPI_SUCCESS;
}
static inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    cfdg_shim_copy(s, r, sn, st);
    return MPI_SUCCESS;
}
static inline int MPI_Alltoall(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) {
    cfdg_shim_copy(s, r, sn, st);
    return MPI_SUCCESS;
}
static inline int MPI_Alltoallv(const void* s, const int* sc, const int* sd, MPI_Datatype st,
                                void* r, const int*, const int* rd, MPI_Datatype, MPI_Comm) {
    if (s == MPI_IN_PLACE) return MPI_SUCCESS;
    const size_t es = cfdg_shim_size(st);
    if (sc[0] > 0) memcpy((char*)r + (size_t)rd[0] * es, (const char*)s + (size_t)sd[0] * es, (size_t)sc[0] * es);
    return MPI_SUCCESS;
}
static inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    cfdg_shim_unreachable("MPI_Isend");
    return 1;
}
static inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) {
    cfdg_shim_unreachable("MPI_Irecv");
    return 1;
}
static inline int MPI_Sendrecv(const void*, int, MPI_Datatype, int, int, void*, int, MPI_Datatype, int, int,
                               MPI_Comm, MPI_Status*) {
    cfdg_shim_unreachable("MPI_Sendrecv");
    return 1;
}
static inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return MPI_SUCCESS; }
static inline double MPI_Wtime(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

#ifdef __cplusplus
}
#endif

#endif
