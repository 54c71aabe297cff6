/*
 * Single-rank mpi.h stub (test infrastructure only).
 *
 * Lets the reference's MPI-path headers (lobpcg_d_multi_mpi.h,
 * lobpcg_z_multi_mpi.h, GridDifferenceKpoint8th.h, mpi_helper.h) compile and
 * run as ONE rank without an MPI library: every communicator has size 1 and
 * rank 0, reductions and gathers copy send to receive, broadcasts do nothing,
 * and a send/receive pair with itself copies the message.
 */
#pragma once
#include <cstdint>
#include <cstring>
#include <cstddef>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct MPI_Status { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 1
#define MPI_COMM_SELF 2
#define MPI_COMM_NULL 0
#define MPI_SUCCESS 0
#define MPI_UNDEFINED (-32766)
#define MPI_ANY_SOURCE (-2)
#define MPI_ANY_TAG (-1)
#define MPI_PROC_NULL (-3)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_REQUEST_NULL 0
#define MPI_IN_PLACE ((void*)1)

#define MPI_DATATYPE_NULL 0
#define MPI_BYTE 1
#define MPI_CHAR 1
#define MPI_C_BOOL 1
#define MPI_INT 4
#define MPI_UINT 4
#define MPI_UNSIGNED 4
#define MPI_FLOAT 4
#define MPI_INT64_T 8
#define MPI_UINT64_T 8
#define MPI_UINT8_T 1
#define MPI_LONG_LONG 8
#define MPI_DOUBLE 8
#define MPI_DOUBLE_COMPLEX 16
#define MPI_C_DOUBLE_COMPLEX 16

#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_BOR 4
#define MPI_LOR 5

inline size_t qg_mpi_stub_bytes(int count, MPI_Datatype t) { return (size_t)count * (size_t)t; }
inline void qg_mpi_stub_copy(const void* s, void* r, int count, MPI_Datatype t) {
    if (s == MPI_IN_PLACE || s == r || count <= 0) return;
    std::memmove(r, s, qg_mpi_stub_bytes(count, t));
}

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_split(MPI_Comm c, int color, int, MPI_Comm* out) { *out = (color == MPI_UNDEFINED) ? MPI_COMM_NULL : c; return 0; }
inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) { qg_mpi_stub_copy(s, r, n, t); return 0; }
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) { qg_mpi_stub_copy(s, r, n, t); return 0; }
inline int MPI_Iallreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm, MPI_Request* q) { qg_mpi_stub_copy(s, r, n, t); if (q) *q = 0; return 0; }
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Sendrecv(const void* s, int sn, MPI_Datatype st, int, int, void* r, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { qg_mpi_stub_copy(s, r, sn, st); return 0; }
inline int MPI_Sendrecv_replace(void*, int, MPI_Datatype, int, int, int, int, MPI_Comm, MPI_Status*) { return 0; }
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { return 0; }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { return 0; }
inline int MPI_Gather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, int, MPI_Comm) { qg_mpi_stub_copy(s, r, sn, st); return 0; }
inline int MPI_Allgather(const void* s, int sn, MPI_Datatype st, void* r, int, MPI_Datatype, MPI_Comm) { qg_mpi_stub_copy(s, r, sn, st); return 0; }
inline int MPI_Gatherv(const void* s, int sn, MPI_Datatype st, void* r, const int*, const int* displs, MPI_Datatype, int, MPI_Comm) {
    qg_mpi_stub_copy(s, (char*)r + (displs ? (size_t)displs[0] * st : 0), sn, st); return 0; }
inline int MPI_Scatter(const void* s, int, MPI_Datatype, void* r, int rn, MPI_Datatype rt, int, MPI_Comm) { qg_mpi_stub_copy(s, r, rn, rt); return 0; }
inline int MPI_Scatterv(const void* s, const int*, const int* displs, MPI_Datatype, void* r, int rn, MPI_Datatype rt, int, MPI_Comm) {
    qg_mpi_stub_copy((const char*)s + (displs ? (size_t)displs[0] * rt : 0), r, rn, rt); return 0; }
inline double MPI_Wtime() { return 0.0; }
