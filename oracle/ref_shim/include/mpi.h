/*
 * Single-rank stand-in for the MPI API, used only to compile the reference
 * M2C sources in place as a CPU oracle (test infrastructure, not product code).
 *
 * Semantics: one process, rank 0, size 1. Collectives copy send -> receive
 * buffers (or do nothing with MPI_IN_PLACE); point-to-point calls are never
 * reached on one rank and abort if they are.
 */
#ifndef M2C_ORACLE_MPI_SHIM_H
#define M2C_ORACLE_MPI_SHIM_H

#include <cstdio>
#include <cstdlib>
#include <cstring>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)
#define MPI_INT 4
#define MPI_INTEGER 4
#define MPI_DOUBLE 8
#define MPI_CHAR 1
#define MPI_SUM 1
#define MPI_MAX 2
#define MPI_MIN 3
#define MPI_ANY_SOURCE (-1)
#define MPI_ANY_TAG (-1)
#define MPI_IN_PLACE ((void*)1)
#define MPI_STATUS_IGNORE ((MPI_Status*)0)
#define MPI_STATUSES_IGNORE ((MPI_Status*)0)
#define MPI_SUCCESS 0

namespace m2c_mpi_shim {
inline size_t type_size(MPI_Datatype t) { return (size_t)t; }
[[noreturn]] inline void unreachable(const char* what) {
  fprintf(stderr, "mpi shim: %s is not available on one rank\n", what);
  abort();
}
inline void copy(const void* s, void* r, int n, MPI_Datatype t) {
  if (s != MPI_IN_PLACE && s != r && n > 0) memcpy(r, s, (size_t)n * type_size(t));
}
}  // namespace m2c_mpi_shim

inline int MPI_Init(int*, char***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Abort(MPI_Comm, int code) { exit(code); }
inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
inline int MPI_Comm_remote_size(MPI_Comm, int* s) { *s = 0; return 0; }
inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* n) { *n = c; return 0; }
inline int MPI_Comm_free(MPI_Comm*) { return 0; }
inline int MPI_Intercomm_create(MPI_Comm, int, MPI_Comm, int, int, MPI_Comm*) {
  m2c_mpi_shim::unreachable("MPI_Intercomm_create");
}
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
inline int MPI_Allreduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  m2c_mpi_shim::copy(s, r, n, t); return 0;
}
inline int MPI_Reduce(const void* s, void* r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  m2c_mpi_shim::copy(s, r, n, t); return 0;
}
inline int MPI_Allgather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, MPI_Comm) {
  m2c_mpi_shim::copy(s, r, n, t); return 0;
}
inline int MPI_Gather(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
  m2c_mpi_shim::copy(s, r, n, t); return 0;
}
inline int MPI_Allgatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d,
                          MPI_Datatype, MPI_Comm) {
  if (s != MPI_IN_PLACE) m2c_mpi_shim::copy(s, (char*)r + (size_t)d[0] * t, n, t);
  return 0;
}
inline int MPI_Gatherv(const void* s, int n, MPI_Datatype t, void* r, const int*, const int* d,
                       MPI_Datatype, int, MPI_Comm) {
  if (s != MPI_IN_PLACE) m2c_mpi_shim::copy(s, (char*)r + (size_t)d[0] * t, n, t);
  return 0;
}
inline int MPI_Scatter(const void* s, int n, MPI_Datatype t, void* r, int, MPI_Datatype, int, MPI_Comm) {
  if (r != MPI_IN_PLACE) m2c_mpi_shim::copy(s, r, n, t);
  return 0;
}
inline int MPI_Scatterv(const void* s, const int*, const int* d, MPI_Datatype t, void* r, int n,
                        MPI_Datatype, int, MPI_Comm) {
  if (r != MPI_IN_PLACE) m2c_mpi_shim::copy((const char*)s + (size_t)d[0] * t, r, n, t);
  return 0;
}
inline int MPI_Send(const void*, int, MPI_Datatype, int, int, MPI_Comm) { m2c_mpi_shim::unreachable("MPI_Send"); }
inline int MPI_Recv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status*) { m2c_mpi_shim::unreachable("MPI_Recv"); }
inline int MPI_Isend(const void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { m2c_mpi_shim::unreachable("MPI_Isend"); }
inline int MPI_Irecv(void*, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request*) { m2c_mpi_shim::unreachable("MPI_Irecv"); }
inline int MPI_Wait(MPI_Request*, MPI_Status*) { return 0; }
inline int MPI_Waitall(int, MPI_Request*, MPI_Status*) { return 0; }

#endif
