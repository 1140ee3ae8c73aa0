/*
 * Single-rank stand-in for <mpi.h>, used only to compile the reference's
 * MPI-tree hot-path translation units into the CPU oracle library
 * (oracle/_ref).  This is test infrastructure, not product code.
 *
 * With one rank every collective the reference issues degenerates to a
 * copy of the caller's own contribution:
 *   - MPI_Allreduce (timestep min, MPI/compute_timestep.cpp:69,101; rung max,
 *     MPI/Scheduler.h:118,142-149; counts, MPI/iterate.cpp:124-126)
 *   - MPI_Alltoall of the per-peer counts (MPI/myMPI.h:122)
 *   - MPI_Allgather / MPI_Bcast (MPI/myMPI.h:236-262)
 * Point-to-point calls are never reached for nproc == 1 (MPI/myMPI.h:212-230
 * loops over dist = 1 .. nproc-1) and abort if they are.
 */
#ifndef FVM_REF_MPI_STUB_H
#define FVM_REF_MPI_STUB_H

#include <cstring>
#include <cstdlib>
#include <cstdio>

typedef int MPI_Datatype;
typedef int MPI_Comm;
typedef int MPI_Op;
typedef int MPI_Request;
typedef struct { int MPI_SOURCE, MPI_TAG, MPI_ERROR; } MPI_Status;

#define MPI_COMM_WORLD 0
#define MPI_SUCCESS 0
#define MPI_INT 1
#define MPI_FLOAT 2
#define MPI_DOUBLE 3
#define MPI_UNSIGNED_LONG_LONG 4
#define MPI_LONG_LONG 5
#define MPI_CHAR 6
#define MPI_BYTE 7
#define MPI_UNSIGNED 8
#define MPI_UNSIGNED_LONG 9
#define MPI_SUM 1
#define MPI_MIN 2
#define MPI_MAX 3
#define MPI_IN_PLACE ((void *)1)

/* sizes of derived (contiguous) types created by MPI_Type_contiguous */
namespace fvm_mpi_stub {
  enum { NTYPE = 64 };
  extern int type_size[NTYPE];
  extern int ntype;
  inline int size_of(MPI_Datatype t) {
    switch (t) {
      case MPI_INT: case MPI_FLOAT: case MPI_UNSIGNED: return 4;
      case MPI_DOUBLE: case MPI_UNSIGNED_LONG_LONG: case MPI_LONG_LONG: case MPI_UNSIGNED_LONG: return 8;
      case MPI_CHAR: case MPI_BYTE: return 1;
      default:
        if (t >= 16 && t < 16 + NTYPE) return type_size[t - 16];
        fprintf(stderr, "mpi stub: unknown datatype %d\n", t);
        abort();
    }
  }
  inline void unreachable(const char *what) {
    fprintf(stderr, "mpi stub: %s is not reachable with one rank\n", what);
    abort();
  }
}

inline int MPI_Init(int *, char ***) { return 0; }
inline int MPI_Finalize() { return 0; }
inline int MPI_Comm_size(MPI_Comm, int *n) { *n = 1; return 0; }
inline int MPI_Comm_rank(MPI_Comm, int *r) { *r = 0; return 0; }
inline int MPI_Barrier(MPI_Comm) { return 0; }
inline double MPI_Wtime() { return 0.0; }
inline int MPI_Abort(MPI_Comm, int code) { exit(code); }

inline int MPI_Allreduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, MPI_Comm) {
  if (s != MPI_IN_PLACE) memmove(r, s, (size_t)n * fvm_mpi_stub::size_of(t));
  return 0;
}
inline int MPI_Reduce(const void *s, void *r, int n, MPI_Datatype t, MPI_Op, int, MPI_Comm) {
  if (s != MPI_IN_PLACE) memmove(r, s, (size_t)n * fvm_mpi_stub::size_of(t));
  return 0;
}
inline int MPI_Alltoall(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  memmove(r, s, (size_t)n * fvm_mpi_stub::size_of(t));
  return 0;
}
inline int MPI_Allgather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, MPI_Comm) {
  memmove(r, s, (size_t)n * fvm_mpi_stub::size_of(t));
  return 0;
}
inline int MPI_Gather(const void *s, int n, MPI_Datatype t, void *r, int, MPI_Datatype, int, MPI_Comm) {
  memmove(r, s, (size_t)n * fvm_mpi_stub::size_of(t));
  return 0;
}
inline int MPI_Bcast(void *, int, MPI_Datatype, int, MPI_Comm) { return 0; }

inline int MPI_Type_contiguous(int n, MPI_Datatype old, MPI_Datatype *t) {
  using namespace fvm_mpi_stub;
  if (ntype >= NTYPE) unreachable("more than 64 derived datatypes");
  type_size[ntype] = n * size_of(old);
  *t = 16 + ntype++;
  return 0;
}
inline int MPI_Type_commit(MPI_Datatype *) { return 0; }
inline int MPI_Type_free(MPI_Datatype *t) { *t = 0; return 0; }

inline int MPI_Send(const void *, int, MPI_Datatype, int, int, MPI_Comm) {
  fvm_mpi_stub::unreachable("MPI_Send"); return 1;
}
inline int MPI_Recv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  fvm_mpi_stub::unreachable("MPI_Recv"); return 1;
}
inline int MPI_Sendrecv(const void *, int, MPI_Datatype, int, int,
                        void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Status *) {
  fvm_mpi_stub::unreachable("MPI_Sendrecv"); return 1;
}
inline int MPI_Isend(const void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  fvm_mpi_stub::unreachable("MPI_Isend"); return 1;
}
inline int MPI_Irecv(void *, int, MPI_Datatype, int, int, MPI_Comm, MPI_Request *) {
  fvm_mpi_stub::unreachable("MPI_Irecv"); return 1;
}
inline int MPI_Waitall(int, MPI_Request *, MPI_Status *) { return 0; }

#endif
