/*
 * Test infrastructure only (oracle). A single-rank stand-in for the MPI API,
 * just wide enough to compile the reference's CPU sources for the ISDF path
 * (src/common/utility.cpp, src/cpu/getpoints_Kmeans_MPI.cpp,
 * src/cpu/getbasis_MPI.cpp, src/common/checkcode.cpp) as one rank.
 *
 * Semantics at world size 1: every collective is a copy from the send buffer
 * to the receive buffer (MPI_IN_PLACE leaves the buffer as it is), Bcast and
 * Barrier do nothing, rank = 0 and size = 1. No product code includes this.
 */
#ifndef ISDF_ORACLE_SHIM_MPI_H
#define ISDF_ORACLE_SHIM_MPI_H

#include <string.h>
#include <time.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)

/* Datatype handles encode the element size in bytes. */
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_DOUBLE_COMPLEX 16
#define MPI_DOUBLE_INT 0x110 /* struct { double; int; } = 16 bytes */

#define MPI_SUM 1
#define MPI_MINLOC 2
#define MPI_MAX 3
#define MPI_MIN 4

#define MPI_IN_PLACE ((void*)1)

static inline size_t isdf_shim_type_size(MPI_Datatype t) {
  return t == MPI_DOUBLE_INT ? 16u : (size_t)t;
}

static inline int MPI_Init(int*, char***) { return 0; }
static inline int MPI_Finalize(void) { return 0; }
static inline int MPI_Abort(MPI_Comm, int code) { return code; }
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Barrier(MPI_Comm) { return 0; }
static inline int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) { *out = c; return 0; }
static inline int MPI_Comm_free(MPI_Comm* c) { *c = MPI_COMM_NULL; return 0; }

static inline double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }

static inline int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op,
                                MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv)
    memmove(recv, send, (size_t)count * isdf_shim_type_size(t));
  return 0;
}

static inline int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op, int,
                             MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv)
    memmove(recv, send, (size_t)count * isdf_shim_type_size(t));
  return 0;
}

static inline int MPI_Allgather(const void* send, int scount, MPI_Datatype st, void* recv, int,
                                MPI_Datatype, MPI_Comm) {
  if (send != MPI_IN_PLACE && send != recv)
    memmove(recv, send, (size_t)scount * isdf_shim_type_size(st));
  return 0;
}

static inline int MPI_Allgatherv(const void* send, int scount, MPI_Datatype st, void* recv,
                                 const int*, const int* displs, MPI_Datatype rt, MPI_Comm) {
  if (send != MPI_IN_PLACE)
    memmove((char*)recv + (size_t)displs[0] * isdf_shim_type_size(rt), send,
            (size_t)scount * isdf_shim_type_size(st));
  return 0;
}

static inline int MPI_Alltoallv(const void* send, const int* scounts, const int* sdispls,
                                MPI_Datatype st, void* recv, const int*, const int* rdispls,
                                MPI_Datatype rt, MPI_Comm) {
  memmove((char*)recv + (size_t)rdispls[0] * isdf_shim_type_size(rt),
          (const char*)send + (size_t)sdispls[0] * isdf_shim_type_size(st),
          (size_t)scounts[0] * isdf_shim_type_size(st));
  return 0;
}

#endif
