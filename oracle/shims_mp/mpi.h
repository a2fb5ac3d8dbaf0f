/*
 * Test infrastructure only (oracle). A p-rank stand-in for the MPI API, wide
 * enough to compile the reference's CPU sources for the ISDF path and to run
 * its KMEAN (src/common/utility.cpp:631-988) as p ranks: each rank is a
 * process forked by oracle/ref_mp_driver.cpp, and the collectives go through
 * one shared-memory region (mpi_mp.cpp).
 *
 * Reduction order. MPI leaves the order in which MPI_Reduce / MPI_Allreduce
 * combine the ranks' contributions to the implementation. This shim combines
 * them as MPICH's binomial-tree reduce does for a commutative operation:
 * at step s = 1, 2, 4, ..., rank q (q a multiple of 2s) adds the partial of
 * rank q + s, so for 4 ranks the sum is (r0 + r1) + (r2 + r3) and for 3 ranks
 * (r0 + r1) + r2. At 2 ranks every implementation agrees (a + b = b + a).
 * MPI_MINLOC keeps the smaller value and, on equal values, the smaller index
 * (the MPI standard's rule). No product code includes this.
 */
#ifndef ISDF_ORACLE_SHIM_MPI_MP_H
#define ISDF_ORACLE_SHIM_MPI_MP_H

#include <stddef.h>

typedef int MPI_Comm;
typedef int MPI_Datatype;
typedef int MPI_Op;

#define MPI_COMM_WORLD 0
#define MPI_COMM_NULL (-1)

/* Datatype handles: the low byte is the element size in bytes. */
#define MPI_INT 4
#define MPI_DOUBLE 8
#define MPI_DOUBLE_COMPLEX 16
#define MPI_DOUBLE_INT 0x110 /* struct { double; int; } = 16 bytes */

#define MPI_SUM 1
#define MPI_MINLOC 2
#define MPI_MAX 3
#define MPI_MIN 4

#define MPI_IN_PLACE ((void*)1)

int MPI_Init(int*, char***);
int MPI_Finalize(void);
int MPI_Abort(MPI_Comm, int code);
int MPI_Comm_rank(MPI_Comm, int* r);
int MPI_Comm_size(MPI_Comm, int* s);
int MPI_Barrier(MPI_Comm);
int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out);
int MPI_Comm_free(MPI_Comm* c);
double MPI_Wtime(void);
int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm);
int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm);
int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op op, int root,
               MPI_Comm);
int MPI_Allgather(const void* send, int scount, MPI_Datatype st, void* recv, int rcount,
                  MPI_Datatype rt, MPI_Comm);
int MPI_Allgatherv(const void* send, int scount, MPI_Datatype st, void* recv, const int* rcounts,
                   const int* displs, MPI_Datatype rt, MPI_Comm);
int MPI_Alltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype st,
                  void* recv, const int* rcounts, const int* rdispls, MPI_Datatype rt, MPI_Comm);

/* Set up by the driver in each forked rank before it calls into the
   reference: the shared region and this process's rank. */
void isdf_shim_mp_attach(void* region, int rank);
/* Bytes of shared memory a run of `size` ranks with messages of up to
   `slot_bytes` bytes per rank needs. */
size_t isdf_shim_mp_region_bytes(int size, size_t slot_bytes);
/* Initialises the region (barrier, sizes) in the parent, before the fork. */
int isdf_shim_mp_init(void* region, int size, size_t slot_bytes);
void isdf_shim_mp_destroy(void* region);

#endif
