/* Test-only stand-in for an MPI installation (none exists here): the few
 * declarations include/isdf.hpp's MPI branch uses, at world size 1, so that
 * tests/test_abi.py can compile and link that branch. */
#ifndef ISDF_TEST_MPI_STUB_H
#define ISDF_TEST_MPI_STUB_H
#define MPI_VERSION 3
typedef int MPI_Comm;
typedef int MPI_Datatype;
#define MPI_COMM_WORLD 0
#define MPI_INT 4
#define MPI_BYTE 1
static inline int MPI_Comm_rank(MPI_Comm, int* r) { *r = 0; return 0; }
static inline int MPI_Comm_size(MPI_Comm, int* s) { *s = 1; return 0; }
static inline int MPI_Bcast(void*, int, MPI_Datatype, int, MPI_Comm) { return 0; }
#endif
