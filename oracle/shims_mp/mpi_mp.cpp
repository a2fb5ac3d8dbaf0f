// Test infrastructure only (oracle). The p-rank MPI stand-in declared in
// mpi.h of this directory: ranks are processes forked by
// oracle/ref_mp_driver.cpp that share one anonymous MAP_SHARED region. Every
// collective copies the rank's contribution into its slot, meets the others
// at a process-shared barrier, and reads what it needs. Reductions combine
// the slots in binomial-tree order (see mpi.h). A message larger than a slot
// ends the rank with exit status 3.
#include "mpi.h"

#include <pthread.h>
#include <stdio.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include <algorithm>

namespace {

struct Header {
  pthread_barrier_t bar;
  int size;
  size_t slot;  // bytes per rank slot (after its 2 * size int header)
};

Header* g_hdr = nullptr;
int g_rank = 0;

size_t elem_size(MPI_Datatype t) { return t == MPI_DOUBLE_INT ? 16u : (size_t)(t & 0xff); }

size_t slot_stride(int size, size_t slot) {
  return ((2 * (size_t)size * sizeof(int) + slot) + 63) & ~(size_t)63;
}

char* slot_base(int q) {
  char* first = reinterpret_cast<char*>(g_hdr) + ((sizeof(Header) + 63) & ~(size_t)63);
  return first + (size_t)q * slot_stride(g_hdr->size, g_hdr->slot);
}
int* slot_ints(int q) { return reinterpret_cast<int*>(slot_base(q)); }
char* slot_data(int q) { return slot_base(q) + 2 * (size_t)g_hdr->size * sizeof(int); }

void fail(const char* what, size_t bytes) {
  fprintf(stderr, "mpi shim rank %d: %s of %zu bytes exceeds the slot (%zu)\n", g_rank, what,
          bytes, g_hdr ? g_hdr->slot : (size_t)0);
  _exit(3);
}

void barrier() {
  if (g_hdr && g_hdr->size > 1) pthread_barrier_wait(&g_hdr->bar);
}

struct DoubleInt {
  double v;
  int i;
};

void combine(char* d, const char* s, int count, MPI_Datatype t, MPI_Op op) {
  if (t == MPI_DOUBLE) {
    double* a = reinterpret_cast<double*>(d);
    const double* b = reinterpret_cast<const double*>(s);
    for (int i = 0; i < count; ++i) {
      if (op == MPI_SUM) a[i] = a[i] + b[i];
      else if (op == MPI_MAX) a[i] = std::max(a[i], b[i]);
      else if (op == MPI_MIN) a[i] = std::min(a[i], b[i]);
    }
  } else if (t == MPI_INT) {
    int* a = reinterpret_cast<int*>(d);
    const int* b = reinterpret_cast<const int*>(s);
    for (int i = 0; i < count; ++i) {
      if (op == MPI_SUM) a[i] = a[i] + b[i];
      else if (op == MPI_MAX) a[i] = std::max(a[i], b[i]);
      else if (op == MPI_MIN) a[i] = std::min(a[i], b[i]);
    }
  } else if (t == MPI_DOUBLE_COMPLEX) {
    double* a = reinterpret_cast<double*>(d);
    const double* b = reinterpret_cast<const double*>(s);
    for (int i = 0; i < 2 * count; ++i) a[i] = a[i] + b[i];
  } else if (t == MPI_DOUBLE_INT) {
    DoubleInt* a = reinterpret_cast<DoubleInt*>(d);
    const DoubleInt* b = reinterpret_cast<const DoubleInt*>(s);
    for (int i = 0; i < count; ++i) {
      if (b[i].v < a[i].v) a[i] = b[i];
      else if (b[i].v == a[i].v && b[i].i < a[i].i) a[i].i = b[i].i;
    }
  }
}

// Binomial tree over ranks relative to root: at step s, relative rank q
// (a multiple of 2s) takes in relative rank q + s. The result is left in
// root's slot.
void tree_reduce(int count, MPI_Datatype t, MPI_Op op, int root) {
  const int p = g_hdr->size;
  for (int s = 1; s < p; s *= 2)
    for (int q = 0; q + s < p; q += 2 * s)
      combine(slot_data((q + root) % p), slot_data((q + s + root) % p), count, t, op);
}

}  // namespace

void isdf_shim_mp_attach(void* region, int rank) {
  g_hdr = reinterpret_cast<Header*>(region);
  g_rank = rank;
}

size_t isdf_shim_mp_region_bytes(int size, size_t slot_bytes) {
  return ((sizeof(Header) + 63) & ~(size_t)63) + (size_t)size * slot_stride(size, slot_bytes);
}

int isdf_shim_mp_init(void* region, int size, size_t slot_bytes) {
  Header* h = reinterpret_cast<Header*>(region);
  h->size = size;
  h->slot = slot_bytes;
  pthread_barrierattr_t at;
  if (pthread_barrierattr_init(&at)) return -1;
  if (pthread_barrierattr_setpshared(&at, PTHREAD_PROCESS_SHARED)) return -1;
  int rc = pthread_barrier_init(&h->bar, &at, (unsigned)size);
  pthread_barrierattr_destroy(&at);
  return rc ? -1 : 0;
}

void isdf_shim_mp_destroy(void* region) {
  pthread_barrier_destroy(&reinterpret_cast<Header*>(region)->bar);
}

int MPI_Init(int*, char***) { return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Abort(MPI_Comm, int code) {
  _exit(code ? code : 1);
}
int MPI_Comm_rank(MPI_Comm, int* r) {
  *r = g_hdr ? g_rank : 0;
  return 0;
}
int MPI_Comm_size(MPI_Comm, int* s) {
  *s = g_hdr ? g_hdr->size : 1;
  return 0;
}
int MPI_Barrier(MPI_Comm) {
  barrier();
  return 0;
}
int MPI_Comm_split(MPI_Comm c, int, int, MPI_Comm* out) {
  *out = c;
  return 0;
}
int MPI_Comm_free(MPI_Comm* c) {
  *c = MPI_COMM_NULL;
  return 0;
}
double MPI_Wtime(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

int MPI_Bcast(void* buf, int count, MPI_Datatype t, int root, MPI_Comm) {
  if (!g_hdr || g_hdr->size == 1) return 0;
  const size_t bytes = (size_t)count * elem_size(t);
  if (bytes > g_hdr->slot) fail("MPI_Bcast", bytes);
  if (g_rank == root) memcpy(slot_data(root), buf, bytes);
  barrier();
  if (g_rank != root) memcpy(buf, slot_data(root), bytes);
  barrier();
  return 0;
}

int MPI_Reduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op op, int root,
               MPI_Comm) {
  const size_t bytes = (size_t)count * elem_size(t);
  const void* src = send == MPI_IN_PLACE ? recv : send;
  if (!g_hdr || g_hdr->size == 1) {
    if (src != recv) memmove(recv, src, bytes);
    return 0;
  }
  if (bytes > g_hdr->slot) fail("MPI_Reduce", bytes);
  memcpy(slot_data(g_rank), src, bytes);
  barrier();
  if (g_rank == root) {
    tree_reduce(count, t, op, root);
    memcpy(recv, slot_data(root), bytes);
  }
  barrier();
  return 0;
}

int MPI_Allreduce(const void* send, void* recv, int count, MPI_Datatype t, MPI_Op op, MPI_Comm) {
  const size_t bytes = (size_t)count * elem_size(t);
  const void* src = send == MPI_IN_PLACE ? recv : send;
  if (!g_hdr || g_hdr->size == 1) {
    if (src != recv) memmove(recv, src, bytes);
    return 0;
  }
  if (bytes > g_hdr->slot) fail("MPI_Allreduce", bytes);
  memcpy(slot_data(g_rank), src, bytes);
  barrier();
  if (g_rank == 0) tree_reduce(count, t, op, 0);
  barrier();
  memcpy(recv, slot_data(0), bytes);
  barrier();
  return 0;
}

int MPI_Allgather(const void* send, int scount, MPI_Datatype st, void* recv, int rcount,
                  MPI_Datatype rt, MPI_Comm) {
  const size_t rb = (size_t)rcount * elem_size(rt);
  const void* src = send == MPI_IN_PLACE ? (const char*)recv + (size_t)g_rank * rb : send;
  const size_t sb = send == MPI_IN_PLACE ? rb : (size_t)scount * elem_size(st);
  if (!g_hdr || g_hdr->size == 1) {
    if (src != recv) memmove(recv, src, sb);
    return 0;
  }
  if (sb > g_hdr->slot) fail("MPI_Allgather", sb);
  memcpy(slot_data(g_rank), src, sb);
  barrier();
  for (int q = 0; q < g_hdr->size; ++q) memcpy((char*)recv + (size_t)q * rb, slot_data(q), rb);
  barrier();
  return 0;
}

int MPI_Allgatherv(const void* send, int scount, MPI_Datatype st, void* recv, const int* rcounts,
                   const int* displs, MPI_Datatype rt, MPI_Comm) {
  const size_t re = elem_size(rt);
  const void* src = send == MPI_IN_PLACE ? (const char*)recv + (size_t)displs[g_rank] * re : send;
  const size_t sb =
      send == MPI_IN_PLACE ? (size_t)rcounts[g_rank] * re : (size_t)scount * elem_size(st);
  if (!g_hdr || g_hdr->size == 1) {
    memmove((char*)recv + (size_t)displs[0] * re, src, sb);
    return 0;
  }
  if (sb > g_hdr->slot) fail("MPI_Allgatherv", sb);
  memcpy(slot_data(g_rank), src, sb);
  barrier();
  for (int q = 0; q < g_hdr->size; ++q)
    memcpy((char*)recv + (size_t)displs[q] * re, slot_data(q), (size_t)rcounts[q] * re);
  barrier();
  return 0;
}

int MPI_Alltoallv(const void* send, const int* scounts, const int* sdispls, MPI_Datatype st,
                  void* recv, const int* rcounts, const int* rdispls, MPI_Datatype rt, MPI_Comm) {
  const size_t se = elem_size(st), re = elem_size(rt);
  if (!g_hdr || g_hdr->size == 1) {
    memmove((char*)recv + (size_t)rdispls[0] * re, (const char*)send + (size_t)sdispls[0] * se,
            (size_t)scounts[0] * se);
    return 0;
  }
  const int p = g_hdr->size;
  size_t total = 0;
  for (int q = 0; q < p; ++q) total = std::max(total, (size_t)(sdispls[q] + scounts[q]) * se);
  if (total > g_hdr->slot) fail("MPI_Alltoallv", total);
  int* hdr = slot_ints(g_rank);
  for (int q = 0; q < p; ++q) {
    hdr[q] = scounts[q];
    hdr[p + q] = sdispls[q];
  }
  memcpy(slot_data(g_rank), send, total);
  barrier();
  for (int q = 0; q < p; ++q) {
    const int* h = slot_ints(q);
    const size_t n = (size_t)std::min(h[g_rank], rcounts[q]) * re;
    memcpy((char*)recv + (size_t)rdispls[q] * re, slot_data(q) + (size_t)h[p + g_rank] * se, n);
  }
  barrier();
  return 0;
}
