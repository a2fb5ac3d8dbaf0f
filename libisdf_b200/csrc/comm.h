// Collective transports of the grid-row sharded solve (comm.cpp).
//
// A sharded solve runs one rank per GPU; each rank holds a block of grid rows
// of psi and needs three exchanges: an all-gather of variable-size blocks
// (the weights, the K-means partial sums and nearest points, the psi rows at
// the pivots) and, for the reference's column-cyclic theta layout, an
// all-to-all. Both are stream-ordered: they take effect in order with the
// kernels on the given stream.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "arena.h"

namespace isdf_b200 {

struct Transport {
  int rank = 0;
  int size = 1;
  int device = 0;
  // per-rank device workspace and stream of the sharded solve
  char* ws = nullptr;
  size_t ws_cap = 0;
  cudaStream_t stream = nullptr;
  // (size + 1) status records of kStatusBytes for the ranks' agreement before
  // an exchange (records 0..size-1 received, record size sent); allocated
  // when the communicator is made, so that a rank whose solve fails can
  // still take part
  static constexpr size_t kStatusBytes = 256;
  char* status = nullptr;

  virtual ~Transport();
  // Rank q's send_bytes (= counts[q]) land at d_recv + displs[q] on every rank.
  virtual int allgatherv(const void* d_send, size_t send_bytes, void* d_recv, const size_t* counts,
                         const size_t* displs, cudaStream_t s) = 0;
  // Rank q receives send_counts[q] bytes from d_send + send_displs[q]; this
  // rank receives recv_counts[q] bytes from rank q at d_recv + recv_displs[q].
  virtual int alltoallv(const void* d_send, const size_t* send_counts, const size_t* send_displs,
                        void* d_recv, const size_t* recv_counts, const size_t* recv_displs,
                        cudaStream_t s) = 0;
  // Ends outstanding and future collectives with an error (failure handling).
  virtual int abort() { return 0; }

  // Makes the rank's stream (once) on its device.
  int ensure_stream();
  // Allocates the status records (once) on the rank's device.
  int ensure_status();
  // Grows the workspace to >= bytes on this rank's device.
  int acquire(size_t bytes, Arena* arena);
};

// The reference's block rule for n items over p ranks (src/common/isdf.cpp:
// 137-141, src/cuda/isdf-gpu.cpp:64-78): the first n % p ranks take one more.
inline long long block_start(long long n, int p, int r) {
  return (long long)r * (n / p) + (r < n % p ? r : n % p);
}
inline long long block_count(long long n, int p, int r) {
  return n / p + (r < n % p ? 1 : 0);
}

}  // namespace isdf_b200
