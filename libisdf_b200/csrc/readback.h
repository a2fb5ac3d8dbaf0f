// Small device-to-host reads of a solve (K-means state, selected points,
// factorisation status) without the copy engines.
//
// A caller that consumes theta on the host streams the previous solve's theta
// out while the next one runs; a cudaMemcpyAsync device-to-host of a few bytes
// queues on the same copy engine behind those large copies, and the solve
// waits for them at every one of its host synchronisation points (one per
// K-means iteration chunk). read_back() instead launches a one-block kernel
// that stores the bytes into mapped pinned host memory (over the bus, no copy
// engine), synchronises the stream and copies them out. The mapped buffer is
// per host thread and grows on demand; a thread that must not allocate (the
// no-allocation fit) switches the mailbox off and reads back by copies.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

namespace isdf_b200 {

// dst <- bytes at dsrc (device) after all prior work on s; bytes % 4 == 0.
// Synchronises s.
int read_back(void* dst, const void* dsrc, size_t bytes, cudaStream_t s);

// Thread-local: false makes read_back use cudaMemcpyAsync (no host allocation).
void set_readback_mailbox(bool on);
bool readback_mailbox();

}  // namespace isdf_b200
