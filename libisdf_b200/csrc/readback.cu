// Small device-to-host reads through mapped pinned host memory (readback.h).
#include <cstring>

#include "common.cuh"
#include "readback.h"

namespace isdf_b200 {

namespace {

__global__ void k_readback(const unsigned* __restrict__ src, volatile unsigned* dst, size_t n) {
  for (size_t i = threadIdx.x + (size_t)blockIdx.x * blockDim.x; i < n;
       i += (size_t)blockDim.x * gridDim.x)
    dst[i] = src[i];
  __threadfence_system();
}

struct Mailbox {
  void* host = nullptr;
  void* dev = nullptr;
  size_t cap = 0;
  bool enabled = true;
  ~Mailbox() {
    if (host) cudaFreeHost(host);
  }
};

thread_local Mailbox tl_mailbox;

constexpr size_t kMinMailbox = 64 << 10;

}  // namespace

void set_readback_mailbox(bool on) { tl_mailbox.enabled = on; }
bool readback_mailbox() { return tl_mailbox.enabled; }

int read_back(void* dst, const void* dsrc, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return ISDF_OK;
  if (bytes % 4 != 0) return record_error(ISDF_ERR_ARG, "read_back: size not a multiple of 4");
  Mailbox& m = tl_mailbox;
  if (m.enabled && m.cap < bytes) {
    if (m.host) {
      ISDF_CUDA(cudaFreeHost(m.host));
      m.host = m.dev = nullptr;
      m.cap = 0;
    }
    size_t cap = kMinMailbox;
    while (cap < bytes) cap *= 2;
    void* h = nullptr;
    if (cudaHostAlloc(&h, cap, cudaHostAllocMapped | cudaHostAllocPortable) == cudaSuccess) {
      void* d = nullptr;
      if (cudaHostGetDevicePointer(&d, h, 0) == cudaSuccess) {
        m.host = h;
        m.dev = d;
        m.cap = cap;
      } else {
        cudaFreeHost(h);
      }
    }
    (void)cudaGetLastError();  // a refused mapping falls back to copies
  }
  if (m.enabled && m.cap >= bytes) {
    const size_t n = bytes / 4;
    const unsigned blocks = (unsigned)(n < 256 * 1024 ? (n + 255) / 256 : 1024);
    k_readback<<<blocks, 256, 0, s>>>(static_cast<const unsigned*>(dsrc),
                                      static_cast<unsigned*>(m.dev), n);
    ISDF_CHECK_LAUNCH();
    ISDF_CUDA(cudaStreamSynchronize(s));
    std::memcpy(dst, m.host, bytes);
    return ISDF_OK;
  }
  ISDF_CUDA(cudaMemcpyAsync(dst, dsrc, bytes, cudaMemcpyDeviceToHost, s));
  ISDF_CUDA(cudaStreamSynchronize(s));
  return ISDF_OK;
}

}  // namespace isdf_b200
