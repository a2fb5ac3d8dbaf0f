// Shared-memory mbarriers and bulk copies (cp.async.bulk, no tensor map, no
// multicast) for the tensor-core pipelines: the INT8 digit GEMM (ozaki.cuh)
// and the warp-specialised FP64 GEMM tile (dgemm.cuh). Every wait is bounded.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace isdf_b200 {

constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t mbar, int count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(mbar), "r"(count));
}

__device__ __forceinline__ void mbar_arrive(uint32_t mbar) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.release.cta.shared::cta.b64 st, [%0];\n}\n" ::"r"(mbar)
      : "memory");
}

__device__ __forceinline__ bool mbar_try(uint32_t mbar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(mbar), "r"(parity)
      : "memory");
  return done != 0;
}

// Bounded wait. Gives up (false) when *abort is set by another thread or when
// the spin limit is reached (then it sets *abort itself).
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, volatile int* abort) {
  for (long long i = 0; i < kSpinLimit; ++i) {
    if (mbar_try(mbar, parity)) return true;
    if ((i & 255) == 255 && *abort) return false;
  }
  *abort = 1;
  return false;
}

// Bounded wait that ignores the abort flag: used for the issued MMAs, which
// complete by themselves and must complete before the TMEM is freed.
__device__ __forceinline__ bool mbar_wait_all(uint32_t mbar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i)
    if (mbar_try(mbar, parity)) return true;
  return false;
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t mbar, uint32_t bytes) {
  asm volatile(
      "{\n .reg .b64 st;\n mbarrier.arrive.expect_tx.release.cta.shared::cta.b64 st, [%0], %1;\n}\n" ::"r"(
          mbar),
      "r"(bytes)
      : "memory");
}

// Contiguous global -> shared copy completing on mbar (bytes and addresses
// multiples of 16).
__device__ __forceinline__ void bulk_copy(uint32_t sdst, const void* gsrc, uint32_t bytes,
                                          uint32_t mbar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          sdst),
      "l"(gsrc), "r"(bytes), "r"(mbar)
      : "memory");
}

}  // namespace isdf_b200
