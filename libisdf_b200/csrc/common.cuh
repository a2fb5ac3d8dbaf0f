// Shared helpers for the ISDF sm_100a kernels.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/isdf_c.h"
#include "errors.h"

namespace isdf_b200 {

constexpr int kNumSMs = 148;  // B200: 2 dies x 74 SMs

inline unsigned grid_for(long long n, int block, int per_thread = 1) {
  long long b = (n + (long long)block * per_thread - 1) / ((long long)block * per_thread);
  if (b < 1) b = 1;
  if (b > 0x7fffffffLL) b = 0x7fffffffLL;
  return (unsigned)b;
}

// Round-to-nearest FP64 arithmetic that the compiler may not contract into
// FMAs: every K-means quantity must round exactly as the reference's x86-64
// build (SSE2, no FMA) rounds it.
__device__ __forceinline__ double radd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double rsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double rmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double rdiv(double a, double b) { return __ddiv_rn(a, b); }

}  // namespace isdf_b200
