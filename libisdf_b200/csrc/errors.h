// Status reporting shared by the device (.cu) and host-only (.cpp) sources:
// the thread-local error slot and the early-return macros of the C ABI.
#pragma once

#include <cuda_runtime.h>

#include "../../include/isdf_c.h"

namespace isdf_b200 {

// Records a CUDA failure in the thread-local error slot and returns the code
// the C ABI hands back to the caller.
int record_cuda_error(cudaError_t e, const char* what, const char* file, int line);
int record_error(int code, const char* msg);
const char* last_error_message();

#define ISDF_CUDA(x)                                                               \
  do {                                                                             \
    cudaError_t e_ = (x);                                                          \
    if (e_ != cudaSuccess) return ::isdf_b200::record_cuda_error(e_, #x, __FILE__, __LINE__); \
  } while (0)

#define ISDF_CHECK_LAUNCH() ISDF_CUDA(cudaGetLastError())

#define ISDF_TRY(x)              \
  do {                           \
    int rc_ = (x);               \
    if (rc_ != ISDF_OK) return rc_; \
  } while (0)

}  // namespace isdf_b200
