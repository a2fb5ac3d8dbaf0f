// Host-side entry points of the fit (fit.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "arena.h"

namespace isdf_b200 {

struct FitArgs {
  const double* d_psi;  // Ng x nstate, ld = Ng
  long long ng;
  int nstate, nocc, nv1, nc1, nv2, nc2;
  int rk;
  const int* piv;   // host, first rk entries used
  double* d_theta;  // Ng x rk, ld = Ng
  // Sharded fit (d_psi holds this rank's grid rows): psi at the pivots,
  // gathered over the ranks, depth-major (B(k, j) = d_psimu[k*rk + j]); C C^T
  // is then formed from it (every element the same product and order of
  // summation as the pivot rows of Z C^T), not gathered from this rank's rows.
  const double* d_psimu = nullptr;
};

struct FitResult {
  int chol_info = 0;
  int launches = 0;
  float t_zct_ms = 0, t_chol_ms = 0, t_solve_ms = 0;  // CUDA-event stage times
  float t_gemm_ms = 0;  // the triangular stage's GEMM launches alone (0: not timed apart)
};

size_t fit_workspace_bytes(long long ng, int nstate, int rk);

// Mixed-precision fit: the large products as INT8-sliced (`slices` = 5..7)
// GEMMs on the tcgen05 tensor cores, FP64 Cholesky and triangular inverse.
size_t fit_mixed_workspace_bytes(long long ng, int nstate, int rk, int slices);
int fit_mixed(const FitArgs& args, Arena& arena, cudaStream_t stream, FitResult* res, int slices);

// C = A * B on the FP64 tensor cores: A column-major (lda), B depth-major
// (B(k, n) = B[k*ldb + n]), C column-major (ldc).
int dgemm_store(int M, int N, int K, const double* A, long long lda, const double* B,
                long long ldb, double* C, long long ldc, cudaStream_t s);
// timed = false skips the stage timers (no CUDA events are created); the
// launches are then only queued on `stream` after the Cholesky check.
int fit_fp64(const FitArgs& args, Arena& arena, cudaStream_t stream, FitResult* res,
             bool timed = true);

}  // namespace isdf_b200
