// Host-side entry points of the QRCP selector (qrcp.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "arena.h"

namespace isdf_b200 {

struct QrcpArgs {
  const double* d_psi;  // Ng x nstate, ld = Ng
  long long ng;
  int nstate, nocc, nv1, nc1, nv2, nc2;
  int mu;
  double factor;   // sketch oversampling: numPre = IRound(sqrt(mu * factor))
  long long seed;  // srand48 seed of the sketch
  int* piv;        // host int[ng]
};

struct QrcpResult {
  int ntot_mg = 0;   // kept columns
  int steps = 0;     // pivots computed (min(mu, numPre^2, ntot_mg))
  int num_pre = 0;
  int recomputes = 0;  // residual norms recomputed exactly (LAPACK's cancellation test)
  int done_early = 0;
  int launches = 0;
};

int qrcp_num_pre(int mu, double factor);
size_t qrcp_workspace_bytes(long long ng, int nstate, int mu, double factor);
int qrcp_select(const QrcpArgs& args, Arena& arena, cudaStream_t stream, QrcpResult* res);

}  // namespace isdf_b200
