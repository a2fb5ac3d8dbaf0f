// Host-side entry points of the check (check.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "arena.h"

namespace isdf_b200 {

struct CheckArgs {
  const double* d_psi;  // Ng x nstate, ld = Ng
  int num_grid[3];
  double length[3];
  int nstate, nocc, nv1, nc1, nv2, nc2;
  int rk;
  const int* piv;        // host, first rk entries
  const double* d_theta;  // Ng x rk, ld = Ng
};

size_t check_workspace_bytes(const int* num_grid, int nstate, int rk, int npair);
int check_run(const CheckArgs& args, Arena& arena, cudaStream_t s, double* fit_err,
              double* coul_err);

// A = Re(zeta^H V zeta) (rk x rk, column-major, device), zeta = FFT(theta columns).
size_t coulomb_matrix_workspace_bytes(const int* num_grid, int rk);
int coulomb_matrix_run(const int* num_grid, const double* length, const double* d_theta, int rk,
                       double* d_A, Arena& arena, cudaStream_t s);

// The check restricted to a list of state pairs (pair index (k - lo1) * n2 +
// (j - lo2)); pairs: host int[npair_sample].
size_t check_sampled_workspace_bytes(const int* num_grid, int rk, int npair_sample);
int check_sampled_run(const CheckArgs& args, const int* pairs, int npair_sample, Arena& arena,
                      cudaStream_t s, double* fit_err, double* coul_err);

}  // namespace isdf_b200
