// Internal declarations shared by api.cu and the serving loop.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <mutex>

#include "../../include/isdf_c.h"
#include "arena.h"

namespace isdf_b200 {

// Base-254 INT8 digits per FP64 operand in the mixed-precision GEMMs.
constexpr int kDefaultMixedSlices = 6;

int iround(double a);
int default_mu(int nv1, int nc1, int nv2, int nc2);
int check_state_ranges(int nocc, int nstate, int nv1, int nc1, int nv2, int nc2);
size_t solve_workspace_bytes(long long ng, int nstate, int mu, int selector, int precision,
                             int check, double qrcp_factor, const int* num_grid, int npair);
int acquire_workspace(size_t bytes, Arena* arena, cudaStream_t* lib_stream);
std::mutex& workspace_mutex();
int record_error(int code, const char* msg);

// Guards the one-time per-device kernel attribute settings.
std::mutex& attr_mutex();

// A caller-owned workspace and stream for one solve (the serving loop's slots).
// fit_lock (optional): held around the fit of a large system (Ng rk^2 at
// least kSerialFitWork), so that large fits run one at a time while other
// requests' selections and small fits overlap them.
struct KmeansResult;
struct SolveResources {
  char* base;
  size_t cap;
  cudaStream_t stream;
  std::mutex* fit_lock = nullptr;
  // K-means selection already done (the serving loop's batched selections):
  // piv holds its result and the solve starts at the fit
  const KmeansResult* preselected = nullptr;
};
constexpr double kSerialFitWork = 1e13;

// Device workspace one solve with these parameters needs.
size_t request_footprint(const isdf_domain_t* dom, int nstate, int nv1, int nc1, int nv2, int nc2,
                         int mu_points, int selector, int check, const isdf_options_t* opt);

int solve(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1, int nc1,
          int nv2, int nc2, int mu_points, double* d_theta, int* piv, int kmeans_max_iter,
          int selector, int check, const isdf_options_t* opt, isdf_report_t* rep,
          const SolveResources* res);

}  // namespace isdf_b200
