// Internal declarations shared by api.cu and the serving loop.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include <mutex>

#include "arena.h"

namespace isdf_b200 {

int iround(double a);
int default_mu(int nv1, int nc1, int nv2, int nc2);
size_t solve_workspace_bytes(long long ng, int nstate, int mu, int selector, int precision,
                             int check, double qrcp_factor, const int* num_grid, int npair);
int acquire_workspace(size_t bytes, Arena* arena, cudaStream_t* lib_stream);
std::mutex& workspace_mutex();

}  // namespace isdf_b200
