// Host-side entry points of the K-means selector (kmeans.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>

#include "arena.h"

namespace isdf_b200 {

constexpr int kKmeansMaxMu = 12288;  // per-tile label histograms live in 48 KB of shared memory

struct KmeansArgs {
  const double* d_w;  // device weight[ng]
  long long ng;
  int num_grid[3];
  double length[3];
  int mu;
  int max_iter;
  long long rand_seed;  // >= 0: srand() first
  int* piv;             // host int[ng]; read first when warm != 0
  int warm = 0;         // start from the previous pivots in piv (utility.cpp:725-749)
};

struct KmeansResult {
  int rk_eff = 0;
  int iters = 0;
  int npt = 0;
  int launches = 0;
  double search_frac = 0;  // share of point assignments that ran the cell search
  int warm_pivots = -1;    // warm start: previous pivots kept as initial centroids
};

size_t kmeans_workspace_bytes(long long ng, int mu);

// Batched selection of small systems in one cooperative launch (the serving
// loop's batches): cold start only, ng <= kKmeansBatchMaxNg, mu <= kKmeansBatchMaxMu.
// piv and the results equal kmeans_select()'s for each request.
constexpr int kKmeansBatchMaxMu = 512;
constexpr long long kKmeansBatchMaxNg = 1 << 20;
size_t kmeans_batch_workspace_bytes(long long ng, int mu);
int kmeans_select_batch(const KmeansArgs* args, int count, Arena& arena, cudaStream_t stream,
                        KmeansResult* res);
int kmeans_weight(const double* d_psi, long long ng, int nocc, int nv1, int nc1, int nv2, int nc2,
                  double* d_w, cudaStream_t stream);
// shard != nullptr: this rank's part of the p-rank selection (the
// reference's KMEAN at world size p, utility.cpp:682-969): it assigns and
// folds its own block of the point list, the partial sums are exchanged
// through `shard` every iteration and combined in binomial-tree order, the
// nearest points by MINLOC. Every rank gets the same piv.
struct Transport;
constexpr int kKmeansMaxRanks = 64;
size_t kmeans_shard_workspace_bytes(long long ng, int mu, int ranks);
int kmeans_select(const KmeansArgs& args, Arena& arena, cudaStream_t stream, KmeansResult* res,
                  Transport* shard = nullptr);

}  // namespace isdf_b200
