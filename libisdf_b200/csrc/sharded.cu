// The grid-row sharded ISDF solve: one rank per GPU, the reference's p-rank
// GPU layout (src/common/isdf.cpp:132-188 -> src/cuda/isdf-gpu.cpp:9-403).
//
// Rank r holds the grid rows [start_r, start_r + count_r) of psi. The stages:
//  1. weights of the own rows, all-gathered into the full weight vector
//     (isdf-gpu.cpp:39-100: calculateKmeansWeight + MPI_Allgatherv);
//  2. the p-rank K-means selection (kmeans.cu, kmeans_select with a
//     transport: utility.cpp:682-969 at world size p);
//  3. psi at the pivots: every rank packs the pivot rows it owns (piv is
//     sorted, so they are a contiguous range of pivots), one all-gather
//     assembles them on every rank (the reference moves the same rows with
//     AlltoallBackward / AlltoallForward / MPI_Allgatherv, isdf-gpu.cpp:
//     138-214);
//  4. the fit of the own rows: Z C^T on them, C C^T from the gathered pivot
//     rows on every rank (the reference gathers the same numbers: each rank
//     contributes its pivot rows of Z C^T and an MPI_Allreduce sums them,
//     isdf-gpu.cpp:276-341; here no exchange is needed), Cholesky on every
//     rank, the triangular products on the own rows;
//  5. theta_layout ISDF_THETA_CYCLIC: the rows-to-cyclic-columns exchange of
//     GPU_AlltoallBackward (utility.cpp:444-526): pack by destination, one
//     all-to-all, one 2-D copy per source into the caller's Ng x w_r block.
// No kernel waits on another rank; every exchange is a transport call
// ordered on the rank's stream.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>
#include <vector>

#include "arena.h"
#include "comm.h"
#include "common.cuh"
#include "fit.h"
#include "kmeans.h"
#include "readback.h"
#include "solve.h"

isdf_b200::Transport* isdf_comm_transport(isdf_comm_t* c);

namespace isdf_b200 {

namespace {

// packed[(nu - nu0) * nstate + k] = psi_local(local[nu - nu0], k)
__global__ void k_pack_pivot_rows(const double* __restrict__ psi, long long rows, int nstate,
                                  const int* __restrict__ local, int count,
                                  double* __restrict__ packed) {
  const long long total = (long long)count * nstate;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int j = (int)(e / nstate), k = (int)(e % nstate);
    packed[e] = psi[(long long)local[j] + (long long)k * rows];
  }
}

// Bm[k * rk + nu] = rows[nu * nstate + k] (the fit's depth-major B operand)
__global__ void k_pivot_rows_to_depth(const double* __restrict__ rows, int rk, int nstate,
                                      double* __restrict__ Bm) {
  const long long total = (long long)rk * nstate;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int k = (int)(e / rk), nu = (int)(e % rk);
    Bm[e] = rows[(long long)nu * nstate + k];
  }
}

// Column j of the local rows T (count x rk, ld = count) goes to rank j % p as
// its column j / p: packed by destination, destination d's block holding its
// w_d columns one after another (GPU_AlltoallBackward's recvk map,
// src/cuda/cuda_utils.cu:89-99).
__global__ void k_pack_cyclic(const double* __restrict__ T, long long count, int rk, int p,
                              double* __restrict__ P) {
  const long long total = count * rk;
  const int base = rk / p, extra = rk % p;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long i = e % count;
    const int j = (int)(e / count);
    const int d = j % p, c = j / p;
    const long long col = (long long)d * base + (d < extra ? d : extra) + c;
    P[col * count + i] = T[e];
  }
}

// The ranks' agreement before an exchange. Every rank all-gathers its status
// and the arguments the exchanges depend on. If a rank failed, or was called
// with arguments other than rank 0's, every rank returns an error. Otherwise
// the others would wait inside a collective that the failed rank never joins:
// NCCL has no timeout of its own. A failed rank returns its own code and
// message; the others return ISDF_ERR_COMM naming it, or ISDF_ERR_ARG when the
// arguments differ.
constexpr int kStatusWords = (int)(Transport::kStatusBytes / sizeof(long long));
struct RankStatus {
  long long v[kStatusWords] = {};  // v[0]: status; v[1..n): the shared arguments
  int n = 1;
  void add(long long x) {
    if (n < kStatusWords) v[n++] = x;
  }
  void add(double x) {
    long long b;
    std::memcpy(&b, &x, sizeof(b));
    add(b);
  }
};

int agree(Transport* T, int rc, RankStatus mine, cudaStream_t s, const char* stage) {
  const int p = T->size;
  if (!T->status) return record_error(ISDF_ERR_COMM, "sharded solve: no status buffer");
  mine.v[0] = rc;
  constexpr size_t sz = Transport::kStatusBytes;
  static_assert(sizeof(RankStatus::v) == sz, "status record size");
  char* send = T->status + (size_t)p * sz;
  ISDF_CUDA(cudaMemcpyAsync(send, mine.v, sz, cudaMemcpyHostToDevice, s));
  std::vector<size_t> cnt(p, sz), dsp(p);
  for (int q = 0; q < p; ++q) dsp[q] = (size_t)q * sz;
  ISDF_TRY(T->allgatherv(send, sz, T->status, cnt.data(), dsp.data(), s));
  std::vector<long long> all((size_t)p * kStatusWords);
  ISDF_CUDA(cudaMemcpyAsync(all.data(), T->status, (size_t)p * sz, cudaMemcpyDeviceToHost, s));
  ISDF_CUDA(cudaStreamSynchronize(s));
  if (rc != ISDF_OK) return rc;
  char msg[160];
  for (int q = 0; q < p; ++q) {
    const long long* w = all.data() + (size_t)q * kStatusWords;
    if (w[0] != ISDF_OK) {
      std::snprintf(msg, sizeof(msg), "%s: rank %d failed (status %lld)", stage, q, w[0]);
      return record_error(ISDF_ERR_COMM, msg);
    }
  }
  for (int q = 1; q < p; ++q) {
    const long long* w = all.data() + (size_t)q * kStatusWords;
    for (int k = 1; k < mine.n; ++k)
      if (w[k] != all[k]) {
        std::snprintf(msg, sizeof(msg),
                      "%s: rank %d was called with other arguments than rank 0 (argument %d)",
                      stage, q, k);
        return record_error(ISDF_ERR_ARG, msg);
      }
  }
  return ISDF_OK;
}

struct Stopwatch {
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
  double ms() const {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
        .count();
  }
};

}  // namespace

static size_t sharded_workspace_bytes(long long ng, long long cnt, int nstate, int rk, int p,
                                      int precision, int layout) {
  Arena a;
  a.counting = true;
  a.take<double>((size_t)ng);   // the full weight vector
  a.take<double>((size_t)cnt);  // this rank's weights
  const size_t sel = kmeans_shard_workspace_bytes(ng, rk, p);
  Arena f;
  f.counting = true;
  f.take<int>((size_t)rk);                    // own pivot rows (local indices)
  f.take<double>((size_t)rk * nstate);        // packed own pivot rows
  f.take<double>((size_t)rk * nstate);        // all pivot rows, pivot-major
  f.take<double>((size_t)rk * nstate);        // all pivot rows, depth-major
  if (layout == ISDF_THETA_CYCLIC) {
    const long long wr = rk / p + 1;
    const size_t tb = (size_t)std::max(cnt * rk, ng * wr);
    f.take<double>(tb);  // the fitted rows, later the received blocks
    f.take<double>(tb);  // the rows packed by destination
  }
  const size_t fit = f.off + (precision == ISDF_PRECISION_MIXED
                                  ? fit_mixed_workspace_bytes(cnt, nstate, rk, 7)
                                  : fit_workspace_bytes(cnt, nstate, rk));
  return a.off + std::max(sel, fit) + 4096;
}

// The argument checks of the sharded solve; *ng and *rk are set on success.
static int check_sharded_args(const isdf_domain_t* dom, const double* d_psirow,
                              const double* d_theta, const int* piv, int p, int nocc, int nstate,
                              int nv1, int nc1, int nv2, int nc2, int mu_points, int layout,
                              int kmeans_max_iter, const isdf_options_t& opt, long long* ng,
                              int* rk) {
  if (!dom || !d_psirow || !d_theta || !piv) return record_error(ISDF_ERR_ARG, "null pointer");
  if (dom->num_grid[0] <= 0 || dom->num_grid[1] <= 0 || dom->num_grid[2] <= 0)
    return record_error(ISDF_ERR_ARG, "empty grid");
  *ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
  if (*ng < p) return record_error(ISDF_ERR_ARG, "sharded solve: fewer grid points than ranks");
  ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
  if (kmeans_max_iter < 0) return record_error(ISDF_ERR_ARG, "negative K-means iteration cap");
  *rk = mu_points == 0 ? default_mu(nv1, nc1, nv2, nc2) : mu_points;
  if (*rk <= 0 || *rk > *ng) return record_error(ISDF_ERR_ARG, "mu outside [1, Ng]");
  if (*rk > kKmeansMaxMu) return record_error(ISDF_ERR_UNSUPPORTED, "mu above the K-means limit");
  if (layout != ISDF_THETA_ROWS && layout != ISDF_THETA_CYCLIC)
    return record_error(ISDF_ERR_ARG, "unknown theta layout");
  if (opt.precision != ISDF_PRECISION_FP64 && opt.precision != ISDF_PRECISION_MIXED)
    return record_error(ISDF_ERR_ARG, "unknown precision");
  if (opt.precision == ISDF_PRECISION_MIXED && (opt.mixed_slices < 5 || opt.mixed_slices > 7))
    return record_error(ISDF_ERR_ARG, "mixed_slices must be 5, 6 or 7");
  if (opt.refine_steps != 0)
    return record_error(ISDF_ERR_UNSUPPORTED,
                        "refine_steps must be 0: FP64 refinement of the theta solve is not built");
  return ISDF_OK;
}

// The grid and the K-means arguments every rank must share.
static void add_domain(RankStatus* st, const isdf_domain_t* dom) {
  for (int i = 0; i < 3; ++i) st->add((long long)(dom ? dom->num_grid[i] : 0));
  for (int i = 0; i < 3; ++i) st->add(dom ? dom->length[i] : 0.0);
}

int solve_sharded(Transport* T, const isdf_domain_t* dom, const double* d_psirow, int nocc,
                  int nstate, int nv1, int nc1, int nv2, int nc2, int mu_points, double* d_theta,
                  int layout, int* piv, int kmeans_max_iter, const isdf_options_t* opt_in,
                  isdf_report_t* rep_out) {
  Stopwatch total;
  isdf_options_t opt;
  isdf_default_options(&opt);
  if (opt_in) opt = *opt_in;
  isdf_report_t rep;
  std::memset(&rep, 0, sizeof(rep));
  if (!T) return record_error(ISDF_ERR_ARG, "null comm");
  const int p = T->size, r = T->rank;
  // Every check below ends in the agreement rather than in an early return,
  // so that a rank that fails them still meets the others there.
  int rc = T->ensure_stream();
  cudaStream_t s = opt.stream ? (cudaStream_t)opt.stream : T->stream;
  long long ng = 0;
  int rk = 0;
  if (rc == ISDF_OK)
    rc = check_sharded_args(dom, d_psirow, d_theta, piv, p, nocc, nstate, nv1, nc1, nv2, nc2,
                            mu_points, layout, kmeans_max_iter, opt, &ng, &rk);
  RankStatus mine;
  add_domain(&mine, dom);
  for (long long x : {(long long)nocc, (long long)nstate, (long long)nv1, (long long)nc1,
                      (long long)nv2, (long long)nc2, (long long)rk, (long long)kmeans_max_iter,
                      (long long)layout, (long long)opt.precision, (long long)opt.mixed_slices,
                      opt.rand_seed, (long long)opt.kmeans_warm_start})
    mine.add(x);
  rep.rk_requested = rk;
  const long long start = rc == ISDF_OK ? block_start(ng, p, r) : 0;
  const long long cnt = rc == ISDF_OK ? block_count(ng, p, r) : 0;
  Arena arena;
  if (rc == ISDF_OK)
    rc = T->acquire(sharded_workspace_bytes(ng, cnt, nstate, rk, p, opt.precision, layout),
                    &arena);
  ISDF_TRY(agree(T, rc, mine, s, "sharded solve"));
  double* d_w = arena.take<double>((size_t)ng);
  double* d_wloc = arena.take<double>((size_t)cnt);
  const size_t mark = arena.off;

  // 1. weights: own rows, then the all-gather by the row blocks
  ISDF_TRY(kmeans_weight(d_psirow, cnt, nocc, nv1, nc1, nv2, nc2, d_wloc, s));
  std::vector<size_t> wc(p), wd(p);
  for (int q = 0; q < p; ++q) {
    wc[q] = sizeof(double) * (size_t)block_count(ng, p, q);
    wd[q] = sizeof(double) * (size_t)block_start(ng, p, q);
  }
  ISDF_TRY(T->allgatherv(d_wloc, wc[r], d_w, wc.data(), wd.data(), s));

  // 2. the p-rank K-means selection
  KmeansArgs ka;
  ka.d_w = d_w;
  ka.ng = ng;
  for (int i = 0; i < 3; ++i) {
    ka.num_grid[i] = dom->num_grid[i];
    ka.length[i] = dom->length[i];
  }
  ka.mu = rk;
  ka.max_iter = kmeans_max_iter;
  ka.rand_seed = opt.rand_seed;
  ka.piv = piv;
  ka.warm = opt.kmeans_warm_start;
  KmeansResult kr;
  ISDF_TRY(kmeans_select(ka, arena, s, &kr, T));
  rep.rk_eff = kr.rk_eff;
  rep.kmeans_iters = kr.iters;
  rep.npt = kr.npt;
  rep.kmeans_search_frac = (float)kr.search_frac;
  rep.kmeans_warm_pivots = kr.warm_pivots;
  rep.kernel_launches = 1 + kr.launches;
  rep.t_select_ms = total.ms();
  const int rke = kr.rk_eff;

  // 3. psi at the pivots (piv[0..rke) ascending: rank q owns a contiguous range)
  Stopwatch fit_clock;
  arena.off = mark;
  int* d_local = arena.take<int>((size_t)rk);
  double* d_own = arena.take<double>((size_t)rk * nstate);
  double* d_rows = arena.take<double>((size_t)rk * nstate);
  double* d_Bm = arena.take<double>((size_t)rk * nstate);
  double *d_T = nullptr, *d_P = nullptr;
  const long long wr = block_count(rk, p, r);
  if (layout == ISDF_THETA_CYCLIC) {
    const size_t tb = (size_t)std::max(cnt * rk, ng * (long long)(rk / p + 1));
    d_T = arena.take<double>(tb);
    d_P = arena.take<double>(tb);
  }
  std::vector<int> nu0(p + 1);  // rank q owns the pivots [nu0[q], nu0[q + 1])
  for (int q = 0; q <= p; ++q)  // block_start(ng, p, p) = ng
    nu0[q] = (int)(std::lower_bound(piv, piv + rke, (int)block_start(ng, p, q)) - piv);
  const int own = nu0[r + 1] - nu0[r];
  if (own > 0) {
    std::vector<int> local(own);
    for (int j = 0; j < own; ++j) local[j] = piv[nu0[r] + j] - (int)start;
    ISDF_CUDA(cudaMemcpyAsync(d_local, local.data(), sizeof(int) * own, cudaMemcpyHostToDevice, s));
    k_pack_pivot_rows<<<grid_for((long long)own * nstate, 256), 256, 0, s>>>(d_psirow, cnt, nstate,
                                                                            d_local, own, d_own);
    ISDF_CHECK_LAUNCH();
  }
  std::vector<size_t> pc(p), pd(p);
  for (int q = 0; q < p; ++q) {
    pc[q] = sizeof(double) * (size_t)(nu0[q + 1] - nu0[q]) * nstate;
    pd[q] = sizeof(double) * (size_t)nu0[q] * nstate;
  }
  ISDF_TRY(T->allgatherv(d_own, pc[r], d_rows, pc.data(), pd.data(), s));
  k_pivot_rows_to_depth<<<grid_for((long long)rke * nstate, 256), 256, 0, s>>>(d_rows, rke, nstate,
                                                                               d_Bm);
  ISDF_CHECK_LAUNCH();

  // 4. the fit of the own rows
  double* rows_out = layout == ISDF_THETA_ROWS ? d_theta : d_T;
  FitArgs fa;
  fa.d_psi = d_psirow;
  fa.ng = cnt;
  fa.nstate = nstate;
  fa.nocc = nocc;
  fa.nv1 = nv1;
  fa.nc1 = nc1;
  fa.nv2 = nv2;
  fa.nc2 = nc2;
  fa.rk = rke;
  fa.piv = piv;
  fa.d_theta = rows_out;
  fa.d_psimu = d_Bm;
  FitResult fr;
  rc = opt.precision == ISDF_PRECISION_MIXED ? fit_mixed(fa, arena, s, &fr, opt.mixed_slices)
                                             : fit_fp64(fa, arena, s, &fr);
  rep.chol_info = fr.chol_info;
  rep.kernel_launches += fr.launches + 2;
  rep.t_zct_ms = fr.t_zct_ms;
  rep.t_chol_ms = fr.t_chol_ms;
  rep.t_solve_ms = fr.t_solve_ms;
  rep.t_gemm_ms = fr.t_gemm_ms > 0.f ? fr.t_gemm_ms : fr.t_solve_ms;
  if (rc == ISDF_OK && rke < rk) {
    const cudaError_t e = cudaMemsetAsync(rows_out + (size_t)rke * cnt, 0,
                                          sizeof(double) * (size_t)(rk - rke) * cnt, s);
    if (e != cudaSuccess) rc = record_cuda_error(e, "cudaMemsetAsync (theta tail)", __FILE__, __LINE__);
  }
  // theta's all-to-all is the one exchange after the fit
  if (layout == ISDF_THETA_CYCLIC) rc = agree(T, rc, mine, s, "sharded solve (theta exchange)");
  if (rc != ISDF_OK) {
    if (rep_out) *rep_out = rep;
    return rc;
  }

  // 5. the reference's column-cyclic layout
  if (layout == ISDF_THETA_CYCLIC) {
    k_pack_cyclic<<<grid_for(cnt * rk, 256, 4), 256, 0, s>>>(d_T, cnt, rk, p, d_P);
    ISDF_CHECK_LAUNCH();
    std::vector<size_t> sc(p), sd(p), rcn(p), rd(p);
    for (int q = 0; q < p; ++q) {
      sc[q] = sizeof(double) * (size_t)block_count(rk, p, q) * cnt;
      sd[q] = sizeof(double) * (size_t)block_start(rk, p, q) * cnt;
      rcn[q] = sizeof(double) * (size_t)wr * block_count(ng, p, q);
      rd[q] = sizeof(double) * (size_t)wr * block_start(ng, p, q);
    }
    double* d_R = d_T;  // the fitted rows are packed already
    ISDF_TRY(T->alltoallv(d_P, sc.data(), sd.data(), d_R, rcn.data(), rd.data(), s));
    for (int q = 0; q < p && wr > 0; ++q) {
      const long long cq = block_count(ng, p, q), sq = block_start(ng, p, q);
      ISDF_CUDA(cudaMemcpy2DAsync(d_theta + sq, sizeof(double) * (size_t)ng,
                                  d_R + (size_t)wr * sq, sizeof(double) * (size_t)cq,
                                  sizeof(double) * (size_t)cq, (size_t)wr,
                                  cudaMemcpyDeviceToDevice, s));
    }
  }
  ISDF_CUDA(cudaStreamSynchronize(s));
  rep.t_fit_ms = fit_clock.ms();
  rep.t_total_ms = total.ms();
  if (rep_out) *rep_out = rep;
  return ISDF_OK;
}

int kmeans_select_sharded(Transport* T, const isdf_domain_t* dom, const double* d_w, int mu,
                          int max_iter, long long rand_seed, int* piv, int* rk_eff, int* iters,
                          int* npt) {
  if (!T) return record_error(ISDF_ERR_ARG, "null comm");
  // as in solve_sharded: the checks end in the ranks' agreement
  int rc = T->ensure_stream();
  long long ng = 0;
  if (rc == ISDF_OK) {
    if (!dom || !d_w || !piv) {
      rc = record_error(ISDF_ERR_ARG, "null pointer");
    } else if (dom->num_grid[0] <= 0 || dom->num_grid[1] <= 0 || dom->num_grid[2] <= 0) {
      rc = record_error(ISDF_ERR_ARG, "empty grid");
    } else {
      ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
      if (max_iter < 0)
        rc = record_error(ISDF_ERR_ARG, "negative K-means iteration cap");
      else if (mu <= 0 || mu > ng)
        rc = record_error(ISDF_ERR_ARG, "mu outside [1, Ng]");
      else if (mu > kKmeansMaxMu)
        rc = record_error(ISDF_ERR_UNSUPPORTED, "mu above the K-means limit");
    }
  }
  RankStatus mine;
  add_domain(&mine, dom);
  for (long long x : {(long long)mu, (long long)max_iter, rand_seed}) mine.add(x);
  Arena arena;
  if (rc == ISDF_OK)
    rc = T->acquire(kmeans_shard_workspace_bytes(ng, mu, T->size) + 4096, &arena);
  ISDF_TRY(agree(T, rc, mine, T->stream, "sharded K-means selection"));
  KmeansArgs ka;
  ka.d_w = d_w;
  ka.ng = ng;
  for (int i = 0; i < 3; ++i) {
    ka.num_grid[i] = dom->num_grid[i];
    ka.length[i] = dom->length[i];
  }
  ka.mu = mu;
  ka.max_iter = max_iter;
  ka.rand_seed = rand_seed;
  ka.piv = piv;
  KmeansResult kr;
  ISDF_TRY(kmeans_select(ka, arena, T->stream, &kr, T));
  ISDF_CUDA(cudaStreamSynchronize(T->stream));
  if (rk_eff) *rk_eff = kr.rk_eff;
  if (iters) *iters = kr.iters;
  if (npt) *npt = kr.npt;
  return ISDF_OK;
}

}  // namespace isdf_b200

using namespace isdf_b200;

extern "C" {

int isdf_solve_sharded(isdf_comm_t* comm, const isdf_domain_t* dom, const double* d_psirow,
                       int nocc, int nstate, int nv1, int nc1, int nv2, int nc2, int mu_points,
                       double* d_theta, int theta_layout, int* piv, int kmeans_max_iter,
                       const isdf_options_t* opt, isdf_report_t* rep) {
  try {
    Transport* T = isdf_comm_transport(comm);
    if (!T) return record_error(ISDF_ERR_ARG, "null comm");
    ISDF_CUDA(cudaSetDevice(T->device));
    return solve_sharded(T, dom, d_psirow, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_theta,
                         theta_layout, piv, kmeans_max_iter, opt, rep);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_kmeans_select_sharded(isdf_comm_t* comm, const isdf_domain_t* dom, const double* d_w,
                               int mu, int max_iter, long long rand_seed, int* piv, int* rk_eff,
                               int* iters, int* npt) {
  try {
    Transport* T = isdf_comm_transport(comm);
    if (!T) return record_error(ISDF_ERR_ARG, "null comm");
    ISDF_CUDA(cudaSetDevice(T->device));
    return kmeans_select_sharded(T, dom, d_w, mu, max_iter, rand_seed, piv, rk_eff, iters, npt);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

}  // extern "C"
