// C ABI of libisdf_b200 (include/isdf_c.h): argument checks, the per-device
// workspace, the stream, and the stage order of one ISDF solve.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "arena.h"
#include "check.h"
#include "common.cuh"
#include "fit.h"
#include "kmeans.h"
#include "qrcp.h"
#include "solve.h"

namespace isdf_b200 {

static thread_local std::string g_last_error;

int record_error(int code, const char* msg) {
  g_last_error = msg ? msg : "";
  return code;
}

int record_cuda_error(cudaError_t e, const char* what, const char* file, int line) {
  char buf[512];
  std::snprintf(buf, sizeof(buf), "%s failed: %s (%s:%d)", what, cudaGetErrorString(e), file,
                line);
  g_last_error = buf;
  return e == cudaErrorMemoryAllocation ? ISDF_ERR_NOMEM : ISDF_ERR_CUDA;
}

const char* last_error_message() { return g_last_error.c_str(); }

// ---------------------------------------------------------------- workspace
namespace {

constexpr int kMaxDevices = 64;
struct DeviceCache {
  std::mutex mu;
  char* buf = nullptr;
  size_t cap = 0;
  cudaStream_t stream = nullptr;
};
DeviceCache g_cache[kMaxDevices];

}  // namespace

int device_cache(int* dev_out, DeviceCache** out) {
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return record_error(ISDF_ERR_UNSUPPORTED, "device index");
  *dev_out = dev;
  *out = &g_cache[dev];
  return ISDF_OK;
}

// Grows the cached device buffer of the current device to >= bytes.
int acquire_workspace(size_t bytes, Arena* arena, cudaStream_t* lib_stream) {
  int dev;
  DeviceCache* c = nullptr;
  ISDF_TRY(device_cache(&dev, &c));
  if (!c->stream) ISDF_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  if (c->cap < bytes) {
    if (c->buf) {
      ISDF_CUDA(cudaDeviceSynchronize());
      ISDF_CUDA(cudaFree(c->buf));
      c->buf = nullptr;
      c->cap = 0;
    }
    cudaError_t e = cudaMalloc((void**)&c->buf, bytes);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return record_error(ISDF_ERR_NOMEM, "workspace allocation failed");
    }
    c->cap = bytes;
  }
  arena->base = c->buf;
  arena->cap = c->cap;
  arena->off = 0;
  arena->counting = false;
  if (lib_stream) *lib_stream = c->stream;
  return ISDF_OK;
}

std::mutex& workspace_mutex() {
  int dev = 0;
  (void)cudaGetDevice(&dev);
  if (dev < 0 || dev >= kMaxDevices) dev = 0;
  return g_cache[dev].mu;
}

static double ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// IRound of include/common/utility.hpp:18-23.
int iround(double a) {
  int b = 0;
  if (a > 0) b = (a - (int)a < 0.5) ? (int)a : ((int)a + 1);
  else b = ((int)a - a < 0.5) ? (int)a : ((int)a - 1);
  return b;
}

int default_mu(int nv1, int nc1, int nv2, int nc2) {
  return iround(std::sqrt((double)((nc1 + nv1) * (nc2 + nv2))) * 8.0);
}

int check_state_ranges(int nocc, int nstate, int nv1, int nc1, int nv2, int nc2) {
  if (nstate <= 0 || nv1 < 0 || nc1 < 0 || nv2 < 0 || nc2 < 0)
    return record_error(ISDF_ERR_ARG, "negative state counts");
  if (nv1 + nc1 <= 0 || nv2 + nc2 <= 0) return record_error(ISDF_ERR_ARG, "empty state sets");
  if (nocc - nv1 < 0 || nocc + nc1 > nstate || nocc - nv2 < 0 || nocc + nc2 > nstate)
    return record_error(ISDF_ERR_ARG, "state window outside [0, nstate)");
  return ISDF_OK;
}

constexpr size_t kCheckMaxBytes = 48ull << 30;

size_t solve_workspace_bytes(long long ng, int nstate, int mu, int selector, int precision,
                             int check, double qrcp_factor, const int* num_grid, int npair) {
  (void)precision;
  Arena a;
  a.counting = true;
  a.take<double>((size_t)ng);  // weight
  size_t sel = selector == ISDF_SELECT_QRCP ? qrcp_workspace_bytes(ng, nstate, mu, qrcp_factor)
                                            : kmeans_workspace_bytes(ng, mu);
  size_t fit = precision == ISDF_PRECISION_MIXED ? fit_mixed_workspace_bytes(ng, nstate, mu, 7)
                                                 : fit_workspace_bytes(ng, nstate, mu);
  size_t chk = (check && num_grid) ? check_workspace_bytes(num_grid, nstate, mu, npair) : 0;
  size_t big = sel > fit ? sel : fit;
  if (chk > big) big = chk;
  return a.off + big + 4096;
}

std::mutex& attr_mutex() {
  static std::mutex m;
  return m;
}

size_t request_footprint(const isdf_domain_t* dom, int nstate, int nv1, int nc1, int nv2, int nc2,
                         int mu_points, int selector, int check, const isdf_options_t* opt) {
  const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
  const int rk = mu_points == 0 ? default_mu(nv1, nc1, nv2, nc2) : mu_points;
  return solve_workspace_bytes(ng, nstate, rk, selector, opt ? opt->precision : 0, check,
                               opt ? opt->qrcp_oversample : 1.5, dom->num_grid,
                               (nv1 + nc1) * (nv2 + nc2));
}

int solve(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1, int nc1,
          int nv2, int nc2, int mu_points, double* d_theta, int* piv, int kmeans_max_iter,
          int selector, int check, const isdf_options_t* opt_in, isdf_report_t* rep_out,
          const SolveResources* res) {
  auto t0 = std::chrono::steady_clock::now();
  isdf_options_t opt;
  isdf_default_options(&opt);
  if (opt_in) opt = *opt_in;
  isdf_report_t rep;
  std::memset(&rep, 0, sizeof(rep));
  if (!dom || !d_psi || !d_theta || !piv) return record_error(ISDF_ERR_ARG, "null pointer");
  const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
  if (dom->num_grid[0] <= 0 || dom->num_grid[1] <= 0 || dom->num_grid[2] <= 0)
    return record_error(ISDF_ERR_ARG, "empty grid");
  ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
  if (kmeans_max_iter < 0) return record_error(ISDF_ERR_ARG, "negative K-means iteration cap");
  const int rk = mu_points == 0 ? default_mu(nv1, nc1, nv2, nc2) : mu_points;
  if (rk <= 0 || rk > ng) return record_error(ISDF_ERR_ARG, "mu outside [1, Ng]");
  if (selector != ISDF_SELECT_KMEANS && selector != ISDF_SELECT_QRCP)
    return record_error(ISDF_ERR_ARG, "unknown selector");
  if (opt.precision != ISDF_PRECISION_FP64 && opt.precision != ISDF_PRECISION_MIXED)
    return record_error(ISDF_ERR_ARG, "unknown precision");
  if (opt.precision == ISDF_PRECISION_MIXED && (opt.mixed_slices < 5 || opt.mixed_slices > 7))
    return record_error(ISDF_ERR_ARG, "mixed_slices must be 5, 6 or 7");
  if (opt.refine_steps != 0)
    return record_error(ISDF_ERR_UNSUPPORTED,
                        "refine_steps must be 0: FP64 refinement of the theta solve is not built");
  if (check && check_workspace_bytes(dom->num_grid, nstate, rk, (nv1 + nc1) * (nv2 + nc2)) >
                   kCheckMaxBytes)
    return record_error(ISDF_ERR_UNSUPPORTED,
                        "check: O(Ng * Npair) pair spectra exceed the device budget at this size");
  if (selector == ISDF_SELECT_KMEANS && rk > kKmeansMaxMu)
    return record_error(ISDF_ERR_UNSUPPORTED, "mu above the K-means limit");
  if (selector == ISDF_SELECT_QRCP && !(opt.qrcp_oversample > 0.0))
    return record_error(ISDF_ERR_ARG, "QRCP oversampling factor must be positive");
  rep.rk_requested = rk;

  const size_t need = solve_workspace_bytes(ng, nstate, rk, selector, opt.precision, check,
                                            opt.qrcp_oversample, dom->num_grid,
                                            (nv1 + nc1) * (nv2 + nc2));
  std::unique_lock<std::mutex> lock;
  Arena arena;
  cudaStream_t s;
  if (res) {  // the caller's workspace and stream (the serving loop)
    if (res->cap < need) return record_error(ISDF_ERR_NOMEM, "solve: workspace below footprint");
    arena.base = res->base;
    arena.cap = res->cap;
    arena.off = 0;
    s = res->stream;
  } else {
    lock = std::unique_lock<std::mutex>(workspace_mutex());
    cudaStream_t lib_stream;
    ISDF_TRY(acquire_workspace(need, &arena, &lib_stream));
    s = opt.stream ? (cudaStream_t)opt.stream : lib_stream;
  }
  double* d_w = arena.take<double>((size_t)ng);
  const size_t mark = arena.off;

  int rk_fit = rk;
  if (selector == ISDF_SELECT_KMEANS && res && res->preselected) {
    const KmeansResult& kr = *res->preselected;
    rep.rk_eff = kr.rk_eff;
    rep.kmeans_iters = kr.iters;
    rep.npt = kr.npt;
    rep.kmeans_warm_pivots = -1;
    rep.kernel_launches = kr.launches;
    rk_fit = kr.rk_eff;
  } else if (selector == ISDF_SELECT_KMEANS) {
    // (a) K-means selection
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
    ISDF_TRY(kmeans_weight(d_psi, ng, nocc, nv1, nc1, nv2, nc2, d_w, s));
    KmeansResult kr;
    ISDF_TRY(kmeans_select(ka, arena, s, &kr));
    rep.rk_eff = kr.rk_eff;
    rep.kmeans_iters = kr.iters;
    rep.npt = kr.npt;
    rep.kmeans_search_frac = (float)kr.search_frac;
    rep.kmeans_warm_pivots = kr.warm_pivots;
    rep.kernel_launches = 1 + kr.launches;
    rk_fit = kr.rk_eff;
  } else {
    // (b) QRCP selection (src/common/isdf.cpp:66-70 -> getpoints_QRCP.cpp); the
    // fit then uses mu pivots, as the reference's getbasis does.
    QrcpArgs qa;
    qa.d_psi = d_psi;
    qa.ng = ng;
    qa.nstate = nstate;
    qa.nocc = nocc;
    qa.nv1 = nv1;
    qa.nc1 = nc1;
    qa.nv2 = nv2;
    qa.nc2 = nc2;
    qa.mu = rk;
    qa.factor = opt.qrcp_oversample;
    qa.seed = opt.qrcp_seed;
    qa.piv = piv;
    QrcpResult qr;
    ISDF_TRY(qrcp_select(qa, arena, s, &qr));
    rep.rk_eff = rk;
    rep.kmeans_iters = 0;
    rep.npt = qr.ntot_mg;
    rep.kernel_launches = qr.launches;
    rep.qrcp_steps = qr.steps;
    rep.qrcp_norm_recomputes = qr.recomputes;
    rep.kmeans_warm_pivots = -1;
  }
  rep.t_select_ms = ms_since(t0);

  // (c, d) fit with the selected points (the GPU path fits with the shrunk
  // rk, isdf-gpu.cpp:12,99); columns past rk_eff are zero-filled.
  std::unique_lock<std::mutex> fit_guard;
  if (res && res->fit_lock && (double)ng * rk_fit * rk_fit >= kSerialFitWork)
    fit_guard = std::unique_lock<std::mutex>(*res->fit_lock);
  auto t1 = std::chrono::steady_clock::now();
  arena.off = mark;
  FitArgs fa;
  fa.d_psi = d_psi;
  fa.ng = ng;
  fa.nstate = nstate;
  fa.nocc = nocc;
  fa.nv1 = nv1;
  fa.nc1 = nc1;
  fa.nv2 = nv2;
  fa.nc2 = nc2;
  fa.rk = rk_fit;
  fa.piv = piv;
  fa.d_theta = d_theta;
  FitResult fr;
  int rc = opt.precision == ISDF_PRECISION_MIXED ? fit_mixed(fa, arena, s, &fr, opt.mixed_slices)
                                                 : fit_fp64(fa, arena, s, &fr);
  rep.chol_info = fr.chol_info;
  rep.kernel_launches += fr.launches;
  rep.t_zct_ms = fr.t_zct_ms;
  rep.t_chol_ms = fr.t_chol_ms;
  rep.t_solve_ms = fr.t_solve_ms;
  rep.t_gemm_ms = fr.t_gemm_ms > 0.f ? fr.t_gemm_ms : fr.t_solve_ms;
  if (rc != ISDF_OK) {
    if (rep_out) *rep_out = rep;
    return rc;
  }
  if (rk_fit < rk)
    ISDF_CUDA(cudaMemsetAsync(d_theta + (size_t)rk_fit * ng, 0,
                              sizeof(double) * (size_t)(rk - rk_fit) * ng, s));
  ISDF_CUDA(cudaStreamSynchronize(s));
  rep.t_fit_ms = ms_since(t1);
  if (fit_guard.owns_lock()) fit_guard.unlock();
  if (check) {
    // (e) the check of src/common/isdf.cpp:193-206 -> checkcode.cpp
    auto t2 = std::chrono::steady_clock::now();
    arena.off = mark;
    CheckArgs ca;
    ca.d_psi = d_psi;
    for (int i = 0; i < 3; ++i) {
      ca.num_grid[i] = dom->num_grid[i];
      ca.length[i] = dom->length[i];
    }
    ca.nstate = nstate;
    ca.nocc = nocc;
    ca.nv1 = nv1;
    ca.nc1 = nc1;
    ca.nv2 = nv2;
    ca.nc2 = nc2;
    ca.rk = rk_fit;
    ca.piv = piv;
    ca.d_theta = d_theta;
    ISDF_TRY(check_run(ca, arena, s, &rep.fit_err, &rep.coul_err));
    rep.t_check_ms = ms_since(t2);
  }
  rep.t_total_ms = ms_since(t0);
  if (rep_out) *rep_out = rep;
  return ISDF_OK;
}

}  // namespace isdf_b200

using namespace isdf_b200;

extern "C" {

void isdf_default_options(isdf_options_t* opt) {
  if (!opt) return;
  std::memset(opt, 0, sizeof(*opt));
  opt->precision = ISDF_PRECISION_FP64;
  opt->refine_steps = 0;
  opt->qrcp_oversample = 1.5;
  opt->qrcp_seed = 41;
  opt->rand_seed = -1;
  opt->stream = nullptr;
  opt->mixed_slices = kDefaultMixedSlices;
}

int isdf_solve(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1,
               int nc1, int nv2, int nc2, int mu_points, double* d_theta, int* piv,
               int kmeans_max_iter, int selector, int check, const isdf_options_t* opt,
               isdf_report_t* rep) {
  try {
    return solve(dom, d_psi, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_theta, piv,
                 kmeans_max_iter, selector, check, opt, rep, nullptr);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  } catch (...) {
    return record_error(ISDF_ERR_CUDA, "unknown exception");
  }
}

int isdf_kmeans_weight(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1,
                       int nv2, int nc2, double* d_w, void* stream) {
  if (!d_psi || !d_w || ng <= 0) return record_error(ISDF_ERR_ARG, "bad weight arguments");
  ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
  return kmeans_weight(d_psi, ng, nocc, nv1, nc1, nv2, nc2, d_w, (cudaStream_t)stream);
}

int isdf_kmeans_select(const isdf_domain_t* dom, const double* d_w, int mu, int max_iter,
                       long long rand_seed, int* piv, int* rk_eff, int* iters, int* npt,
                       void* stream) {
  try {
    if (!dom || !d_w || !piv) return record_error(ISDF_ERR_ARG, "null pointer");
    const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
    if (ng <= 0 || mu <= 0 || mu > ng || max_iter < 0) return record_error(ISDF_ERR_ARG, "sizes");
    if (mu > kKmeansMaxMu) return record_error(ISDF_ERR_UNSUPPORTED, "mu above the K-means limit");
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    ISDF_TRY(acquire_workspace(kmeans_workspace_bytes(ng, mu) + 4096, &arena, &ls));
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
    ISDF_TRY(kmeans_select(ka, arena, stream ? (cudaStream_t)stream : ls, &kr));
    if (rk_eff) *rk_eff = kr.rk_eff;
    if (iters) *iters = kr.iters;
    if (npt) *npt = kr.npt;
    return ISDF_OK;
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_kmeans_select_batch(int count, const isdf_domain_t* doms, const double* const* d_w,
                             const int* mu, const int* max_iter, long long rand_seed,
                             int* const* piv, int* rk_eff, int* iters, int* npt, void* stream) {
  try {
    if (count <= 0 || !doms || !d_w || !mu || !max_iter || !piv)
      return record_error(ISDF_ERR_ARG, "kmeans batch: null argument");
    std::vector<KmeansArgs> args(count);
    size_t need = 4096;
    for (int r = 0; r < count; ++r) {
      const isdf_domain_t& d = doms[r];
      const long long ng = (long long)d.num_grid[0] * d.num_grid[1] * d.num_grid[2];
      if (!d_w[r] || !piv[r] || d.num_grid[0] <= 0 || d.num_grid[1] <= 0 || d.num_grid[2] <= 0 ||
          mu[r] <= 0 || mu[r] > ng || max_iter[r] < 0)
        return record_error(ISDF_ERR_ARG, "kmeans batch: bad request");
      KmeansArgs& a = args[r];
      a.d_w = d_w[r];
      a.ng = ng;
      for (int i = 0; i < 3; ++i) {
        a.num_grid[i] = d.num_grid[i];
        a.length[i] = d.length[i];
      }
      a.mu = mu[r];
      a.max_iter = max_iter[r];
      a.rand_seed = rand_seed;
      a.piv = piv[r];
      need += kmeans_batch_workspace_bytes(ng, mu[r]);
    }
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    ISDF_TRY(acquire_workspace(need, &arena, &ls));
    std::vector<KmeansResult> res(count);
    ISDF_TRY(kmeans_select_batch(args.data(), count, arena, stream ? (cudaStream_t)stream : ls,
                                 res.data()));
    for (int r = 0; r < count; ++r) {
      if (rk_eff) rk_eff[r] = res[r].rk_eff;
      if (iters) iters[r] = res[r].iters;
      if (npt) npt[r] = res[r].npt;
    }
    return ISDF_OK;
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_fit(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1, int nv2,
             int nc2, int rk, const int* piv, double* d_theta, int precision, int refine_steps,
             int* chol_info, void* stream) {
  try {
    if (!d_psi || !d_theta || !piv || ng <= 0 || rk <= 0 || rk > ng)
      return record_error(ISDF_ERR_ARG, "bad fit arguments");
    if (refine_steps != 0)
      return record_error(ISDF_ERR_UNSUPPORTED,
                          "refine_steps must be 0: FP64 refinement of the theta solve is not built");
    ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
    for (int j = 0; j < rk; ++j)
      if (piv[j] < 0 || piv[j] >= ng) return record_error(ISDF_ERR_ARG, "pivot outside the grid");
    if (precision != ISDF_PRECISION_FP64 && precision != ISDF_PRECISION_MIXED)
      return record_error(ISDF_ERR_ARG, "unknown precision");
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    const size_t need = precision == ISDF_PRECISION_MIXED
                            ? fit_mixed_workspace_bytes(ng, nstate, rk, kDefaultMixedSlices)
                            : fit_workspace_bytes(ng, nstate, rk);
    ISDF_TRY(acquire_workspace(need + 4096, &arena, &ls));
    FitArgs fa;
    fa.d_psi = d_psi;
    fa.ng = ng;
    fa.nstate = nstate;
    fa.nocc = nocc;
    fa.nv1 = nv1;
    fa.nc1 = nc1;
    fa.nv2 = nv2;
    fa.nc2 = nc2;
    fa.rk = rk;
    fa.piv = piv;
    fa.d_theta = d_theta;
    FitResult fr;
    cudaStream_t s = stream ? (cudaStream_t)stream : ls;
    int rc = precision == ISDF_PRECISION_MIXED ? fit_mixed(fa, arena, s, &fr, kDefaultMixedSlices)
                                               : fit_fp64(fa, arena, s, &fr);
    if (chol_info) *chol_info = fr.chol_info;
    if (rc == ISDF_OK) ISDF_CUDA(cudaStreamSynchronize(s));
    return rc;
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_check(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate, int nv1,
               int nc1, int nv2, int nc2, int rk, const int* piv, const double* d_theta,
               double* fit_err, double* coul_err, void* stream) {
  try {
    if (!dom || !d_psi || !d_theta || !piv || !fit_err || !coul_err)
      return record_error(ISDF_ERR_ARG, "null pointer");
    const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
    if (ng <= 0 || rk <= 0 || rk > ng) return record_error(ISDF_ERR_ARG, "sizes");
    ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
    for (int j = 0; j < rk; ++j)
      if (piv[j] < 0 || piv[j] >= ng) return record_error(ISDF_ERR_ARG, "pivot outside the grid");
    const size_t need = check_workspace_bytes(dom->num_grid, nstate, rk, (nv1 + nc1) * (nv2 + nc2));
    if (need > kCheckMaxBytes)
      return record_error(ISDF_ERR_UNSUPPORTED, "check: pair spectra exceed the device budget");
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    ISDF_TRY(acquire_workspace(need + 4096, &arena, &ls));
    CheckArgs ca;
    ca.d_psi = d_psi;
    for (int i = 0; i < 3; ++i) {
      ca.num_grid[i] = dom->num_grid[i];
      ca.length[i] = dom->length[i];
    }
    ca.nstate = nstate;
    ca.nocc = nocc;
    ca.nv1 = nv1;
    ca.nc1 = nc1;
    ca.nv2 = nv2;
    ca.nc2 = nc2;
    ca.rk = rk;
    ca.piv = piv;
    ca.d_theta = d_theta;
    return check_run(ca, arena, stream ? (cudaStream_t)stream : ls, fit_err, coul_err);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_check_sampled(const isdf_domain_t* dom, const double* d_psi, int nocc, int nstate,
                       int nv1, int nc1, int nv2, int nc2, int rk, const int* piv,
                       const double* d_theta, int npair_sample, const int* pairs,
                       double* fit_err, double* coul_err, void* stream) {
  try {
    if (!dom || !d_psi || !d_theta || !piv || !pairs || !fit_err || !coul_err)
      return record_error(ISDF_ERR_ARG, "null pointer");
    const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
    if (ng <= 0 || rk <= 0 || rk > ng) return record_error(ISDF_ERR_ARG, "sizes");
    ISDF_TRY(check_state_ranges(nocc, nstate, nv1, nc1, nv2, nc2));
    const int npair = (nv1 + nc1) * (nv2 + nc2);
    if (npair_sample < 1 || npair_sample > 4096)
      return record_error(ISDF_ERR_ARG, "sampled check: npair_sample in [1, 4096]");
    for (int i = 0; i < npair_sample; ++i)
      if (pairs[i] < 0 || pairs[i] >= npair)
        return record_error(ISDF_ERR_ARG, "sampled check: pair index outside [0, Npair)");
    for (int j = 0; j < rk; ++j)
      if (piv[j] < 0 || piv[j] >= ng) return record_error(ISDF_ERR_ARG, "pivot outside the grid");
    const size_t need = check_sampled_workspace_bytes(dom->num_grid, rk, npair_sample);
    if (need > kCheckMaxBytes)
      return record_error(ISDF_ERR_UNSUPPORTED, "sampled check: buffers exceed the device budget");
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    ISDF_TRY(acquire_workspace(need + 4096, &arena, &ls));
    CheckArgs ca;
    ca.d_psi = d_psi;
    for (int i = 0; i < 3; ++i) {
      ca.num_grid[i] = dom->num_grid[i];
      ca.length[i] = dom->length[i];
    }
    ca.nstate = nstate;
    ca.nocc = nocc;
    ca.nv1 = nv1;
    ca.nc1 = nc1;
    ca.nv2 = nv2;
    ca.nc2 = nc2;
    ca.rk = rk;
    ca.piv = piv;
    ca.d_theta = d_theta;
    return check_sampled_run(ca, pairs, npair_sample, arena, stream ? (cudaStream_t)stream : ls,
                             fit_err, coul_err);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

int isdf_coulomb_matrix(const isdf_domain_t* dom, const double* d_theta, int rk, double* d_A,
                        void* stream) {
  try {
    if (!dom || !d_theta || !d_A) return record_error(ISDF_ERR_ARG, "null pointer");
    const long long ng = (long long)dom->num_grid[0] * dom->num_grid[1] * dom->num_grid[2];
    if (dom->num_grid[0] <= 0 || dom->num_grid[1] <= 0 || dom->num_grid[2] <= 0 || rk <= 0 ||
        rk > ng)
      return record_error(ISDF_ERR_ARG, "sizes");
    const size_t need = coulomb_matrix_workspace_bytes(dom->num_grid, rk);
    std::lock_guard<std::mutex> lock(workspace_mutex());
    Arena arena;
    cudaStream_t ls;
    ISDF_TRY(acquire_workspace(need + 4096, &arena, &ls));
    return coulomb_matrix_run(dom->num_grid, dom->length, d_theta, rk, d_A, arena,
                              stream ? (cudaStream_t)stream : ls);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  }
}

const char* isdf_last_error(void) { return last_error_message(); }

const char* isdf_status_string(int code) {
  switch (code) {
    case ISDF_OK: return "ok";
    case ISDF_ERR_ARG: return "invalid argument";
    case ISDF_ERR_CUDA: return "CUDA error";
    case ISDF_ERR_NOMEM: return "out of device memory";
    case ISDF_ERR_NOT_SPD: return "C C^T + eps I is not positive definite";
    case ISDF_ERR_TIMEOUT: return "device wait timed out";
    case ISDF_ERR_UNSUPPORTED: return "unsupported shape or option";
    case ISDF_ERR_CANCELLED: return "cancelled";
    case ISDF_ERR_BUSY: return "queue full";
    case ISDF_ERR_COMM: return "collective failed";
    default: return "unknown status";
  }
}

size_t isdf_workspace_bytes(long long ng, int nstate, int mu, int selector, int precision,
                            int check) {
  (void)check;  // the check's buffers depend on the grid's shape: see the request variant
  return solve_workspace_bytes(ng, nstate, mu, selector, precision, 0, 1.5, nullptr, 0);
}

size_t isdf_request_workspace_bytes(const isdf_domain_t* dom, int nstate, int nv1, int nc1,
                                    int nv2, int nc2, int mu_points, int selector, int check,
                                    const isdf_options_t* opt) {
  if (!dom || nstate <= 0 || nv1 < 0 || nc1 < 0 || nv2 < 0 || nc2 < 0 || nv1 + nc1 <= 0 ||
      nv2 + nc2 <= 0 || mu_points < 0)
    return 0;
  for (int i = 0; i < 3; ++i)
    if (dom->num_grid[i] <= 0) return 0;
  return request_footprint(dom, nstate, nv1, nc1, nv2, nc2, mu_points, selector, check, opt);
}

void isdf_release_workspace(void) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return;
  std::lock_guard<std::mutex> lock(g_cache[dev].mu);
  if (g_cache[dev].buf) {
    cudaDeviceSynchronize();
    cudaFree(g_cache[dev].buf);
  }
  g_cache[dev].buf = nullptr;
  g_cache[dev].cap = 0;
}

}  // extern "C"
