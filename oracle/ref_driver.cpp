// Test infrastructure only (oracle). Thin extern "C" entry points into the
// reference's own CPU sources for the ISDF path, compiled unmodified from
// src/common/utility.cpp (KMEAN), src/cpu/getpoints_Kmeans_MPI.cpp (weight +
// KMEAN), src/cpu/getbasis_MPI.cpp (the FP64 fit) and src/common/checkcode.cpp
// + src/common/fourier.cpp (the Coulomb check), with the single-rank MPI and
// FFTW shims in oracle/shims. Built by oracle/build_ref.sh into oracle/_ref/.
//
// Only the tests, the smoke check and the CPU-baseline leg of bench.py load
// the library this file builds; the product never does.
#include "isdf.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>

using namespace isdf;

namespace {

Domain make_domain(const int* ng, const double* len) {
  Domain d;
  d.length = Point3(len[0], len[1], len[2]);
  d.posStart = Point3(0.0, 0.0, 0.0);
  d.numGrid = Index3(ng[0], ng[1], ng[2]);
  d.numGridFine = Index3(ng[0], ng[1], ng[2]);
  return d;
}

// Routes the reference's log stream (isdfOFS) into a string for one call.
struct LogCapture {
  std::stringbuf buf;
  std::streambuf* old;
  LogCapture() {
    std::ostream& os = isdfOFS;
    old = os.rdbuf(&buf);
    os.clear();
    os.precision(17);
  }
  ~LogCapture() {
    std::ostream& os = isdfOFS;
    os.rdbuf(old);
  }
  std::string str() const { return buf.str(); }
};

int parse_after(const std::string& log, const std::string& key, double* out) {
  size_t p = log.rfind(key);
  if (p == std::string::npos) return -1;
  *out = std::strtod(log.c_str() + p + key.size(), nullptr);
  return 0;
}

void copy_log(const std::string& s, char* log, int loglen) {
  if (!log || loglen <= 0) return;
  std::snprintf(log, (size_t)loglen, "%s", s.c_str());
}

}  // namespace

extern "C" {

// Weight w(r) = sum_{S2} psi^2 * sum_{S1} psi^2, the loop of
// src/cpu/getpoints_Kmeans_MPI.cpp:33-45 restated for one rank (the reference
// keeps it inside getpoints_Kmeans_MPI, which also runs KMEAN).
void ref_weight(const double* psi, int ng_total, int nocc, int nv1, int nc1, int nv2, int nc2,
                double* w) {
  std::vector<double> sumI(ng_total, 0.0), sumJ(ng_total, 0.0);
  for (int i = nocc - nv2; i < nocc + nc2; i++)
    for (int kk = 0; kk < ng_total; kk++)
      sumI[kk] += psi[(size_t)i * ng_total + kk] * psi[(size_t)i * ng_total + kk];
  for (int j = nocc - nv1; j < nocc + nc1; j++)
    for (int kk = 0; kk < ng_total; kk++)
      sumJ[kk] += psi[(size_t)j * ng_total + kk] * psi[(size_t)j * ng_total + kk];
  for (int kk = 0; kk < ng_total; kk++) w[kk] = 0.0 + sumI[kk] * sumJ[kk];
}

// The reference's KMEAN called directly with the caller's piv, as an SCF
// loop that keeps piv between solves would call it: when piv[0] != piv[1] on
// entry KMEAN starts from those pivots (src/common/utility.cpp:725-749), the
// warm start that the reference's ISDF() never reaches because it zeroes piv
// first (src/common/isdf.cpp:174-175). w: the weight; *reused: the count the
// reference logs as "Reusable pivots" (-1 when it logged none).
int ref_kmeans_warm(const double* w, const int* ng, const double* len, int mu, int iters,
                    int* piv, int* rk_eff, int* n_iter, int* reused, char* log, int loglen) {
  try {
    LogCapture cap;
    Domain dom = make_domain(ng, len);
    const int n = dom.NumGridTotal();
    DblNumVec weight(n);
    std::memcpy(weight.Data(), w, sizeof(double) * n);
    Int rk = mu;
    KMEAN(n, weight, rk, 1e-5, iters, 1e-8, dom, piv);
    *rk_eff = rk;
    std::string s = cap.str();
    double v = -1;
    *n_iter = parse_after(s, "Converged in ", &v) == 0 ? (int)v : -1;
    v = -1;
    *reused = parse_after(s, "Reusable pivots: ", &v) == 0 ? (int)v : -1;
    copy_log(s, log, loglen);
    return 0;
  } catch (const std::exception& e) {
    copy_log(e.what(), log, loglen);
    return -1;
  }
}

// The K-means point selection of the GPU ISDF() path: weight, then KMEAN
// (src/common/utility.cpp:631-988) with the tolerances of
// src/cuda/isdf-gpu.cpp:31-32, piv zeroed first as src/common/isdf.cpp:174-175
// does. rk_eff receives the (possibly shrunk) number of selected points.
// When cross_check is set the reference's getpoints_Kmeans_MPI is also run on
// the same input and its piv must equal this one (returns -100 otherwise).
int ref_kmeans_piv(const double* psi, const int* ng, const double* len, int nocc, int nstate,
                   int nv1, int nc1, int nv2, int nc2, int mu, int iters, unsigned rand_seed,
                   int cross_check, int* piv, int* rk_eff, int* n_iter, double* weight_out,
                   char* log, int loglen) {
  try {
    LogCapture cap;
    Domain dom = make_domain(ng, len);
    const int n = dom.NumGridTotal();
    DblNumVec weight(n);
    ref_weight(psi, n, nocc, nv1, nc1, nv2, nc2, weight.Data());
    if (weight_out) std::memcpy(weight_out, weight.Data(), sizeof(double) * n);
    std::memset(piv, 0, sizeof(int) * n);
    Int rk = mu;
    std::srand(rand_seed);
    KMEAN(n, weight, rk, 1e-5, iters, 1e-8, dom, piv);
    *rk_eff = rk;
    std::string s = cap.str();
    double it = -1;
    *n_iter = parse_after(s, "Converged in ", &it) == 0 ? (int)it : -1;
    if (cross_check) {
      std::vector<int> piv2(n, 0);
      DblNumMat psiRow(n, nstate, false, const_cast<double*>(psi));
      IntNumVec pv(n, false, piv2.data());
      Int ntot = n, mu_ = mu, it_ = iters;
      Real tmpi = 0.0;
      std::srand(rand_seed);
      isdffunc::getpoints_Kmeans_MPI(psiRow, dom, nocc, nv1, nc1, nv2, nc2, ntot, mu_, pv, tmpi,
                                     it_);
      if (std::memcmp(piv2.data(), piv, sizeof(int) * n) != 0) return -100;
    }
    copy_log(s, log, loglen);
    return 0;
  } catch (const std::exception& e) {
    copy_log(e.what(), log, loglen);
    return -1;
  }
}

// The FP64 fit of src/cpu/getbasis_MPI.cpp:9-250 at one rank: gather psi(mu),
// GEMM (+ second GEMM when S1 != S2), Hadamard product, C C^T gather, +eps*I,
// dpotrf, two dtrsm. theta is Ng x rk column-major. Pass the rk that the
// selector produced (the GPU path fits with the shrunk rk, isdf-gpu.cpp:99).
int ref_getbasis(const double* psi, const int* ng, const double* len, int nocc, int nstate,
                 int nv1, int nc1, int nv2, int nc2, int rk, const int* piv, double* theta,
                 char* log, int loglen) {
  try {
    LogCapture cap;
    Domain dom = make_domain(ng, len);
    const int n = dom.NumGridTotal();
    DblNumMat psiRow(n, nstate, false, const_cast<double*>(psi));
    DblNumMat psiCol(n, nstate);
    std::memcpy(psiCol.Data(), psi, sizeof(double) * (size_t)n * nstate);
    IntNumVec pv(n, false, const_cast<int*>(piv));
    DblNumMat out(n, rk, false, theta);
    Int ntot = n;
    Real tmpi = 0.0;
    isdffunc::getbasis_MPI(psiRow, psiCol, dom, nocc, nv1, nc1, nv2, nc2, ntot, rk, out, pv, tmpi);
    copy_log(cap.str(), log, loglen);
    return 0;
  } catch (const std::exception& e) {
    copy_log(e.what(), log, loglen);
    return -1;
  }
}

// The check of src/common/checkcode.cpp:54-313 (pair-density fit error and
// truncated-Coulomb 4-index error), read back from the lines it prints.
int ref_checkcode(const double* psi, const int* ng, const double* len, int nocc, int nstate,
                  int nv1, int nc1, int nv2, int nc2, int rk, const int* piv, const double* theta,
                  double* fit_err, double* coul_err, char* log, int loglen) {
  try {
    LogCapture cap;
    Domain dom = make_domain(ng, len);
    const int n = dom.NumGridTotal();
    DblNumMat psiRow(n, nstate, false, const_cast<double*>(psi));
    DblNumMat psiCol(n, nstate);
    std::memcpy(psiCol.Data(), psi, sizeof(double) * (size_t)n * nstate);
    IntNumVec pv(n, false, const_cast<int*>(piv));
    DblNumMat th(n, rk);
    std::memcpy(th.Data(), theta, sizeof(double) * (size_t)n * rk);
    Int ntot = n;
    Fourier fft;
    fft.Initialize(dom);
    isdffunc::checkcode(psiRow, psiCol, dom, nocc, nv1, nc1, nv2, nc2, ntot, rk, th, pv, fft);
    std::string s = cap.str();
    copy_log(s, log, loglen);
    if (parse_after(s, "sqrt((rhoij-rho^hat)^2)/sqrt(rhoij^2)=", fit_err)) return -2;
    if (parse_after(s, "sqrt((ijkl-ijkl^hat)^2)/sqrt(ijkl^2) =", coul_err)) return -3;
    return 0;
  } catch (const std::exception& e) {
    copy_log(e.what(), log, loglen);
    return -1;
  }
}

// Seconds for one K-means Lloyd step of the reference at full size: its
// pdist2 (utility.cpp:598-615) of npt grid points against rk centroids and its
// findMin over centroids (utility.cpp:535-562), i.e. the per-iteration work of
// KMEAN's loop (utility.cpp:878-901). Best of `repeats`.
double ref_bench_kmeans_step(int npt, int rk, int repeats) {
  DblNumMat grid(npt, 3), cen(rk, 3), D;
  for (int i = 0; i < npt; i++) {
    grid(i, 0) = (i % 97) * 0.25;
    grid(i, 1) = ((i / 97) % 89) * 0.25;
    grid(i, 2) = (i / (97 * 89)) * 0.25;
  }
  for (int j = 0; j < rk; j++)
    for (int d = 0; d < 3; d++) cen(j, d) = grid((int)((long long)j * npt / rk), d) + 0.01;
  IntNumVec label;
  double best = 1e300;
  for (int r = 0; r < repeats; r++) {
    double t0 = MPI_Wtime();
    pdist2(grid, cen, D);
    findMin(D, 1, label);
    double t = MPI_Wtime() - t0;
    if (t < best) best = t;
  }
  return best;
}

// Seconds for the reference's KMEAN (src/common/utility.cpp:631-988) on the
// weight w of a grid ng x len with KmeansMaxIter = iters: the whole routine
// as the reference runs it (filter, coordinates, initial assignment, `iters`
// Lloyd iterations each with its host centroid update, pdist2 and findMin,
// the final per-centroid argmin and the piv build). piv: scratch int[Ng].
double ref_bench_kmean(const double* w, const int* ng, const double* len, int mu, int iters,
                       int* piv) {
  LogCapture cap;
  Domain dom = make_domain(ng, len);
  const int n = dom.NumGridTotal();
  DblNumVec weight(n);
  std::memcpy(weight.Data(), w, sizeof(double) * n);
  std::memset(piv, 0, sizeof(int) * n);
  Int rk = mu;
  const double t0 = MPI_Wtime();
  KMEAN(n, weight, rk, 1e-5, iters, 1e-8, dom, piv);
  return MPI_Wtime() - t0;
}

// The QRCP sketch of src/cpu/getpoints_QRCP.cpp:143-189 at rank 0:
// srand48(seed) (the caller's seed; isdf.cpp:68 uses 41), G1 then G2 filled
// column by column with GaussianRandom (include/common/utility.hpp:455-471),
// each orthonormalised by lapack::Orth (dgesvd jobu='O', src/cpu/lapack.cpp:115-147).
void ref_qrcp_sketch(int k1, int k2, int num_pre, long seed, double* g1, double* g2) {
  srand48(seed);
  DblNumMat G1(k1, num_pre), G2(k2, num_pre);
  SetValue(G1, 0.0);
  SetValue(G2, 0.0);
  GaussianRandom(G1);
  GaussianRandom(G2);
  lapack::Orth(k1, num_pre, G1.Data(), k1);
  lapack::Orth(k2, num_pre, G2.Data(), k2);
  std::memcpy(g1, G1.Data(), sizeof(double) * (size_t)k1 * num_pre);
  std::memcpy(g2, G2.Data(), sizeof(double) * (size_t)k2 * num_pre);
}

// The raw Gaussian draws (before Orth), same order.
void ref_qrcp_gaussians(int k1, int k2, int num_pre, long seed, double* g1, double* g2) {
  srand48(seed);
  DblNumMat G1(k1, num_pre), G2(k2, num_pre);
  GaussianRandom(G1);
  GaussianRandom(G2);
  std::memcpy(g1, G1.Data(), sizeof(double) * (size_t)k1 * num_pre);
  std::memcpy(g2, G2.Data(), sizeof(double) * (size_t)k2 * num_pre);
}

// The reference's integer rounding IRound (include/common/utility.hpp:18-23),
// used for the default mu and the QRCP sketch width.
int ref_iround(double a) { return IRound(a); }

}  // extern "C"
