// Test infrastructure only (oracle): a CPU restatement of the reference's
// K-means interpolation-point selection for one rank, written to reproduce
// its floating-point results bit for bit. It is the checker for the GPU
// K-means kernels and the "port" CPU baseline; product code never links it.
//
// Reference behaviour followed (file:line in the reference tree):
//  * weight  w(r) = (sum_{S2} psi^2) * (sum_{S1} psi^2), sequential sums per
//    point, S2 first: src/cpu/getpoints_Kmeans_MPI.cpp:33-45.
//  * KMEAN: src/common/utility.cpp:631-988, at world size 1 (nptLocal = n):
//    - filter w > 1e-8 * max(w, 0) (findMax starts at 0.0,
//      include/common/numvec_impl.hpp:259-266), utility.cpp:646-665;
//    - the index list keeps its zero-initialised tail, so points i >= npt
//      alias grid point 0 with weight w[0] and join every assignment and
//      update (utility.cpp:648,659,707-713);
//    - coordinates from the grid index by the formula of utility.cpp:711-713;
//    - initial centroids = the first rk kept points (utility.cpp:750-762), or
//      with a warm start (piv[0] != piv[1] on entry, utility.cpp:725-749) the
//      previous pivots whose weight passes the filter, topped up with the
//      first kept points not among them (port_kmeans_warm; the reference's
//      ISDF() zeroes piv first, so only a caller of KMEAN reaches this);
//    - distances ((dx*dx + dy*dy) + dz*dz), no FMA (utility.cpp:598-615);
//    - per-point argmin over centroids, first minimum wins (utility.cpp:579-595);
//    - centroid sums accumulated in point order (utility.cpp:814-822);
//    - empty clusters replaced by the last centroid, rk-- (utility.cpp:831-853);
//    - stop once <= 1e-5 * n labels change or after max_iter (utility.cpp:812-922);
//    - per-centroid nearest point, first minimum over points (std::min_element,
//      utility.cpp:564-578,926-945), sorted and de-duplicated (unique,
//      utility.cpp:617-629), rk shrinks to the distinct count (utility.cpp:970-972);
//    - piv = [selected ascending | the other grid points ascending]
//      (utility.cpp:973-983).
//  * the npt < rk early return with std::random_shuffle (utility.cpp:667-681).
//
// Build: g++ -O2 -std=c++14 -fopenmp (no -march: no FMA contraction, like
// the reference's build, Makefile:102,159). OpenMP splits only loops whose
// iterations are independent (per-point argmin, per-centroid nearest point),
// so the result does not depend on the thread count.
#include <cstdlib>
#include <cstring>
#include <vector>
#include <algorithm>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

inline void coords(int tmp, const int* nG, const double* dx, double* gx, double* gy, double* gz) {
  *gx = (tmp % nG[0]) * dx[0];
  *gy = (tmp % (nG[0] * nG[1]) - *gx / dx[0]) / nG[0] * dx[1];
  *gz = (tmp - *gx / dx[0] - *gy / dx[1] * nG[0]) / (nG[0] * nG[1]) * dx[2];
}

// libstdc++'s std::random_shuffle(first, last) loop, driven by std::rand().
void shuffle_like_libstdcxx(int* first, int* last) {
  if (first == last) return;
  for (int* i = first + 1; i != last; ++i) {
    int* j = first + std::rand() % ((i - first) + 1);
    if (i != j) std::swap(*i, *j);
  }
}

}  // namespace

extern "C" {

void port_weight(const double* psi, long long ng, int nocc, int nv1, int nc1, int nv2, int nc2,
                 double* w) {
  for (long long kk = 0; kk < ng; kk++) {
    double sumI = 0.0, sumJ = 0.0;
    for (int i = nocc - nv2; i < nocc + nc2; i++) {
      double v = psi[(size_t)i * ng + kk];
      sumI += v * v;
    }
    for (int j = nocc - nv1; j < nocc + nc1; j++) {
      double v = psi[(size_t)j * ng + kk];
      sumJ += v * v;
    }
    w[kk] = 0.0 + sumI * sumJ;
  }
}

// Returns rk_eff (>= 1) or a negative code. iters_out: Lloyd iterations run
// (-1 on the early-return branch). rand_seed >= 0 reseeds std::rand first
// (only the early-return branch draws from it); < 0 keeps the process state.
// warm != 0: piv holds the previous pivots on entry (used when piv[0] !=
// piv[1]); *warm_used receives how many of them were kept (-1: cold start).
//
// ranks > 1 restates KMEAN run as that many MPI ranks (utility.cpp:682-700,
// 813-830, 946-969): rank r owns the points [r n/p + min(r, n%p), +n/p +
// (r < n%p)) of the n-long index list (zero tail included) and folds its
// own centroid sums in its point order; the ranks' sums are combined by a
// binomial tree (at step s = 1, 2, 4, ..., rank q takes in rank q + s: the
// order of MPICH's binomial reduce, and the only order at 2 ranks); the
// nearest point of each centroid is each rank's first minimum, then the
// smallest distance over the ranks with ties to the smaller grid index
// (MPI_MINLOC). Everything else is the one-rank algorithm.
int port_kmeans_ranks(const double* w, int n, const int* nG, const double* len, int rk,
                      int max_iter, long long rand_seed, int* piv, int* iters_out, int warm,
                      int* warm_used, int ranks) {
  if (ranks < 1 || ranks > n) return -3;
  if (rand_seed >= 0) std::srand((unsigned)rand_seed);
  const double kmeans_tol = 1e-5, df_tol = 1e-8;
  std::vector<int> prev;
  if (warm && n > 1 && piv[0] != piv[1]) {
    prev.assign(piv, piv + rk);
    for (int v : prev)
      if (v < 0 || v >= n) return -2;
  }
  if (warm_used) *warm_used = -1;
  std::memset(piv, 0, sizeof(int) * (size_t)n);
  double maxW = 0.0;
  for (int i = 0; i < n; i++)
    if (w[i] > maxW) maxW = w[i];
  std::vector<int> index(n, 0);
  int npt = 0;
  for (int i = 0; i < n; i++)
    if (w[i] > df_tol * maxW) index[npt++] = i;
  *iters_out = -1;
  if (npt < rk) {
    int k0 = 0, k1 = 0;
    for (int i = 0; i < npt; i++) {
      if (i == index[k0]) {
        piv[k0] = i;
        k0 = std::min(k0 + 1, rk - 1);
      } else {
        piv[npt + k1] = i;
        k1++;
      }
    }
    shuffle_like_libstdcxx(piv + npt, piv + n);
    return rk;
  }
  double dx[3];
  for (int i = 0; i < 3; i++) dx[i] = len[i] / nG[i];
  std::vector<double> gx(n), gy(n), gz(n), wl(n);
  for (int i = 0; i < n; i++) {
    int tmp = index[i];  // i >= npt: the zero tail, grid point 0
    wl[i] = w[tmp];
    coords(tmp, nG, dx, &gx[i], &gy[i], &gz[i]);
  }
  std::vector<double> cx(rk), cy(rk), cz(rk), cnt(rk);
  std::vector<int> cinit(index.begin(), index.begin() + rk);
  if (!prev.empty()) {
    cinit.clear();
    for (int i = 0; i < rk; i++)
      if (w[prev[i]] > df_tol * maxW) cinit.push_back(prev[i]);
    if (warm_used) *warm_used = (int)cinit.size();
    std::vector<char> in(n, 0);
    for (int c : cinit) in[c] = 1;
    for (int k = 0; (int)cinit.size() < rk && k < npt; k++)
      if (!in[index[k]]) cinit.push_back(index[k]);
  }
  for (int j = 0; j < rk; j++) coords(cinit[j], nG, dx, &cx[j], &cy[j], &cz[j]);

  auto dist = [&](int i, int j) {
    double d1 = gx[i] - cx[j], d2 = gy[i] - cy[j], d3 = gz[i] - cz[j];
    return d1 * d1 + d2 * d2 + d3 * d3;
  };
  // rank r's point range
  std::vector<int> lo(ranks + 1);
  for (int r = 0; r <= ranks; ++r) lo[r] = r * (n / ranks) + std::min(r, n % ranks);
  std::vector<int> label(n), last(n);
  // Each point's argmin is independent, so the points are split over
  // OpenMP threads; every distance is still evaluated exactly as above.
  auto assign = [&]() {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; i++) {
      double best = dist(i, 0);
      int bj = 0;
      for (int j = 1; j < rk; j++) {
        double d = dist(i, j);
        if (d < best) {
          best = d;
          bj = j;
        }
      }
      label[i] = bj;
    }
  };
  assign();
  const double maxF = kmeans_tol * n;
  int flag = n, s = 0;
  while (flag > maxF && s < max_iter) {
    std::fill(cnt.begin(), cnt.end(), 0.0);
    std::fill(cx.begin(), cx.end(), 0.0);
    std::fill(cy.begin(), cy.end(), 0.0);
    std::fill(cz.begin(), cz.end(), 0.0);
    if (ranks == 1) {
      for (int i = 0; i < n; i++) {
        int t = label[i];
        cnt[t] += wl[i];
        cx[t] += wl[i] * gx[i];
        cy[t] += wl[i] * gy[i];
        cz[t] += wl[i] * gz[i];
      }
    } else {
      // per-rank sums [cnt | cx | cy | cz], then the binomial combine
      std::vector<std::vector<double>> part(ranks, std::vector<double>(4 * (size_t)rk, 0.0));
      for (int r = 0; r < ranks; ++r) {
        double* q = part[r].data();
        for (int i = lo[r]; i < lo[r + 1]; i++) {
          int t = label[i];
          q[t] += wl[i];
          q[rk + t] += wl[i] * gx[i];
          q[2 * rk + t] += wl[i] * gy[i];
          q[3 * rk + t] += wl[i] * gz[i];
        }
      }
      for (int st = 1; st < ranks; st *= 2)
        for (int r = 0; r + st < ranks; r += 2 * st)
          for (size_t e = 0; e < 4 * (size_t)rk; ++e) part[r][e] = part[r][e] + part[r + st][e];
      for (int t = 0; t < rk; ++t) {
        cnt[t] = part[0][t];
        cx[t] = part[0][rk + t];
        cy[t] = part[0][2 * rk + t];
        cz[t] = part[0][3 * rk + t];
      }
    }
    for (int i = 0; i < rk; i++) {
      if (cnt[i] != 0.0) {
        cx[i] = cx[i] / cnt[i];
        cy[i] = cy[i] / cnt[i];
        cz[i] = cz[i] / cnt[i];
      } else {
        rk--;
        cx[i] = cx[rk];
        cy[i] = cy[rk];
        cz[i] = cz[rk];
        cnt[i] = cnt[rk];
        i--;
      }
    }
    cx.resize(rk);
    cy.resize(rk);
    cz.resize(rk);
    cnt.resize(rk);
    last = label;
    assign();
    flag = 0;
    for (int i = 0; i < n; i++)
      if (last[i] != label[i]) flag++;
    s++;
  }
  *iters_out = s;
  // Nearest point to each centroid: each rank's first minimum over its
  // points, then the smallest distance over the ranks, ties to the smaller
  // grid index (at one rank: the first minimum over all points).
  std::vector<int> sel(rk);
#pragma omp parallel for schedule(dynamic, 16)
  for (int j = 0; j < rk; j++) {
    double gbest = 0.0;
    int gsel = -1;
    for (int r = 0; r < ranks; ++r) {
      double best = dist(lo[r], j);
      int bi = lo[r];
      for (int i = lo[r] + 1; i < lo[r + 1]; i++) {
        double d = dist(i, j);
        if (d < best) {
          best = d;
          bi = i;
        }
      }
      const int g = index[bi];
      if (gsel < 0 || best < gbest || (best == gbest && g < gsel)) {
        gbest = best;
        gsel = g;
      }
    }
    sel[j] = gsel;
  }
  std::sort(sel.begin(), sel.end());
  sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
  rk = (int)sel.size();
  int k0 = 0, k1 = 0;
  for (int i = 0; i < n; i++) {
    if (i == sel[k0]) {
      piv[k0] = i;
      k0 = std::min(k0 + 1, rk - 1);
    } else {
      piv[rk + k1] = i;
      k1++;
    }
  }
  return rk;
}

int port_kmeans_warm(const double* w, int n, const int* nG, const double* len, int rk,
                     int max_iter, long long rand_seed, int* piv, int* iters_out, int warm,
                     int* warm_used) {
  return port_kmeans_ranks(w, n, nG, len, rk, max_iter, rand_seed, piv, iters_out, warm,
                           warm_used, 1);
}

int port_kmeans(const double* w, int n, const int* nG, const double* len, int rk, int max_iter,
                long long rand_seed, int* piv, int* iters_out) {
  return port_kmeans_warm(w, n, nG, len, rk, max_iter, rand_seed, piv, iters_out, 0, nullptr);
}

int port_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

}  // extern "C"
