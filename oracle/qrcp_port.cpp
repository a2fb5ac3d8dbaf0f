// Test infrastructure only (oracle): a CPU restatement of the column-pivoted
// Householder QR that the reference's QRCP selector runs on its MG matrix
// (src/cpu/getpoints_QRCP.cpp:436-457 calls ScaLAPACK pdgeqpf through
// src/cpu/scalapack.cpp:33-64; at one rank that is the algorithm of LAPACK
// dgeqpf). It is the checker for the GPU QRCP kernels; product code never
// links it. tests/test_qrcp.py pins it against the LAPACK dgeqpf that scipy's
// OpenBLAS exports (the same pivots on test matrices, including a matrix whose
// pivots differ between downdated and recomputed column norms).
//
// dgeqpf, step i (0-based) of the unblocked loop:
//   pvt = i + idamax(vn1[i..n))                (the first maximal norm)
//   swap columns i and pvt, their jpvt entries and norms
//   H(i) = dlarfg(a[i:m, i]); a[i:m, i+1:n] = H(i) a[i:m, i+1:n]      (dlarf)
//   for every later column j with vn1[j] != 0 (LAPACK Working Note 176):
//     temp  = max(0, 1 - (|a[i, j]| / vn1[j])^2)
//     temp2 = temp * (vn1[j] / vn2[j])^2
//     temp2 <= sqrt(eps): vn1[j] = vn2[j] = ||a[i+1:m, j]||   (recomputed)
//     else:               vn1[j] = vn1[j] * sqrt(temp)         (downdated)
// with eps = 2^-53 (dlamch('Epsilon')).
//
// Extra outputs for the pivot test: per step, the column dgeqpf would pick
// (free_choice), the largest remaining norm (max_norm) and the norm of the
// column actually taken (taken_norm). `forced` (optional) names the column to
// take at each step (-1: dgeqpf's own choice), so that a run can follow
// another implementation's pivot sequence through a near-tie and still check
// every later step.
//
// Build: part of libisdf_port.so (oracle/Makefile), -O2 without -march (no
// FMA contraction); OpenMP over columns, whose updates are independent, so
// the result does not depend on the thread count.
#include <cmath>
#include <cstring>
#include <vector>

namespace {

// ||x||_2 with an extended-precision sum of squares.
double nrm2(const double* x, long long n) {
  long double s = 0.0L;
  for (long long i = 0; i < n; ++i) s += (long double)x[i] * (long double)x[i];
  return (double)std::sqrt(s);
}

double lapy2(double x, double y) {
  const double xa = std::fabs(x), ya = std::fabs(y);
  const double w = xa > ya ? xa : ya, z = xa > ya ? ya : xa;
  if (z == 0.0) return w;
  return w * std::sqrt(1.0 + (z / w) * (z / w));
}

}  // namespace

extern "C" {

// MG columns for the kept grid points idx[0..ntot): column c holds
// x[i + j*p] = B(idx[c], i) * A(idx[c], j)  (getpoints_QRCP.cpp:228-235,
// 272-284), A and B Ng x p column-major. mg: p^2 x ntot, column-major.
void port_qrcp_mg(const double* A, const double* B, long long ng, int p, const int* idx, int ntot,
                  double* mg) {
  const long long m = (long long)p * p;
#pragma omp parallel for schedule(static)
  for (int c = 0; c < ntot; ++c) {
    const long long r = idx[c];
    double* col = mg + (long long)c * m;
    for (int j = 0; j < p; ++j) {
      const double a = A[r + (long long)j * ng];
      for (int i = 0; i < p; ++i) col[i + (long long)j * p] = B[r + (long long)i * ng] * a;
    }
  }
}

// dgeqpf on a (m x n, column-major, lda = m, overwritten) for kmax steps.
// jpvt[n]: on exit the original column ids in pivoted order. Returns the
// number of recomputed norms, or -1 when a forced column was taken already.
long long port_dgeqpf(double* a, long long m, long long n, int kmax, const int* forced,
                      int* jpvt, int* free_choice, double* max_norm, double* taken_norm) {
  const double tol3z = std::sqrt(std::ldexp(1.0, -53));
  std::vector<double> vn1(n), vn2(n);
  std::vector<long long> where(n);  // original id -> current position
  for (long long j = 0; j < n; ++j) {
    jpvt[j] = (int)j;
    where[j] = j;
  }
#pragma omp parallel for schedule(static)
  for (long long j = 0; j < n; ++j) {
    vn1[j] = nrm2(a + j * m, m);
    vn2[j] = vn1[j];
  }
  long long recomputes = 0;
  const long long steps = kmax < (m < n ? m : n) ? kmax : (m < n ? m : n);
  for (long long i = 0; i < steps; ++i) {
    long long pvt = i;
    for (long long j = i + 1; j < n; ++j)
      if (vn1[j] > vn1[pvt]) pvt = j;  // idamax: the first maximum
    if (free_choice) free_choice[i] = jpvt[pvt];
    if (max_norm) max_norm[i] = vn1[pvt];
    if (forced && forced[i] >= 0) {
      if (forced[i] >= n || where[forced[i]] < i) return -1;  // not a remaining column
      pvt = where[forced[i]];
    }
    if (taken_norm) taken_norm[i] = vn1[pvt];
    if (pvt != i) {
      double* x = a + pvt * m;
      double* y = a + i * m;
      for (long long r = 0; r < m; ++r) {
        const double t = x[r];
        x[r] = y[r];
        y[r] = t;
      }
      const int t = jpvt[pvt];
      jpvt[pvt] = jpvt[i];
      jpvt[i] = t;
      where[jpvt[pvt]] = pvt;
      where[jpvt[i]] = i;
      vn1[pvt] = vn1[i];
      vn2[pvt] = vn2[i];
    }
    // dlarfg on a[i:m, i]
    double* v = a + i * m + i;
    const long long len = m - i;
    double tau = 0.0;
    const double alpha = v[0];
    const double xnorm = len > 1 ? nrm2(v + 1, len - 1) : 0.0;
    if (xnorm != 0.0) {
      const double beta = -std::copysign(lapy2(alpha, xnorm), alpha);
      tau = (beta - alpha) / beta;
      const double sc = 1.0 / (alpha - beta);
      for (long long r = 1; r < len; ++r) v[r] *= sc;
      v[0] = beta;
    }
    // apply H(i) = I - tau v v^T (v[0] = 1) to the later columns, then
    // update their norms
    const double aii = v[0];
    v[0] = 1.0;
    long long rec = 0;
#pragma omp parallel for schedule(static) reduction(+ : rec)
    for (long long j = i + 1; j < n; ++j) {
      double* c = a + j * m + i;
      if (tau != 0.0) {
        double w = 0.0;
        for (long long r = 0; r < len; ++r) w += v[r] * c[r];
        w *= tau;
        for (long long r = 0; r < len; ++r) c[r] -= w * v[r];
      }
      if (vn1[j] != 0.0) {
        double temp = std::fabs(c[0]) / vn1[j];
        temp = 1.0 - temp * temp;
        temp = temp > 0.0 ? temp : 0.0;
        const double q = vn1[j] / vn2[j];
        const double temp2 = temp * q * q;
        if (temp2 <= tol3z) {
          if (len > 1) {
            vn1[j] = nrm2(c + 1, len - 1);
            vn2[j] = vn1[j];
          } else {
            vn1[j] = 0.0;
            vn2[j] = 0.0;
          }
          ++rec;
        } else {
          vn1[j] *= std::sqrt(temp);
        }
      }
    }
    v[0] = aii;
    recomputes += rec;
  }
  return recomputes;
}

}  // extern "C"
