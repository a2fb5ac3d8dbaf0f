// FP64 ISDF fit on sm_100a: theta = (Z C^T) (C C^T + eps I)^{-1}.
//
// Reference: src/cuda/isdf-gpu.cpp:112-402 (cuBLAS DGEMM, elementwise
// product kernel, row gather, host +eps, cuSOLVER DPOTRF, two cuBLAS DTRSM)
// and its CPU twin src/cpu/getbasis_MPI.cpp:9-250. Same algorithm, same
// operation order at the level that matters for the result:
//   1. gather psi(mu): B(k, j) = psi(piv_j, k)                (isdf-gpu.cpp:155-213)
//   2. Z C^T = P1 o P2, P = psi_S psi_S(mu)^T, the product fused in the
//      GEMM epilogue                                            (:220-274)
//   3. C C^T(mu, nu) = Z C^T(piv_nu, mu)                         (:281-340)
//   4. eps = 1e-10 * (trace / rk) added to the diagonal         (:346-349)
//   5. lower Cholesky L                                          (:365)
//   6. theta L^T = Z C^T, then theta L = (that), in place        (:372-382)
// Kernels: FP64 tensor-core GEMM tiles (dgemm.cuh: mma.sync m16n8k8 f64),
// the 3-stage cp.async Core for the Z GEMM and the Cholesky panel and
// trailing updates, the warp-specialised bulk-copy WsTile for the
// triangular-solve steps (Core when theta's columns are not 16-byte
// aligned); a single-CTA 64 x 64 diagonal-block factor + inverse.
//
// Triangular solve. For a 64-column block K = [c0, c0+bs) with diagonal block
// L_KK and D = L_KK^{-1}, the forward step of theta L^T = Z is
//   X_K = (Z_K - X_{<K} L_{K,<K}^T) D^T = [X_{<K} | Z_K] . [-L_{K,<K}^T D^T ; D^T]
// and the backward step of theta L = X is
//   T_K = (X_K - T_{>K} L_{>K,K}) D   = [X_K | T_{>K}] . [D ; -L_{>K,K} D].
// Both are one GEMM over a contiguous column range of theta (whose columns
// hold the solved and the pending parts side by side) with a small operand
// W_K built just before the step; each CTA owns a row tile of theta and writes
// block K in place after it has read everything it needs. Only the 64 x 64
// diagonal blocks are inverted explicitly; every other block takes part by
// substitution, as in a blocked dtrsm.
// theta is column-major Ng x rk (ld = Ng), overwritten in place.
#include <mutex>
#include <vector>

#include "arena.h"
#include "common.cuh"
#include "solve.h"
#include "dgemm.cuh"
#include "fit.h"
#include "ozaki.cuh"
#include "readback.h"

namespace isdf_b200 {

namespace {

constexpr int kNB = 64;  // Cholesky / triangular-solve block size

using CoreZ = dmma::Core<128, 128>;  // Z GEMM, Cholesky trailing update
using CoreN = dmma::Core<128, 64>;   // panel and triangular-solve steps
using WsN = dmma::WsTile<64, 64, 2, 2, 16, 4>;  // triangular-solve steps, 3 CTAs per SM

// 16-byte cp.async needs 16-byte aligned rows: base aligned, even leading dimension.
__host__ __device__ inline bool vec2_ok(const void* a, long long lda, const void* b,
                                        long long ldb) {
  return ((reinterpret_cast<size_t>(a) | reinterpret_cast<size_t>(b)) & 15) == 0 &&
         (lda % 2) == 0 && (ldb % 2) == 0;
}

// ----------------------------------------------------------- Z C^T GEMM
// mode 0: C = acc*acc (S1 = S2); mode 1: C = acc (first factor);
// mode 2: C = C * acc (second factor, S1 != S2).
template <int MODE, int VEC>
__global__ void __launch_bounds__(256) k_gemm_z(int M, int N, int K, const double* __restrict__ A,
                                                long long lda, const double* __restrict__ B,
                                                long long ldb, double* __restrict__ C,
                                                long long ldc) {
  extern __shared__ double smem[];
  const int n0 = blockIdx.x * CoreZ::BN;
  const long long m0 = (long long)blockIdx.y * CoreZ::BM;
  CoreZ core;
  core.zero();
  const int m_rem = (int)(M - m0 < CoreZ::BM ? M - m0 : CoreZ::BM);
  core.run<VEC>(smem, A + m0, lda, B + n0, ldb, m_rem, N - n0, 0, K);
  core.for_each([&](int r, int c, double v) {
    if (r < m_rem && n0 + c < N) {
      double* p = C + (m0 + r) + (long long)(n0 + c) * ldc;
      if (MODE == 0) *p = v * v;
      else if (MODE == 1) *p = v;
      else *p = *p * v;
    }
  });
}

// The same product on the warp-specialised tile (16-byte aligned operands,
// even sizes and leading dimensions).
template <int MODE>
__global__ void __launch_bounds__(WsN::THREADS, 3)
    k_gemm_zws(int M, int N, int K, const double* __restrict__ A, long long lda,
               const double* __restrict__ B, long long ldb, double* __restrict__ C, long long ldc,
               int* err) {
  extern __shared__ __align__(128) double smem[];
  // one-dimensional grid, column tiles fastest: the CTAs in flight share their A rows in L2
  const int ncol = (N + WsN::BN - 1) / WsN::BN;
  const int n0 = (int)(blockIdx.x % ncol) * WsN::BN;
  const long long m0 = (long long)(blockIdx.x / ncol) * WsN::BM;
  const int m_rem = (int)(M - m0 < WsN::BM ? M - m0 : WsN::BM);
  const int n_rem = N - n0 < WsN::BN ? N - n0 : WsN::BN;
  WsN tile;
  if (!tile.run(smem, A + m0, lda, m_rem, B + n0, ldb, n_rem, K, err)) return;
  if (WsN::producer()) return;
  tile.for_each([&](int r, int c, double v) {
    if (r < m_rem && c < n_rem) {
      double* p = C + (m0 + r) + (long long)(n0 + c) * ldc;
      if (MODE == 0) *p = v * v;
      else if (MODE == 1) *p = v;
      else *p = *p * v;
    }
  });
}

// ----------------------------------------------------------- gathers
// Bm[k*rk + j] = psi[piv_j + (k0 + k)*ng]  (depth-major B operand)
__global__ void k_gather_psimu(const double* __restrict__ psi, long long ng, int nstate,
                               const int* __restrict__ piv, int rk, double* __restrict__ Bm) {
  const long long total = (long long)nstate * rk;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int k = (int)(e / rk), j = (int)(e % rk);
    Bm[e] = psi[(long long)piv[j] + (long long)k * ng];
  }
}

// P(mu, nu) = Z(piv_nu, mu), column-major rk x rk.
__global__ void k_gather_cct(const double* __restrict__ Z, long long ng,
                             const int* __restrict__ piv, int rk, double* __restrict__ P) {
  const long long total = (long long)rk * rk;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int mu = (int)(e % rk), nu = (int)(e / rk);
    P[e] = Z[(long long)piv[nu] + (long long)mu * ng];
  }
}

// trace in index order, eps = 1e-10 * (trace / rk), diagonal += eps
__global__ void k_regularise(double* P, int rk, double* eps_out) {
  __shared__ double eps;
  if (threadIdx.x == 0) {
    double tr = 0.0;
    for (int i = 0; i < rk; ++i) tr = radd(tr, P[(long long)i * rk + i]);
    eps = rmul(1e-10, rdiv(tr, (double)rk));
    *eps_out = eps;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < rk; i += blockDim.x) {
    double* d = P + (long long)i * rk + i;
    *d = radd(*d, eps);
  }
}

// ----------------------------------------------------------- Cholesky
// Factors the diagonal block A[k0:k0+bs, k0:k0+bs] (lower, in place) and
// writes its inverse X = L_kk^{-1} twice, padded to 64 x 64 with zeros:
//   dinvT[k*64 + n] = X(n, k)   (right factor of a forward step)
//   dinv [k*64 + n] = X(k, n)   (right factor of a backward step)
// info: first failing global column + 1 (kept if already set).
__global__ void __launch_bounds__(256) k_potf2(double* A, int lda, int k0, int bs,
                                               double* __restrict__ dinvT,
                                               double* __restrict__ dinv, int* info) {
  extern __shared__ double potf2_smem[];
  double(*a)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(potf2_smem);  // a[row][col]
  double(*x)[kNB + 1] = reinterpret_cast<double(*)[kNB + 1]>(potf2_smem + kNB * (kNB + 1));
  const int tid = threadIdx.x;
  for (int e = tid; e < kNB * kNB; e += 256) {
    int r = e % kNB, c = e / kNB;
    a[r][c] = (r < bs && c < bs && r >= c) ? A[(long long)(k0 + r) + (long long)(k0 + c) * lda]
                                           : 0.0;
    x[r][c] = 0.0;
  }
  __syncthreads();
  // right-looking: the trailing update on a 16 x 16 thread grid (thread
  // (ty, tx) takes rows ty, ty + 16, ... and columns tx, tx + 16, ...)
  const int ty = tid >> 4, tx = tid & 15;
  for (int j = 0; j < bs; ++j) {
    if (tid == 0) {
      double d = a[j][j];
      if (!(d > 0.0)) atomicCAS(info, 0, k0 + j + 1);
      a[j][j] = sqrt(d);
    }
    __syncthreads();
    const double djj = a[j][j];
    for (int i = j + 1 + tid; i < bs; i += 256) a[i][j] = a[i][j] / djj;
    __syncthreads();
    for (int i = j + 1 + ty; i < bs; i += 16) {
      const double lij = a[i][j];
      for (int c = j + 1 + tx; c <= i; c += 16) a[i][c] -= lij * a[c][j];
    }
    __syncthreads();
  }
  // X = L^{-1} row by row, x(i, c) = -(sum_{c <= k < i} L(i, k) x(k, c)) / L(i, i):
  // four threads per column, each summing every fourth k
  {
    const int c = tid >> 2, part = tid & 3;
    for (int i = 0; i < bs; ++i) {
      double sum = 0.0;
      if (c < i)
        for (int k = c + part; k < i; k += 4) sum = fma(a[i][k], x[k][c], sum);
      sum += __shfl_xor_sync(0xffffffffu, sum, 1);
      sum += __shfl_xor_sync(0xffffffffu, sum, 2);
      if (part == 0 && c <= i) x[i][c] = c == i ? 1.0 / a[i][i] : -sum / a[i][i];
      __syncthreads();
    }
  }
  for (int e = tid; e < kNB * kNB; e += 256) {
    int r = e % kNB, c = e / kNB;
    if (r < bs && c < bs) A[(long long)(k0 + r) + (long long)(k0 + c) * lda] = r >= c ? a[r][c] : 0.0;
    int k = e / kNB, n = e % kNB;
    dinvT[e] = x[n][k];
    dinv[e] = x[k][n];
  }
}

// Panel: L[k0+bs:, k0:k0+bs] = A[k0+bs:, k0:k0+bs] * X^T, in place (a CTA
// reads its whole row tile before it writes it back).
template <int VEC>
__global__ void __launch_bounds__(256) k_chol_panel(double* A, int lda, int k0, int bs, int n,
                                                    const double* __restrict__ dinvT) {
  extern __shared__ double smem[];
  const int m0 = k0 + bs + blockIdx.x * CoreN::BM;
  CoreN core;
  core.zero();
  core.run<VEC>(smem, A + m0 + (long long)k0 * lda, lda, dinvT, kNB, n - m0, bs, 0, bs);
  core.for_each([&](int r, int c, double v) {
    if (m0 + r < n && c < bs) A[(m0 + r) + (long long)(k0 + c) * lda] = v;
  });
}

// Trailing update of the lower part: A[r, c] -= sum_k L[r, k] L[c, k] for
// r, c >= k0+bs, k in the panel. Tiles wholly above the diagonal are skipped.
template <int VEC>
__global__ void __launch_bounds__(256) k_chol_update(double* A, int lda, int k0, int bs, int n) {
  extern __shared__ double smem[];
  const int base = k0 + bs;
  const int n0 = base + blockIdx.x * CoreZ::BN;
  const int m0 = base + blockIdx.y * CoreZ::BM;
  if (m0 + CoreZ::BM <= n0) return;
  CoreZ core;
  core.zero();
  // B(k, c) = L[n0 + c, k0 + k]
  core.run<VEC>(smem, A + m0 + (long long)k0 * lda, lda, A + n0 + (long long)k0 * lda, lda,
                n - m0, n - n0, 0, bs);
  core.for_each([&](int r, int c, double v) {
    const int gr = m0 + r, gc = n0 + c;
    if (gr < n && gc < n && gr >= gc) A[gr + (long long)gc * lda] -= v;
  });
}

// Clears the strict upper triangle left over in the factor's storage.
__global__ void k_clear_upper(double* L, int n) {
  const long long total = (long long)n * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e % n), c = (int)(e / n);
    if (r < c) L[e] = 0.0;
  }
}

// ----------------------------------------------------------- triangular solve
// W_K (depth-major, 64 columns, W[k*64 + n]) for column block [c0, c0+bs):
//  forward  (rows k < c0+bs): k < c0: -sum_j L(c0+j, k) D^T(j, n);  else D^T(k-c0, n)
//  backward (rows k >= c0):   k >= c0+bs: -sum_j L(k, c0+j) D(j, n); else D(k-c0, n)
// with dT[j*64 + n] = D(n, j) and d[j*64 + n] = D(j, n), D = L_KK^{-1} (zero-padded).
template <bool FORWARD>
__global__ void __launch_bounds__(256) k_build_w(const double* __restrict__ L, int rk, int c0,
                                                 int bs, const double* __restrict__ dmat,
                                                 double* __restrict__ W) {
  __shared__ double ds[kNB * kNB];
  for (int e = threadIdx.x; e < kNB * kNB; e += 256) ds[e] = dmat[e];
  __syncthreads();
  const int n = threadIdx.x & 63;
  const int klo = FORWARD ? 0 : c0, khi = FORWARD ? c0 + bs : rk;
  for (int k = klo + blockIdx.x * 4 + (threadIdx.x >> 6); k < khi; k += gridDim.x * 4) {
    double v;
    if (FORWARD ? (k < c0) : (k >= c0 + bs)) {
      double s = 0.0;
      for (int j = 0; j < bs; ++j) {
        const double l = FORWARD ? L[(c0 + j) + (long long)k * rk] : L[k + (long long)(c0 + j) * rk];
        s = fma(l, ds[j * kNB + n], s);
      }
      v = -s;
    } else {
      v = ds[(k - c0) * kNB + n];
    }
    W[(long long)k * kNB + n] = v;
  }
}

// theta[rows, c0:c0+bs] = theta[rows, kb:ke] * W[kb:ke, 0:bs], in place per row tile.
template <int VEC>
__global__ void __launch_bounds__(256) k_trsm_gemm(double* theta, long long ng, int c0, int bs,
                                                   int kb, int ke, const double* __restrict__ W) {
  extern __shared__ double smem[];
  const long long m0 = (long long)blockIdx.x * CoreN::BM;
  const int m_rem = (int)(ng - m0 < CoreN::BM ? ng - m0 : CoreN::BM);
  CoreN core;
  core.zero();
  core.run<VEC>(smem, theta + m0, ng, W, kNB, m_rem, bs, kb, ke);
  core.for_each([&](int r, int c, double v) {
    if (r < m_rem && c < bs) theta[(m0 + r) + (long long)(c0 + c) * ng] = v;
  });
}

// The same step on the warp-specialised tile (theta 16-byte aligned, Ng even).
__global__ void __launch_bounds__(WsN::THREADS, 3)
    k_trsm_ws(double* theta, long long ng, int c0, int bs, int kb, int ke,
              const double* __restrict__ W, int* err) {
  extern __shared__ __align__(128) double smem[];
  const long long m0 = (long long)blockIdx.x * WsN::BM;
  const int m_rem = (int)(ng - m0 < WsN::BM ? ng - m0 : WsN::BM);
  WsN tile;
  if (!tile.run(smem, theta + m0 + (long long)kb * ng, ng, m_rem, W + (long long)kb * kNB, kNB,
                kNB, ke - kb, err))
    return;
  if (WsN::producer()) return;
  tile.for_each([&](int r, int c, double v) {
    if (r < m_rem && c < bs) theta[(m0 + r) + (long long)(c0 + c) * ng] = v;
  });
}

// ---- L^{-1} by blocked doubling (the mixed form's triangular factors).
// X = L^{-1} is kept twice: Xr row-major (X(i, j) = Xr[i*n + j], which is
// L^{-T} column-major) and Xc column-major. Level s joins the inverted
// diagonal blocks A = [a0, a0+s) and D = [a0+s, a0+2s) pairwise:
//   X(D, A) = -X(D, D) (L(D, A) X(A, A)),
// two FP64 tensor-core GEMMs per pair (K ranges cut to the triangles), all
// pairs of a level in one launch; the 64 x 64 diagonal-block inverses of the
// Cholesky factorisation are level 0.
__global__ void k_trinv_init(const double* __restrict__ dinv, int n, double* __restrict__ Xr,
                             double* __restrict__ Xc) {
  const int c0 = blockIdx.x * kNB, bs = min(kNB, n - c0);
  const double* d = dinv + (size_t)blockIdx.x * kNB * kNB;
  for (int e = threadIdx.x; e < kNB * kNB; e += blockDim.x) {
    const int k = e / kNB, j = e % kNB;
    if (k < bs && j < bs) {
      const double v = d[e];  // X(c0 + k, c0 + j)
      Xr[(long long)(c0 + k) * n + (c0 + j)] = v;
      Xc[(c0 + k) + (long long)(c0 + j) * n] = v;
    }
  }
}

// T(r, c) = sum_{k >= c} L(d0 + r, a0 + k) X(a0 + k, a0 + c), into Tb at X(D, A)'s place.
template <int VEC>
__global__ void __launch_bounds__(256) k_trinv_t(const double* __restrict__ L,
                                                 const double* __restrict__ Xr,
                                                 double* __restrict__ Tb, int n, int s) {
  extern __shared__ double smem[];
  const int a0 = blockIdx.z * 2 * s, d0 = a0 + s;
  if (d0 >= n) return;
  const int a = s, d = min(s, n - d0);
  const int c0 = blockIdx.x * CoreN::BN, r0 = blockIdx.y * CoreN::BM;
  if (c0 >= a || r0 >= d) return;
  CoreN core;
  core.zero();
  core.run<VEC>(smem, L + (d0 + r0) + (long long)a0 * n, n, Xr + (long long)a0 * n + (a0 + c0), n,
                d - r0, a - c0, c0, a);
  core.for_each([&](int r, int c, double v) {
    if (r0 + r < d && c0 + c < a) Tb[(long long)(d0 + r0 + r) * n + (a0 + c0 + c)] = v;
  });
}

// X(d0 + r, a0 + c) = -sum_{k <= r} X(d0 + r, d0 + k) T(k, c).
template <int VEC>
__global__ void __launch_bounds__(256) k_trinv_x(const double* __restrict__ Tb,
                                                 double* __restrict__ Xr, double* Xc, int n,
                                                 int s) {
  extern __shared__ double smem[];
  const int a0 = blockIdx.z * 2 * s, d0 = a0 + s;
  if (d0 >= n) return;
  const int a = s, d = min(s, n - d0);
  const int c0 = blockIdx.x * CoreN::BN, r0 = blockIdx.y * CoreN::BM;
  if (c0 >= a || r0 >= d) return;
  CoreN core;
  core.zero();
  core.run<VEC>(smem, Xc + (d0 + r0) + (long long)d0 * n, n, Tb + (long long)d0 * n + (a0 + c0), n,
                d - r0, a - c0, 0, min(d, r0 + CoreN::BM));
  core.for_each([&](int r, int c, double v) {
    if (r0 + r < d && c0 + c < a) {
      Xr[(long long)(d0 + r0 + r) * n + (a0 + c0 + c)] = -v;
      Xc[(d0 + r0 + r) + (long long)(a0 + c0 + c) * n] = -v;
    }
  });
}

constexpr size_t smem_bytes_potf2 = sizeof(double) * 2 * kNB * (kNB + 1);

template <class K>
int set_attr(K kernel, size_t bytes) {
  ISDF_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  return ISDF_OK;
}

int set_smem_attrs() {
  std::lock_guard<std::mutex> attr_lock(attr_mutex());
  static bool done_dev[64] = {};
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done_dev[dev]) return ISDF_OK;
  ISDF_TRY(set_attr(k_potf2, smem_bytes_potf2));
  ISDF_TRY(set_attr(k_gemm_z<0, 1>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_z<1, 1>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_z<2, 1>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_z<1, 2>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_chol_update<1>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_chol_update<2>, CoreZ::SMEM_BYTES));
  ISDF_TRY(set_attr(k_chol_panel<1>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_chol_panel<2>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trsm_gemm<1>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trsm_ws, WsN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_zws<0>, WsN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_zws<1>, WsN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_gemm_zws<2>, WsN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trinv_t<1>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trinv_t<2>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trinv_x<1>, CoreN::SMEM_BYTES));
  ISDF_TRY(set_attr(k_trinv_x<2>, CoreN::SMEM_BYTES));
  if (dev >= 0 && dev < 64) done_dev[dev] = true;
  return ISDF_OK;
}

struct FitBuffers {
  int* piv;
  double* Bm;
  double* P;  // C C^T, then L (column-major rk x rk)
  double* W;  // one triangular-solve block operand, rk x 64
  double* dinvT;
  double* dinv;
  double* eps;
  int* info;  // [0]: Cholesky (first failing column + 1), [1]: pipeline timeout
  int* err;
};

FitBuffers carve(Arena& a, int nstate, int rk) {
  FitBuffers b;
  const int nblk = (rk + kNB - 1) / kNB;
  b.piv = a.take<int>(rk);
  b.Bm = a.take<double>((size_t)nstate * rk);
  b.P = a.take<double>((size_t)rk * rk);
  b.W = a.take<double>((size_t)rk * kNB);
  b.dinvT = a.take<double>((size_t)nblk * kNB * kNB);
  b.dinv = a.take<double>((size_t)nblk * kNB * kNB);
  b.eps = a.take<double>(1);
  b.info = a.take<int>(2);
  b.err = b.info ? b.info + 1 : nullptr;
  return b;
}

}  // namespace

int dgemm_store(int M, int N, int K, const double* A, long long lda, const double* B,
                long long ldb, double* C, long long ldc, cudaStream_t s) {
  ISDF_TRY(set_smem_attrs());
  dim3 g((unsigned)((N + CoreZ::BN - 1) / CoreZ::BN), (unsigned)((M + CoreZ::BM - 1) / CoreZ::BM));
  if (vec2_ok(A, lda, B, ldb))
    k_gemm_z<1, 2><<<g, 256, CoreZ::SMEM_BYTES, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
  else
    k_gemm_z<1, 1><<<g, 256, CoreZ::SMEM_BYTES, s>>>(M, N, K, A, lda, B, ldb, C, ldc);
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

size_t fit_workspace_bytes(long long ng, int nstate, int rk) {
  (void)ng;
  Arena a;
  a.counting = true;
  carve(a, nstate, rk);
  return a.off;
}

// Lower Cholesky of P (rk x rk, column-major) in place, with per-block
// inverses for the solve. Returns the failing column + 1 in *info (0 = ok).
static int cholesky(const FitBuffers& b, int rk, cudaStream_t s) {
  const int nblk = (rk + kNB - 1) / kNB;
  const bool v2 = (rk % 2) == 0;
  for (int kb = 0; kb < nblk; ++kb) {
    const int k0 = kb * kNB;
    const int bs = min(kNB, rk - k0);
    k_potf2<<<1, 256, smem_bytes_potf2, s>>>(b.P, rk, k0, bs, b.dinvT + (size_t)kb * kNB * kNB,
                                             b.dinv + (size_t)kb * kNB * kNB, b.info);
    const int rem = rk - k0 - bs;
    if (rem > 0) {
      const double* dT = b.dinvT + (size_t)kb * kNB * kNB;
      const unsigned pg = (unsigned)((rem + CoreN::BM - 1) / CoreN::BM);
      dim3 g((rem + CoreZ::BN - 1) / CoreZ::BN, (rem + CoreZ::BM - 1) / CoreZ::BM);
      if (v2) {
        k_chol_panel<2><<<pg, 256, CoreN::SMEM_BYTES, s>>>(b.P, rk, k0, bs, rk, dT);
        k_chol_update<2><<<g, 256, CoreZ::SMEM_BYTES, s>>>(b.P, rk, k0, bs, rk);
      } else {
        k_chol_panel<1><<<pg, 256, CoreN::SMEM_BYTES, s>>>(b.P, rk, k0, bs, rk, dT);
        k_chol_update<1><<<g, 256, CoreZ::SMEM_BYTES, s>>>(b.P, rk, k0, bs, rk);
      }
    }
  }
  k_clear_upper<<<grid_for((long long)rk * rk, 256), 256, 0, s>>>(b.P, rk);
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

// Stage timers: CUDA events on the solve stream.
struct StageEvents {
  cudaEvent_t e[8] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  ~StageEvents() {
    for (auto& x : e)
      if (x) cudaEventDestroy(x);
  }
  int create() {
    for (auto& x : e) ISDF_CUDA(cudaEventCreate(&x));
    return ISDF_OK;
  }
};

int fit_fp64(const FitArgs& args, Arena& arena, cudaStream_t s, FitResult* res, bool timed) {
  const long long ng = args.ng;
  const int rk = args.rk;
  if (ng <= 0 || rk <= 0 || args.nstate <= 0) return record_error(ISDF_ERR_ARG, "fit: bad sizes");
  ISDF_TRY(set_smem_attrs());
  FitBuffers b = carve(arena, args.nstate, rk);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "fit: workspace too small");
  StageEvents ev;
  if (timed) ISDF_TRY(ev.create());
  auto mark = [&](int i) { return timed ? cudaEventRecord(ev.e[i], s) : cudaSuccess; };
  const int nblk_ = (rk + kNB - 1) / kNB;
  const bool same_ = (args.nv1 == args.nv2 && args.nc1 == args.nc2);
  res->launches = 1 + (same_ ? 1 : 2) + 2 + (nblk_ + 2 * (nblk_ - 1) + 1) + 4 * nblk_ +
                  (readback_mailbox() ? 2 : 0);

  ISDF_CUDA(cudaMemsetAsync(b.info, 0, 2 * sizeof(int), s));
  if (args.d_psimu) {
    b.Bm = const_cast<double*>(args.d_psimu);
  } else {
    ISDF_CUDA(cudaMemcpyAsync(b.piv, args.piv, sizeof(int) * rk, cudaMemcpyHostToDevice, s));
    k_gather_psimu<<<grid_for((long long)args.nstate * rk, 256), 256, 0, s>>>(
        args.d_psi, ng, args.nstate, b.piv, rk, b.Bm);
  }

  // Z C^T into theta
  const int lo1 = args.nocc - args.nv1, K1 = args.nv1 + args.nc1;
  const int lo2 = args.nocc - args.nv2, K2 = args.nv2 + args.nc2;
  const bool same = (args.nv1 == args.nv2 && args.nc1 == args.nc2);
  dim3 zg((unsigned)((rk + CoreZ::BN - 1) / CoreZ::BN), (unsigned)((ng + CoreZ::BM - 1) / CoreZ::BM));
  ISDF_CUDA(mark(0));
  const double* A1 = args.d_psi + (long long)lo1 * ng;
  const double* A2 = args.d_psi + (long long)lo2 * ng;
  const double* B1 = b.Bm + (size_t)lo1 * rk;
  const double* B2 = b.Bm + (size_t)lo2 * rk;
  const bool zv2 = vec2_ok(A1, ng, B1, rk) && vec2_ok(A2, ng, B2, rk);
  const size_t zs = CoreZ::SMEM_BYTES;
  // warp-specialised tile: 16-byte aligned operands, Ng and rk even (vec2_ok)
  const unsigned zw = (unsigned)(((rk + WsN::BN - 1) / WsN::BN) * ((ng + WsN::BM - 1) / WsN::BM));
  const int wt = WsN::THREADS;
  const size_t ws = WsN::SMEM_BYTES;
  double* th = args.d_theta;
  if (same) {
    if (zv2) k_gemm_zws<0><<<zw, wt, ws, s>>>((int)ng, rk, K1, A1, ng, B1, rk, th, ng, b.err);
    else k_gemm_z<0, 1><<<zg, 256, zs, s>>>((int)ng, rk, K1, A1, ng, B1, rk, args.d_theta, ng);
  } else if (zv2) {
    k_gemm_zws<1><<<zw, wt, ws, s>>>((int)ng, rk, K1, A1, ng, B1, rk, th, ng, b.err);
    k_gemm_zws<2><<<zw, wt, ws, s>>>((int)ng, rk, K2, A2, ng, B2, rk, th, ng, b.err);
  } else {
    k_gemm_z<1, 1><<<zg, 256, zs, s>>>((int)ng, rk, K1, A1, ng, B1, rk, args.d_theta, ng);
    k_gemm_z<2, 1><<<zg, 256, zs, s>>>((int)ng, rk, K2, A2, ng, B2, rk, args.d_theta, ng);
  }
  ISDF_CHECK_LAUNCH();

  // C C^T, regularisation, Cholesky
  ISDF_CUDA(mark(1));
  if (args.d_psimu) {
    // the Z C^T GEMM on the pivot rows (C C^T is symmetric element for element:
    // the product of rows j and nu sums the same terms in the same order)
    dim3 cg((unsigned)((rk + CoreZ::BN - 1) / CoreZ::BN), (unsigned)((rk + CoreZ::BM - 1) / CoreZ::BM));
    if (same) {
      k_gemm_z<0, 1><<<cg, 256, zs, s>>>(rk, rk, K1, B1, rk, B1, rk, b.P, rk);
    } else {
      k_gemm_z<1, 1><<<cg, 256, zs, s>>>(rk, rk, K1, B1, rk, B1, rk, b.P, rk);
      k_gemm_z<2, 1><<<cg, 256, zs, s>>>(rk, rk, K2, B2, rk, B2, rk, b.P, rk);
    }
  } else {
    k_gather_cct<<<grid_for((long long)rk * rk, 256), 256, 0, s>>>(args.d_theta, ng, b.piv, rk,
                                                                  b.P);
  }
  k_regularise<<<1, 256, 0, s>>>(b.P, rk, b.eps);
  ISDF_TRY(cholesky(b, rk, s));
  ISDF_CUDA(mark(2));
  int info = 0;
  ISDF_TRY(read_back(&info, b.info, sizeof(int), s));
  res->chol_info = info;
  if (info != 0) return record_error(ISDF_ERR_NOT_SPD, "fit: C C^T + eps I is not positive definite");

  // theta L^T = Z C^T (forward over column blocks), then theta L = Y (backward)
  const int nblk = (rk + kNB - 1) / kNB;
  const unsigned tg = (unsigned)((ng + CoreN::BM - 1) / CoreN::BM);
  const unsigned wg = (unsigned)((ng + WsN::BM - 1) / WsN::BM);
  const bool tv2 = vec2_ok(args.d_theta, ng, b.W, kNB);
  auto step = [&](int c0, int bs, int kb, int ke) {
    if (tv2)  // 16-byte aligned columns: bulk copies
      k_trsm_ws<<<wg, WsN::THREADS, WsN::SMEM_BYTES, s>>>(args.d_theta, ng, c0, bs, kb, ke, b.W,
                                                           b.err);
    else
      k_trsm_gemm<1><<<tg, 256, CoreN::SMEM_BYTES, s>>>(args.d_theta, ng, c0, bs, kb, ke, b.W);
  };
  for (int kb = 0; kb < nblk; ++kb) {
    const int c0 = kb * kNB, bs = min(kNB, rk - c0);
    k_build_w<true><<<(c0 + bs + 3) / 4 < 1024 ? (c0 + bs + 3) / 4 : 1024, 256, 0, s>>>(
        b.P, rk, c0, bs, b.dinvT + (size_t)kb * kNB * kNB, b.W);
    step(c0, bs, 0, c0 + bs);
  }
  for (int kb = nblk - 1; kb >= 0; --kb) {
    const int c0 = kb * kNB, bs = min(kNB, rk - c0);
    k_build_w<false><<<(rk - c0 + 3) / 4 < 1024 ? (rk - c0 + 3) / 4 : 1024, 256, 0, s>>>(
        b.P, rk, c0, bs, b.dinv + (size_t)kb * kNB * kNB, b.W);
    step(c0, bs, c0, rk);
  }
  ISDF_CHECK_LAUNCH();
  ISDF_CUDA(mark(3));
  int err = 0;
  ISDF_TRY(read_back(&err, b.err, sizeof(int), s));
  if (err) return record_error(ISDF_ERR_TIMEOUT, "fit: a triangular-solve pipeline wait timed out");
  if (!timed) return ISDF_OK;
  ISDF_CUDA(cudaEventElapsedTime(&res->t_zct_ms, ev.e[0], ev.e[1]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_chol_ms, ev.e[1], ev.e[2]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_solve_ms, ev.e[2], ev.e[3]));
  return ISDF_OK;
}


// ===================================================================== mixed
// Mixed-precision form: the three large products (Z C^T, Y = Z L^{-T},
// theta = Y L^{-1}) as INT8-sliced GEMMs on the tcgen05 tensor cores
// (ozaki.cuh); C C^T, the Cholesky factorisation and L^{-T} stay FP64.
// theta = (Z C^T L^{-T}) L^{-1} with explicit triangular inverses, whose
// truncation (2^-47 of the operand scales at S = 6) stays below the
// conditioning of the fit.

namespace {

constexpr int kSliceTile = 64;  // rows per slicing tile

// Round to the nearest integer (ties to even) on the FP64 add pipe: adding
// 1.5 * 2^52 leaves the rounded value in the low word of the sum (two's
// complement, |x| < 2^31); subtracting it back gives rint(x) exactly.
constexpr double kRoundShift = 6755399441055744.0;
__device__ __forceinline__ double round_shift(double x) { return __dadd_rn(x, kRoundShift); }
constexpr int kSliceK = 32;     // K bytes per slicing tile

// Row-scaled slicing of an M x K FP64 operand, element (m, k) at
// X[m*rs + k*ks], into S int8 slices written in the pre-tiled layout of the
// Ozaki GEMM (ozaki::tiled_offset: blocks of R rows, 32-byte K blocks; the A
// side unstacked with R = 128, the B side stacked with R = 64), rows padded to
// mp and K to kp with zeros, and exponents e[m] (|x| 2^-e < 1/2).
__global__ void k_row_exponent(const double* __restrict__ X, long long rs, long long ks, int M,
                               int K, int* __restrict__ e) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x) {
    double mx = 0.0;
    for (int k = 0; k < K; ++k) mx = fmax(mx, fabs(X[m * rs + k * ks]));
    e[m] = mx > 0.0 ? ilogb(mx) + 2 : 0;
  }
}

// Row exponents from the binade maxima the GEMM epilogue gathered: the same
// e as k_row_exponent computes from the stored values.
__global__ void k_exp_from_max(int* __restrict__ e, int M) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < M; m += gridDim.x * blockDim.x)
    e[m] = e[m] == ozaki::kNoExponent ? 0 : e[m] + 2;
}

template <int S, int R, bool STACKED>
__global__ void __launch_bounds__(256) k_slice(const double* __restrict__ X, long long rs,
                                               long long ks, int M, int K, int mp, int kp,
                                               const int* __restrict__ e, int8_t* __restrict__ P) {
  __shared__ double xs[kSliceTile][kSliceK + 1];
  __shared__ __align__(16) int8_t qs[S][kSliceTile][kSliceK];
  const int m0 = blockIdx.y * kSliceTile, k0 = blockIdx.x * kSliceK;
  const bool mfast = rs == 1;
  for (int i = threadIdx.x; i < kSliceTile * kSliceK; i += 256) {
    const int mi = mfast ? i % kSliceTile : i / kSliceK;
    const int ki = mfast ? i / kSliceTile : i % kSliceK;
    const int m = m0 + mi, k = k0 + ki;
    xs[mi][ki] = (m < M && k < K) ? X[(long long)m * rs + (long long)k * ks] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kSliceTile * kSliceK; i += 256) {
    const int mi = i / kSliceK, ki = i % kSliceK;
    const int m = m0 + mi;
    double r = (m < M) ? ldexp(xs[mi][ki], -e[m]) : 0.0;
#pragma unroll
    for (int t = 0; t < S; ++t) {
      r *= ozaki::kBase;
      const double tq = round_shift(r);
      r -= tq - kRoundShift;
      qs[t][mi][ki] = (int8_t)__double2loint(tq);
    }
  }
  __syncthreads();
  // 16-byte stores: S planes x 64 rows x 2 chunks
  for (int i = threadIdx.x; i < S * kSliceTile * 2; i += 256) {
    const int t = i / (kSliceTile * 2), rem = i % (kSliceTile * 2);
    const int mi = rem / 2, c = rem % 2;
    const int m = m0 + mi;
    if (m < mp && k0 + c * 16 < kp)
      *reinterpret_cast<int4*>(P + ozaki::tiled_offset<S, R, STACKED>(m / R, k0 / ozaki::BKB,
                                                                     kp / ozaki::BKB, t, c,
                                                                     m % R)) =
          *reinterpret_cast<const int4*>(&qs[t][mi][c * 16]);
  }
}


inline int round_up(long long x, int a) { return (int)((x + a - 1) / a * a); }

struct MixedBuffers {
  int8_t *PA, *PB;  // pre-tiled slices of the A (grid rows) and B operands
  int *ea, *eb, *err;
  int *ez, *ey;     // row exponents of Z C^T and Y, gathered by the GEMM epilogues
  double* MT;  // L^{-T}, column-major rk x rk (= L^{-1} row-major)
  double *XC, *TB;  // L^{-1} column-major, and the doubling's scratch
};

MixedBuffers carve_mixed(Arena& a, long long ng, int nstate, int rk, int slices) {
  MixedBuffers b;
  const int kmax = round_up(nstate > rk ? nstate : rk, ozaki::BKB);
  const long long mp = round_up(ng, ozaki::BM);
  const int np = round_up(rk, 128);
  b.PA = a.take<int8_t>((size_t)slices * mp * kmax);
  b.PB = a.take<int8_t>((size_t)slices * np * kmax);
  b.ea = a.take<int>((size_t)mp);
  b.ez = a.take<int>((size_t)mp);
  b.ey = a.take<int>((size_t)mp);
  b.eb = a.take<int>((size_t)np);
  b.err = a.take<int>(1);
  b.MT = a.take<double>((size_t)rk * rk);
  b.XC = a.take<double>((size_t)rk * rk);
  b.TB = a.take<double>((size_t)rk * rk);
  return b;
}

// A side with contiguous rows (rs = 1): one thread per row and 16-column
// K chunk. The warp's loads are 256-byte rows of one column, and the
// thread's digits of one slice form one 16-byte store that lands next to its
// neighbours' in the tiled layout: no shared memory, one pass over X.
template <int S>
__global__ void __launch_bounds__(256) k_slice_rows(const double* __restrict__ X, long long ks,
                                                    int M, int K, int mp, int kp,
                                                    const int* __restrict__ e,
                                                    int8_t* __restrict__ P) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= mp) return;
  const int k0 = blockIdx.y * 16;
  double r[16];
  const double sc = m < M ? ldexp(1.0, -e[m]) : 0.0;
#pragma unroll
  for (int j = 0; j < 16; ++j)
    r[j] = (m < M && k0 + j < K) ? X[m + (long long)(k0 + j) * ks] * sc : 0.0;
  int8_t* dst = P + ozaki::tiled_offset<S, ozaki::BM, false>(m / ozaki::BM, k0 / ozaki::BKB,
                                                             kp / ozaki::BKB, 0,
                                                             (k0 % ozaki::BKB) / 16, m % ozaki::BM);
#pragma unroll
  for (int t = 0; t < S; ++t) {
    unsigned w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      unsigned v = 0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int j = q * 4 + b;
        r[j] *= ozaki::kBase;
        const double tq = round_shift(r[j]);
        r[j] -= tq - kRoundShift;
        v |= ((unsigned)__double2loint(tq) & 0xffu) << (8 * b);
      }
      w[q] = v;
    }
    // slice t of the same row and chunk sits BM * BKB bytes further on
    *reinterpret_cast<uint4*>(dst + (size_t)t * ozaki::BM * ozaki::BKB) =
        make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// A side: R = 128 row blocks; B side: the stacked 64-column blocks.
// gathered = true: e holds the binade maxima from the producing GEMM's
// epilogue, and the pass over X that k_row_exponent makes is saved.
template <int S, bool B_SIDE>
int slice_operand(const double* X, long long rs, long long ks, int M, int K, int mp, int kp,
                  int* e, int8_t* P, cudaStream_t s, bool gathered = false) {
  if (gathered) k_exp_from_max<<<grid_for(M, 256), 256, 0, s>>>(e, M);
  else k_row_exponent<<<grid_for(M, 256), 256, 0, s>>>(X, rs, ks, M, K, e);
  dim3 g((unsigned)(kp / kSliceK), (unsigned)((mp + kSliceTile - 1) / kSliceTile));
  if (B_SIDE) {
    k_slice<S, ozaki::BN, true><<<g, 256, 0, s>>>(X, rs, ks, M, K, mp, kp, e, P);
  } else if (rs == 1) {
    dim3 gr((unsigned)((mp + 255) / 256), (unsigned)(kp / 16));
    k_slice_rows<S><<<gr, 256, 0, s>>>(X, ks, M, K, mp, kp, e, P);
  } else {
    k_slice<S, ozaki::BM, false><<<g, 256, 0, s>>>(X, rs, ks, M, K, mp, kp, e, P);
  }
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

template <int S, int EPI, int KMODE>
int ozaki_gemm(const MixedBuffers& b, const int* ea, int M, int N, int kp, double* C,
               long long ldc, int* rowmax, cudaStream_t s) {
  auto kern = ozaki::k_ozaki_gemm<S, EPI, KMODE>;
  static bool attr[64] = {};
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> attr_lock(attr_mutex());
  if (dev >= 0 && dev < 64 && !attr[dev]) {
    ISDF_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   ozaki::Cfg<S>::SMEM));
    attr[dev] = true;
  }
  if (kp > ozaki::kMaxK)
    return record_error(ISDF_ERR_UNSUPPORTED, "mixed fit: K beyond the INT32-exact limit (16384)");
  const long long tiles =
      (long long)((N + ozaki::BN - 1) / ozaki::BN) * ((M + ozaki::BM - 1) / ozaki::BM);
  if (tiles > 0x7fffffffLL) return record_error(ISDF_ERR_UNSUPPORTED, "mixed fit: too many tiles");
  static int sms[64] = {};
  if (dev >= 0 && dev < 64 && !sms[dev])
    ISDF_CUDA(cudaDeviceGetAttribute(&sms[dev], cudaDevAttrMultiProcessorCount, dev));
  const int nsm = (dev >= 0 && dev < 64 && sms[dev] > 0) ? sms[dev] : kNumSMs;
  const unsigned grid = (unsigned)(tiles < nsm ? tiles : nsm);  // persistent: one CTA per SM
  if (rowmax) ISDF_CUDA(cudaMemsetAsync(rowmax, 0x80, sizeof(int) * (size_t)M, s));
  kern<<<grid, ozaki::kThreads, ozaki::Cfg<S>::SMEM, s>>>(b.PA, b.PB, ea, b.eb, M, N, kp, C, ldc,
                                                          rowmax, b.err);
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

template <int S>
int fit_mixed_s(const FitArgs& args, Arena& arena, cudaStream_t s, FitResult* res) {
  // Z C^T takes one digit fewer than the triangular products (never below 5):
  // its truncation is not amplified by the triangular inverses' dynamic range,
  // and at 5 digits the fitted densities move by 3 % of their error at 6
  // (2.5e-7 against 2.4e-7 at Si216, 1.5e-7 against 1.4e-7 at Si64), while 4
  // digits move them to 2.5e-5
  constexpr int SZ = S > 5 ? S - 1 : S;
  const long long ng = args.ng;
  const int rk = args.rk;
  FitBuffers b = carve(arena, args.nstate, rk);
  MixedBuffers mb = carve_mixed(arena, ng, args.nstate, rk, S);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "mixed fit: workspace too small");
  StageEvents ev;
  ISDF_TRY(ev.create());
  const int mp = round_up(ng, ozaki::BM);
  const int np = round_up(rk, 128);
  ISDF_CUDA(cudaMemsetAsync(b.info, 0, 2 * sizeof(int), s));
  ISDF_CUDA(cudaMemsetAsync(mb.err, 0, sizeof(int), s));
  if (args.d_psimu) {
    b.Bm = const_cast<double*>(args.d_psimu);
  } else {
    ISDF_CUDA(cudaMemcpyAsync(b.piv, args.piv, sizeof(int) * rk, cudaMemcpyHostToDevice, s));
    k_gather_psimu<<<grid_for((long long)args.nstate * rk, 256), 256, 0, s>>>(
        args.d_psi, ng, args.nstate, b.piv, rk, b.Bm);
  }
  ISDF_CUDA(cudaEventRecord(ev.e[0], s));

  // Z C^T = (psi_S1 psi_S1(mu)^T) o (psi_S2 psi_S2(mu)^T)
  const bool same = (args.nv1 == args.nv2 && args.nc1 == args.nc2);
  for (int f = 0; f < (same ? 1 : 2); ++f) {
    const int lo = f == 0 ? args.nocc - args.nv1 : args.nocc - args.nv2;
    const int K = f == 0 ? args.nv1 + args.nc1 : args.nv2 + args.nc2;
    const int kp = round_up(K, ozaki::BKB);
    ISDF_TRY((slice_operand<SZ, false>(args.d_psi + (long long)lo * ng, 1, ng, (int)ng, K, mp, kp,
                                      mb.ea, mb.PA, s)));
    ISDF_TRY((slice_operand<SZ, true>(b.Bm + (size_t)lo * rk, 1, rk, rk, K, np, kp, mb.eb, mb.PB,
                                     s)));
    if (same)
      ISDF_TRY((ozaki_gemm<SZ, 1, 0>(mb, mb.ea, (int)ng, rk, kp, args.d_theta, ng, mb.ez, s)));
    else if (f == 0)
      ISDF_TRY((ozaki_gemm<SZ, 0, 0>(mb, mb.ea, (int)ng, rk, kp, args.d_theta, ng, nullptr, s)));
    else
      ISDF_TRY((ozaki_gemm<SZ, 2, 0>(mb, mb.ea, (int)ng, rk, kp, args.d_theta, ng, mb.ez, s)));
  }
  ISDF_CUDA(cudaEventRecord(ev.e[1], s));

  // C C^T + eps I, Cholesky, L^{-T} (FP64). C C^T is formed here from psi(mu)
  // on the FP64 tensor cores rather than gathered from the sliced Z C^T: the
  // factorisation amplifies the error of C C^T by cond(C C^T) (~1e10), so it
  // must carry FP64 rounding, as in the reference.
  {
    const int lo1 = args.nocc - args.nv1, K1 = args.nv1 + args.nc1;
    const int lo2 = args.nocc - args.nv2, K2 = args.nv2 + args.nc2;
    const double* B1 = b.Bm + (size_t)lo1 * rk;
    const double* B2 = b.Bm + (size_t)lo2 * rk;
    dim3 cg((unsigned)((rk + CoreZ::BN - 1) / CoreZ::BN), (unsigned)((rk + CoreZ::BM - 1) / CoreZ::BM));
    const size_t zs = CoreZ::SMEM_BYTES;
    if (same) {
      k_gemm_z<0, 1><<<cg, 256, zs, s>>>(rk, rk, K1, B1, rk, B1, rk, b.P, rk);
    } else {
      k_gemm_z<1, 1><<<cg, 256, zs, s>>>(rk, rk, K1, B1, rk, B1, rk, b.P, rk);
      k_gemm_z<2, 1><<<cg, 256, zs, s>>>(rk, rk, K2, B2, rk, B2, rk, b.P, rk);
    }
  }
  k_regularise<<<1, 256, 0, s>>>(b.P, rk, b.eps);
  ISDF_TRY(cholesky(b, rk, s));
  int info = 0;
  ISDF_TRY(read_back(&info, b.info, sizeof(int), s));
  res->chol_info = info;
  if (info != 0) return record_error(ISDF_ERR_NOT_SPD, "fit: C C^T + eps I is not positive definite");
  // L^{-T} (= L^{-1} row-major) by blocked doubling from the diagonal-block inverses
  {
    const int nblk = (rk + kNB - 1) / kNB;
    ISDF_CUDA(cudaMemsetAsync(mb.MT, 0, sizeof(double) * (size_t)rk * rk, s));
    ISDF_CUDA(cudaMemsetAsync(mb.XC, 0, sizeof(double) * (size_t)rk * rk, s));
    k_trinv_init<<<nblk, 256, 0, s>>>(b.dinv, rk, mb.MT, mb.XC);
    const bool v2 = vec2_ok(mb.MT, rk, mb.TB, rk);
    for (int lv = kNB; lv < rk; lv *= 2) {
      dim3 g((unsigned)((lv + CoreN::BN - 1) / CoreN::BN), (unsigned)((lv + CoreN::BM - 1) / CoreN::BM),
             (unsigned)((rk + 2 * lv - 1) / (2 * lv)));
      if (v2) {
        k_trinv_t<2><<<g, 256, CoreN::SMEM_BYTES, s>>>(b.P, mb.MT, mb.TB, rk, lv);
        k_trinv_x<2><<<g, 256, CoreN::SMEM_BYTES, s>>>(mb.TB, mb.MT, mb.XC, rk, lv);
      } else {
        k_trinv_t<1><<<g, 256, CoreN::SMEM_BYTES, s>>>(b.P, mb.MT, mb.TB, rk, lv);
        k_trinv_x<1><<<g, 256, CoreN::SMEM_BYTES, s>>>(mb.TB, mb.MT, mb.XC, rk, lv);
      }
    }
    ISDF_CHECK_LAUNCH();
  }
  ISDF_CUDA(cudaEventRecord(ev.e[2], s));

  // Y = Z L^{-T} (L^{-T} upper), then theta = Y L^{-1} (L^{-1} lower), in place in theta
  const int kp = round_up(rk, ozaki::BKB);
  ISDF_TRY((slice_operand<S, false>(args.d_theta, 1, ng, (int)ng, rk, mp, kp, mb.ez, mb.PA, s,
                                    true)));
  ISDF_TRY((slice_operand<S, true>(mb.MT, rk, 1, rk, rk, np, kp, mb.eb, mb.PB, s)));
  ISDF_CUDA(cudaEventRecord(ev.e[4], s));
  ISDF_TRY((ozaki_gemm<S, 0, 1>(mb, mb.ez, (int)ng, rk, kp, args.d_theta, ng, mb.ey, s)));
  ISDF_CUDA(cudaEventRecord(ev.e[5], s));
  ISDF_TRY((slice_operand<S, false>(args.d_theta, 1, ng, (int)ng, rk, mp, kp, mb.ey, mb.PA, s,
                                    true)));
  ISDF_TRY((slice_operand<S, true>(mb.MT, 1, rk, rk, rk, np, kp, mb.eb, mb.PB, s)));
  ISDF_CUDA(cudaEventRecord(ev.e[6], s));
  ISDF_TRY((ozaki_gemm<S, 0, 2>(mb, mb.ey, (int)ng, rk, kp, args.d_theta, ng, nullptr, s)));
  ISDF_CUDA(cudaEventRecord(ev.e[7], s));
  ISDF_CUDA(cudaEventRecord(ev.e[3], s));
  int err = 0;
  ISDF_TRY(read_back(&err, mb.err, sizeof(int), s));
  if (err) return record_error(ISDF_ERR_TIMEOUT, "mixed fit: a tensor-core pipeline wait timed out");
  ISDF_CUDA(cudaEventElapsedTime(&res->t_zct_ms, ev.e[0], ev.e[1]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_chol_ms, ev.e[1], ev.e[2]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_solve_ms, ev.e[2], ev.e[3]));
  float g1 = 0.f, g2 = 0.f;
  ISDF_CUDA(cudaEventElapsedTime(&g1, ev.e[4], ev.e[5]));
  ISDF_CUDA(cudaEventElapsedTime(&g2, ev.e[6], ev.e[7]));
  res->t_gemm_ms = g1 + g2;
  const int nblk = (rk + kNB - 1) / kNB;
  int levels = 0;
  for (int lv = kNB; lv < rk; lv *= 2) ++levels;
  res->launches = 1 + (same ? 3 : 6) * 2 + 2 + (nblk + 2 * (nblk - 1) + 1) + 1 + 2 * levels + 10 +
                  (readback_mailbox() ? 2 : 0);
  return ISDF_OK;
}

}  // namespace

size_t fit_mixed_workspace_bytes(long long ng, int nstate, int rk, int slices) {
  Arena a;
  a.counting = true;
  carve(a, nstate, rk);
  carve_mixed(a, ng, nstate, rk, slices);
  return a.off;
}

int fit_mixed(const FitArgs& args, Arena& arena, cudaStream_t s, FitResult* res, int slices) {
  if (args.ng <= 0 || args.rk <= 0 || args.nstate <= 0)
    return record_error(ISDF_ERR_ARG, "fit: bad sizes");
  if (args.ng > 0x7fffffffLL - 128) return record_error(ISDF_ERR_UNSUPPORTED, "mixed fit: Ng");
  ISDF_TRY(set_smem_attrs());
  switch (slices) {
    case 5: return fit_mixed_s<5>(args, arena, s, res);
    case 6: return fit_mixed_s<6>(args, arena, s, res);
    case 7: return fit_mixed_s<7>(args, arena, s, res);
    default: return record_error(ISDF_ERR_ARG, "mixed fit: slices must be 5, 6 or 7");
  }
}

}  // namespace isdf_b200
