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
// Kernels: one DFMA register-tiled GEMM core (128 x 128 or 128 x 64 CTA
// tiles, 8 x 8 / 8 x 4 outputs per thread, cp.async double buffering) used by
// the Z GEMM, the Cholesky panel / trailing updates and the triangular-solve
// steps; a single-CTA 64 x 64 diagonal-block factor + inverse.
// theta is column-major Ng x rk (ld = Ng), overwritten in place.
#include <vector>

#include "arena.h"
#include "common.cuh"
#include "fit.h"

namespace isdf_b200 {

namespace {

constexpr int kBK = 16;  // k-depth of one smem stage
constexpr int kNB = 64;  // Cholesky / TRSM block size

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool ok) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  int sz = ok ? 8 : 0;
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(sz));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// CTA tile: BM = 16*TM rows, BN = 16*TN columns, 256 threads as 16 x 16.
// Thread (tx, ty) owns rows {i*64 + tx*4 + r} and columns {j*64 + ty*4 + c}.
// A: column-major (row m, depth k) at A[m + k*lda], already offset to the
// tile's first row. B: depth-major (depth k, column n) at B[k*ldb + n],
// already offset to the tile's first column.
template <int TM, int TN>
struct Tile {
  static constexpr int BM = 16 * TM;
  static constexpr int BN = 16 * TN;
  static constexpr int A_STAGE = kBK * BM;
  static constexpr int B_STAGE = kBK * BN;
  static constexpr int SMEM_DOUBLES = 2 * (A_STAGE + B_STAGE);

  __device__ static void load(double* As, double* Bs, const double* A, long long lda,
                              const double* B, long long ldb, int m_rem, int n_rem, int k0,
                              int k_end) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int r = 0; r < A_STAGE / 256; ++r) {
      int e = tid + r * 256;
      int k = e / BM, m = e % BM;
      bool ok = (m < m_rem) && (k0 + k < k_end);
      const double* src = ok ? A + m + (long long)(k0 + k) * lda : A;
      cp_async8(As + e, src, ok);
    }
#pragma unroll
    for (int r = 0; r < B_STAGE / 256; ++r) {
      int e = tid + r * 256;
      int k = e / BN, n = e % BN;
      bool ok = (n < n_rem) && (k0 + k < k_end);
      const double* src = ok ? B + (long long)(k0 + k) * ldb + n : B;
      cp_async8(Bs + e, src, ok);
    }
  }

  // acc += A[0:BM, k_begin:k_end] * B[k_begin:k_end, 0:BN]
  __device__ static void accumulate(double (&acc)[TM][TN], double* smem, const double* A,
                                    long long lda, const double* B, long long ldb, int m_rem,
                                    int n_rem, int k_begin, int k_end) {
    if (k_end <= k_begin) return;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double* As0 = smem;
    double* Bs0 = smem + 2 * A_STAGE;
    const int nk = (k_end - k_begin + kBK - 1) / kBK;
    load(As0, Bs0, A, lda, B, ldb, m_rem, n_rem, k_begin, k_end);
    cp_async_commit();
    for (int t = 0; t < nk; ++t) {
      const int cur = t & 1;
      if (t + 1 < nk) {
        load(As0 + (cur ^ 1) * A_STAGE, Bs0 + (cur ^ 1) * B_STAGE, A, lda, B, ldb, m_rem, n_rem,
             k_begin + (t + 1) * kBK, k_end);
      }
      cp_async_commit();
      cp_async_wait<1>();
      __syncthreads();
      const double* As = As0 + cur * A_STAGE;
      const double* Bs = Bs0 + cur * B_STAGE;
#pragma unroll
      for (int kk = 0; kk < kBK; ++kk) {
        double a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM / 4; ++i) {
          const double2* p = reinterpret_cast<const double2*>(As + kk * BM + i * 64 + tx * 4);
          double2 v0 = p[0], v1 = p[1];
          a[i * 4 + 0] = v0.x;
          a[i * 4 + 1] = v0.y;
          a[i * 4 + 2] = v1.x;
          a[i * 4 + 3] = v1.y;
        }
#pragma unroll
        for (int j = 0; j < TN / 4; ++j) {
          const double2* p = reinterpret_cast<const double2*>(Bs + kk * BN + j * 64 + ty * 4);
          double2 v0 = p[0], v1 = p[1];
          b[j * 4 + 0] = v0.x;
          b[j * 4 + 1] = v0.y;
          b[j * 4 + 2] = v1.x;
          b[j * 4 + 3] = v1.y;
        }
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      __syncthreads();
    }
    cp_async_wait<0>();
  }

  __device__ static int row(int i) { return (i >> 2) * 64 + (threadIdx.x & 15) * 4 + (i & 3); }
  __device__ static int col(int j) { return (j >> 2) * 64 + (threadIdx.x >> 4) * 4 + (j & 3); }
};

// ----------------------------------------------------------- Z C^T GEMM
// mode 0: C = acc*acc (S1 = S2); mode 1: C = acc (first factor);
// mode 2: C = C * acc (second factor, S1 != S2).
template <int MODE>
__global__ void __launch_bounds__(256) k_gemm_z(int M, int N, int K, const double* __restrict__ A,
                                                long long lda, const double* __restrict__ B,
                                                long long ldb, double* __restrict__ C,
                                                long long ldc) {
  using T = Tile<8, 8>;
  extern __shared__ double smem[];
  const int n0 = blockIdx.x * T::BN;
  const long long m0 = (long long)blockIdx.y * T::BM;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  T::accumulate(acc, smem, A + m0, lda, B + n0, ldb, (int)(M - m0 < T::BM ? M - m0 : T::BM), N - n0,
                0, K);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    const int n = n0 + T::col(j);
    if (n >= N) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const long long m = m0 + T::row(i);
      if (m >= M) continue;
      double* c = C + m + (long long)n * ldc;
      if (MODE == 0) *c = acc[i][j] * acc[i][j];
      else if (MODE == 1) *c = acc[i][j];
      else *c = *c * acc[i][j];
    }
  }
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
    const int rem = bs - j - 1;
    for (int e = tid; e < rem * rem; e += 256) {
      int i = j + 1 + e / rem, c = j + 1 + e % rem;
      if (c <= i) a[i][c] -= a[i][j] * a[c][j];
    }
    __syncthreads();
  }
  // X = L^{-1}, one thread per column
  if (tid < bs) {
    const int c = tid;
    x[c][c] = 1.0 / a[c][c];
    for (int i = c + 1; i < bs; ++i) {
      double s = 0.0;
      for (int k = c; k < i; ++k) s = fma(a[i][k], x[k][c], s);
      x[i][c] = -s / a[i][i];
    }
  }
  __syncthreads();
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
__global__ void __launch_bounds__(256) k_chol_panel(double* A, int lda, int k0, int bs, int n,
                                                    const double* __restrict__ dinvT) {
  using T = Tile<8, 4>;
  extern __shared__ double smem[];
  const int m0 = k0 + bs + blockIdx.x * T::BM;
  double acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  double* Ablk = A + m0 + (long long)k0 * lda;
  T::accumulate(acc, smem, Ablk, lda, dinvT, kNB, n - m0, bs, 0, bs);
  __syncthreads();
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    int c = T::col(j);
    if (c >= bs) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int m = m0 + T::row(i);
      if (m < n) A[m + (long long)(k0 + c) * lda] = acc[i][j];
    }
  }
}

// Trailing update of the lower part: A[r, c] -= sum_k L[r, k] L[c, k] for
// r, c >= k0+bs, k in the panel. Tiles wholly above the diagonal are skipped.
__global__ void __launch_bounds__(256) k_chol_update(double* A, int lda, int k0, int bs, int n) {
  using T = Tile<8, 8>;
  extern __shared__ double smem[];
  const int base = k0 + bs;
  const int n0 = base + blockIdx.x * T::BN;
  const int m0 = base + blockIdx.y * T::BM;
  if (m0 + T::BM <= n0) return;
  double acc[8][8];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  const double* Ap = A + m0 + (long long)k0 * lda;
  const double* Bp = A + n0 + (long long)k0 * lda;  // B(k, c) = L[n0 + c, k0 + k]
  T::accumulate(acc, smem, Ap, lda, Bp, lda, n - m0, n - n0, 0, bs);
#pragma unroll
  for (int j = 0; j < 8; ++j) {
    int c = n0 + T::col(j);
    if (c >= n) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      int r = m0 + T::row(i);
      if (r < n && r >= c) A[r + (long long)c * lda] -= acc[i][j];
    }
  }
}

// LT = L^T (column-major), and the strict upper triangle of L cleared.
__global__ void k_transpose_lower(double* L, int n, double* __restrict__ LT) {
  const long long total = (long long)n * n;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    int r = (int)(e % n), c = (int)(e / n);
    double v = r >= c ? L[e] : 0.0;
    if (r < c) L[e] = 0.0;
    LT[(long long)c + (long long)r * n] = v;
  }
}

// ----------------------------------------------------------- triangular solve
// One column block [c0, c0+bs) of one sweep, for a 128-row tile of theta:
//   out = (theta[rows, c0:c0+bs] - theta[rows, kr] * B[kr, c0:c0+bs]) * D
// forward  (theta L^T = Z): kr = [0, c0),       B(k, n) = L(c0+n, k) = L[c0+n + k*rk]
// backward (theta L = Y):   kr = [c0+bs, rk),   B(k, n) = L(k, c0+n) = LT[c0+n + k*rk]
// D = the padded inverse of the diagonal block (dinvT forward, dinv backward).
// Rows are independent, so each CTA overwrites its own tile in place.
__global__ void __launch_bounds__(256) k_trsm_step(double* theta, long long ng, int rk,
                                                   const double* __restrict__ Bop, int c0, int bs,
                                                   int k_begin, int k_end,
                                                   const double* __restrict__ D) {
  using T = Tile<8, 4>;
  extern __shared__ double smem[];
  const long long m0 = (long long)blockIdx.x * T::BM;
  const int m_rem = (int)(ng - m0 < T::BM ? ng - m0 : T::BM);
  double acc[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  T::accumulate(acc, smem, theta + m0, ng, Bop + c0, rk, m_rem, bs, k_begin, k_end);
  __syncthreads();
  // stage t = rhs - acc (128 x 64, column-major, ld 128) and D (64 x 64)
  double* ts = smem;
  double* ds = smem + T::BM * kNB;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = T::col(j);
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = T::row(i);
      double v = 0.0;
      if (r < m_rem && c < bs) v = theta[m0 + r + (long long)(c0 + c) * ng] - acc[i][j];
      ts[r + c * T::BM] = v;
    }
  }
  for (int e = threadIdx.x; e < kNB * kNB; e += 256) ds[e] = D[e];
  __syncthreads();
  double out[8][4];
#pragma unroll
  for (int i = 0; i < 8; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) out[i][j] = 0.0;
  for (int k = 0; k < kNB; ++k) {
    double a[8], b[4];
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = ts[T::row(i) + k * T::BM];
#pragma unroll
    for (int j = 0; j < 4; ++j) b[j] = ds[k * kNB + T::col(j)];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) out[i][j] = fma(a[i], b[j], out[i][j]);
  }
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const int c = T::col(j);
    if (c >= bs) continue;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
      const int r = T::row(i);
      if (r < m_rem) theta[m0 + r + (long long)(c0 + c) * ng] = out[i][j];
    }
  }
}

constexpr size_t smem_bytes_88 = sizeof(double) * Tile<8, 8>::SMEM_DOUBLES;
constexpr size_t smem_bytes_84 = sizeof(double) * Tile<8, 4>::SMEM_DOUBLES;
constexpr size_t smem_bytes_trsm =
    sizeof(double) * ((Tile<8, 4>::SMEM_DOUBLES > 128 * kNB + kNB * kNB)
                          ? Tile<8, 4>::SMEM_DOUBLES
                          : 128 * kNB + kNB * kNB);

constexpr size_t smem_bytes_potf2 = sizeof(double) * 2 * kNB * (kNB + 1);

int set_smem_attrs() {
  static bool done_dev[64] = {};
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done_dev[dev]) return ISDF_OK;
  ISDF_CUDA(cudaFuncSetAttribute(k_potf2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_potf2));
  ISDF_CUDA(cudaFuncSetAttribute(k_gemm_z<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_88));
  ISDF_CUDA(cudaFuncSetAttribute(k_gemm_z<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_88));
  ISDF_CUDA(cudaFuncSetAttribute(k_gemm_z<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_88));
  ISDF_CUDA(cudaFuncSetAttribute(k_chol_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_88));
  ISDF_CUDA(cudaFuncSetAttribute(k_chol_panel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_84));
  ISDF_CUDA(cudaFuncSetAttribute(k_trsm_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem_bytes_trsm));
  if (dev >= 0 && dev < 64) done_dev[dev] = true;
  return ISDF_OK;
}

struct FitBuffers {
  int* piv;
  double* Bm;
  double* P;   // C C^T, then L (column-major rk x rk)
  double* LT;  // L^T
  double* dinvT;
  double* dinv;
  double* eps;
  int* info;
};

FitBuffers carve(Arena& a, int nstate, int rk) {
  FitBuffers b;
  const int nblk = (rk + kNB - 1) / kNB;
  b.piv = a.take<int>(rk);
  b.Bm = a.take<double>((size_t)nstate * rk);
  b.P = a.take<double>((size_t)rk * rk);
  b.LT = a.take<double>((size_t)rk * rk);
  b.dinvT = a.take<double>((size_t)nblk * kNB * kNB);
  b.dinv = a.take<double>((size_t)nblk * kNB * kNB);
  b.eps = a.take<double>(1);
  b.info = a.take<int>(1);
  return b;
}

}  // namespace

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
  for (int kb = 0; kb < nblk; ++kb) {
    const int k0 = kb * kNB;
    const int bs = min(kNB, rk - k0);
    k_potf2<<<1, 256, smem_bytes_potf2, s>>>(b.P, rk, k0, bs, b.dinvT + (size_t)kb * kNB * kNB,
                              b.dinv + (size_t)kb * kNB * kNB, b.info);
    const int rem = rk - k0 - bs;
    if (rem > 0) {
      k_chol_panel<<<(rem + 127) / 128, 256, smem_bytes_84, s>>>(
          b.P, rk, k0, bs, rk, b.dinvT + (size_t)kb * kNB * kNB);
      dim3 g((rem + 127) / 128, (rem + 127) / 128);
      k_chol_update<<<g, 256, smem_bytes_88, s>>>(b.P, rk, k0, bs, rk);
    }
  }
  k_transpose_lower<<<grid_for((long long)rk * rk, 256), 256, 0, s>>>(b.P, rk, b.LT);
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

// Stage timers: CUDA events on the solve stream.
struct StageEvents {
  cudaEvent_t e[4] = {nullptr, nullptr, nullptr, nullptr};
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
  res->launches = 1 + (same_ ? 1 : 2) + 2 + (nblk_ + 2 * (nblk_ - 1) + 1) + 2 * nblk_;

  ISDF_CUDA(cudaMemcpyAsync(b.piv, args.piv, sizeof(int) * rk, cudaMemcpyHostToDevice, s));
  ISDF_CUDA(cudaMemsetAsync(b.info, 0, sizeof(int), s));
  k_gather_psimu<<<grid_for((long long)args.nstate * rk, 256), 256, 0, s>>>(
      args.d_psi, ng, args.nstate, b.piv, rk, b.Bm);

  // Z C^T into theta
  const int lo1 = args.nocc - args.nv1, K1 = args.nv1 + args.nc1;
  const int lo2 = args.nocc - args.nv2, K2 = args.nv2 + args.nc2;
  const bool same = (args.nv1 == args.nv2 && args.nc1 == args.nc2);
  dim3 zg((unsigned)((rk + 127) / 128), (unsigned)((ng + 127) / 128));
  ISDF_CUDA(mark(0));
  if (same) {
    k_gemm_z<0><<<zg, 256, smem_bytes_88, s>>>((int)ng, rk, K1, args.d_psi + (long long)lo1 * ng,
                                               ng, b.Bm + (size_t)lo1 * rk, rk, args.d_theta, ng);
  } else {
    k_gemm_z<1><<<zg, 256, smem_bytes_88, s>>>((int)ng, rk, K1, args.d_psi + (long long)lo1 * ng,
                                               ng, b.Bm + (size_t)lo1 * rk, rk, args.d_theta, ng);
    k_gemm_z<2><<<zg, 256, smem_bytes_88, s>>>((int)ng, rk, K2, args.d_psi + (long long)lo2 * ng,
                                               ng, b.Bm + (size_t)lo2 * rk, rk, args.d_theta, ng);
  }
  ISDF_CHECK_LAUNCH();

  // C C^T, regularisation, Cholesky
  ISDF_CUDA(mark(1));
  k_gather_cct<<<grid_for((long long)rk * rk, 256), 256, 0, s>>>(args.d_theta, ng, b.piv, rk, b.P);
  k_regularise<<<1, 256, 0, s>>>(b.P, rk, b.eps);
  ISDF_TRY(cholesky(b, rk, s));
  ISDF_CUDA(mark(2));
  int info = 0;
  ISDF_CUDA(cudaMemcpyAsync(&info, b.info, sizeof(int), cudaMemcpyDeviceToHost, s));
  ISDF_CUDA(cudaStreamSynchronize(s));
  res->chol_info = info;
  if (info != 0) return record_error(ISDF_ERR_NOT_SPD, "fit: C C^T + eps I is not positive definite");

  // theta L^T = Z C^T (forward over column blocks), then theta L = Y (backward)
  const int nblk = (rk + kNB - 1) / kNB;
  const unsigned tg = (unsigned)((ng + 127) / 128);
  for (int kb = 0; kb < nblk; ++kb) {
    const int c0 = kb * kNB, bs = min(kNB, rk - c0);
    k_trsm_step<<<tg, 256, smem_bytes_trsm, s>>>(args.d_theta, ng, rk, b.P, c0, bs, 0, c0,
                                                 b.dinvT + (size_t)kb * kNB * kNB);
  }
  for (int kb = nblk - 1; kb >= 0; --kb) {
    const int c0 = kb * kNB, bs = min(kNB, rk - c0);
    k_trsm_step<<<tg, 256, smem_bytes_trsm, s>>>(args.d_theta, ng, rk, b.LT, c0, bs, c0 + bs, rk,
                                                 b.dinv + (size_t)kb * kNB * kNB);
  }
  ISDF_CHECK_LAUNCH();
  ISDF_CUDA(mark(3));
  if (!timed) return ISDF_OK;
  ISDF_CUDA(cudaEventSynchronize(ev.e[3]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_zct_ms, ev.e[0], ev.e[1]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_chol_ms, ev.e[1], ev.e[2]));
  ISDF_CUDA(cudaEventElapsedTime(&res->t_solve_ms, ev.e[2], ev.e[3]));
  return ISDF_OK;
}

}  // namespace isdf_b200
