// FP64 tensor-core GEMM core for sm_100a: mma.sync.aligned.m16n8k8 .f64.
//
// tcgen05 has no FP64 kind; on B200 the FP64 MMA path (mma.sync f64) runs at
// the full FP64 rate (measured ~37 TFLOP/s, DFMA ~34). CTA tile BM x BN with
// 8 warps (2 x 4), warp tile (BM/2) x (BN/4), BK = 16 per shared-memory stage,
// 3-stage cp.async pipeline (16-byte copies when both operands are 16-byte
// aligned with even leading dimensions, 8-byte copies otherwise).
//
// Operands: A column-major, A(m, k) = A[m + k*lda] (the tile's first row
// already applied); B depth-major, B(k, n) = B[k*ldb + n] (the tile's first
// column already applied). Shared-memory rows are padded by 8 doubles so the
// four k-rows a warp's fragment load touches fall on alternating bank halves.
#pragma once

#include <cuda_runtime.h>

#include "mbarrier.cuh"

namespace isdf_b200 {

namespace dmma {

constexpr int BK = 16;
constexpr int STAGES = 3;
constexpr int PAD = 8;

__device__ __forceinline__ void cp_async(void* smem, const void* gmem, int bytes, int src_bytes) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if (bytes == 16)
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_bytes));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem),
                 "r"(src_bytes));
}
__device__ __forceinline__ void commit() { asm volatile("cp.async.commit_group;\n"); }
template <int N>
__device__ __forceinline__ void wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

__device__ __forceinline__ void mma_16x8x8(double (&c)[4], const double (&a)[4],
                                           const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, "
      "{%8,%9}, {%0,%1,%2,%3};\n"
      : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

template <int BM_, int BN_>
struct Core {
  static constexpr int BM = BM_, BN = BN_;
  static constexpr int WM = BM / 2, WN = BN / 4;  // warp tile
  static constexpr int MT = WM / 16, NT = WN / 8;  // mma tiles per warp
  static constexpr int LDA_S = BM + PAD, LDB_S = BN + PAD;
  static constexpr int A_STAGE = BK * LDA_S, B_STAGE = BK * LDB_S;
  static constexpr int SMEM_DOUBLES = STAGES * (A_STAGE + B_STAGE);
  static constexpr size_t SMEM_BYTES = sizeof(double) * SMEM_DOUBLES;

  double acc[MT][NT][4];

  __device__ void zero() {
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
  }

  template <int VEC>
  __device__ static void load_stage(double* As, double* Bs, const double* A, long long lda,
                                    const double* B, long long ldb, int m_rem, int n_rem, int k0,
                                    int k_end) {
    const int tid = threadIdx.x;
    // A: BK rows (k) of BM contiguous doubles (m)
    constexpr int A_CHUNKS = BK * BM / VEC;
#pragma unroll
    for (int r = 0; r < A_CHUNKS / 256; ++r) {
      const int e = tid + r * 256;
      const int k = e / (BM / VEC), m = (e % (BM / VEC)) * VEC;
      int valid = (k0 + k < k_end) ? min(VEC, max(0, m_rem - m)) : 0;
      const double* src = valid ? A + m + (long long)(k0 + k) * lda : A;
      cp_async(As + k * LDA_S + m, src, VEC * 8, valid * 8);
    }
    constexpr int B_CHUNKS = BK * BN / VEC;
#pragma unroll
    for (int r = 0; r < B_CHUNKS / 256; ++r) {
      const int e = tid + r * 256;
      const int k = e / (BN / VEC), n = (e % (BN / VEC)) * VEC;
      int valid = (k0 + k < k_end) ? min(VEC, max(0, n_rem - n)) : 0;
      const double* src = valid ? B + (long long)(k0 + k) * ldb + n : B;
      cp_async(Bs + k * LDB_S + n, src, VEC * 8, valid * 8);
    }
  }

  __device__ void compute_stage(const double* As, const double* Bs) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp >> 2) * WM, wn0 = (warp & 3) * WN;
#pragma unroll
    for (int kk = 0; kk < BK; kk += 8) {
      double a[MT][4], b[NT][2];
#pragma unroll
      for (int i = 0; i < MT; ++i) {
        const double* p = As + (kk + t) * LDA_S + wm0 + i * 16 + g;
        a[i][0] = p[0];
        a[i][1] = p[8];
        a[i][2] = p[4 * LDA_S];
        a[i][3] = p[4 * LDA_S + 8];
      }
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const double* p = Bs + (kk + t) * LDB_S + wn0 + j * 8 + g;
        b[j][0] = p[0];
        b[j][1] = p[4 * LDB_S];
      }
#pragma unroll
      for (int i = 0; i < MT; ++i)
#pragma unroll
        for (int j = 0; j < NT; ++j) mma_16x8x8(acc[i][j], a[i], b[j]);
    }
  }

  // acc += A[0:BM, k_begin:k_end] * B[k_begin:k_end, 0:BN]
  template <int VEC>
  __device__ void run(double* smem, const double* A, long long lda, const double* B,
                      long long ldb, int m_rem, int n_rem, int k_begin, int k_end) {
    if (k_end <= k_begin) return;
    double* As = smem;
    double* Bs = smem + STAGES * A_STAGE;
    const int nk = (k_end - k_begin + BK - 1) / BK;
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
      if (s < nk)
        load_stage<VEC>(As + s * A_STAGE, Bs + s * B_STAGE, A, lda, B, ldb, m_rem, n_rem,
                        k_begin + s * BK, k_end);
      commit();
    }
    for (int t = 0; t < nk; ++t) {
      wait<STAGES - 2>();
      __syncthreads();
      const int nt = t + STAGES - 1;
      if (nt < nk) {
        const int st = nt % STAGES;
        load_stage<VEC>(As + st * A_STAGE, Bs + st * B_STAGE, A, lda, B, ldb, m_rem, n_rem,
                        k_begin + nt * BK, k_end);
      }
      commit();
      const int cs = t % STAGES;
      compute_stage(As + cs * A_STAGE, Bs + cs * B_STAGE);
    }
    wait<0>();
    __syncthreads();
  }

  // Calls f(row, col, value) for every accumulator element (tile-relative).
  template <class F>
  __device__ void for_each(F f) const {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp >> 2) * WM, wn0 = (warp & 3) * WN;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int r = wm0 + i * 16 + g, c = wn0 + j * 8 + 2 * t;
        f(r, c, acc[i][j][0]);
        f(r, c + 1, acc[i][j][1]);
        f(r + 8, c, acc[i][j][2]);
        f(r + 8, c + 1, acc[i][j][3]);
      }
  }
};

// A row of zeros: the source of the warp-specialised tile's copies for the
// columns and rows outside the operands.
static __device__ __align__(128) double g_zero_row[256];

// Warp-specialised FP64 tensor-core tile. WGM x WGN consumer warps compute
// the BM x BN tile with mma.sync f64 (warp tile (BM/WGM) x (BN/WGN)); one
// producer warp fills an ST-deep ring of BK-deep stages with bulk copies:
// per stage BK columns of A (BM contiguous doubles each) and BK rows of B (BN
// contiguous doubles each), each into a padded shared-memory row (same
// fragment layout as Core), all completing on the stage's "full" mbarrier by
// transaction count. A column or row past K, and the rows / columns past
// m_rem / n_rem, are copied from a zero row, so every stage carries the same
// byte count and the fragments never read stale shared memory. Each consumer
// warp releases a stage through its "empty" mbarrier after a proxy fence (its
// shared-memory reads are generic-proxy accesses, the refill an async-proxy
// write: without the fence, served solves running side by side saw stages
// overwritten under the readers), so nothing in the K loop synchronises the
// whole CTA.
// Requirements (host-checked): A and B 16-byte aligned; lda, ldb, m_rem and
// n_rem even.
template <int BM_, int BN_, int WGM, int WGN, int BK_, int ST_>
struct WsTile {
  static constexpr int BM = BM_, BN = BN_, BK = BK_, ST = ST_;
  static constexpr int NW = WGM * WGN, THREADS = NW * 32 + 32;
  static constexpr int WM = BM / WGM, WN = BN / WGN;
  static constexpr int MT = WM / 16, NT = WN / 8;
  static constexpr int LDA_S = BM + PAD, LDB_S = BN + PAD;
  static constexpr int A_STAGE = BK * LDA_S, B_STAGE = BK * LDB_S;
  static constexpr size_t BAR_OFF = sizeof(double) * ST * (A_STAGE + B_STAGE);
  static constexpr size_t SMEM_BYTES = BAR_OFF + 16 * ST + 16;
  static constexpr uint32_t STAGE_TX = (uint32_t)(BK * (BM + BN) * sizeof(double));
  static_assert(BM <= 256 && BN <= 256, "zero row");
  static_assert(WM % 16 == 0 && WN % 8 == 0 && BK % 8 == 0, "tile shape");

  double acc[MT][NT][4];

  __device__ static bool producer() { return (threadIdx.x >> 5) == NW; }

  // acc = A[0:m_rem, 0:K] * B[0:K, 0:n_rem] (zero outside), with
  // A(m, k) = A[m + k*lda] and B(k, n) = B[k*ldb + n]. Every thread of the
  // CTA calls it. Returns false (and sets *err) when a wait ran out; the
  // producer warp returns with acc unset.
  __device__ bool run(void* smem, const double* A, long long lda, int m_rem, const double* B,
                      long long ldb, int n_rem, int K, int* err) {
    uint8_t* base = static_cast<uint8_t*>(smem);
    double* As = reinterpret_cast<double*>(base);
    double* Bs = As + ST * A_STAGE;
    const uint32_t fb = smem_u32(base + BAR_OFF), eb = fb + 8u * ST;
    volatile int* abortp = reinterpret_cast<volatile int*>(base + BAR_OFF + 16 * ST);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    if (tid == 0) {
      for (int i = 0; i < ST; ++i) {
        mbar_init(fb + 8u * i, 1);
        mbar_init(eb + 8u * i, NW);
      }
      *abortp = 0;
      asm volatile("fence.mbarrier_init.release.cluster;\n");
    }
    __syncthreads();
    const int nk = K > 0 ? (K + BK - 1) / BK : 0;
    bool ok = true;
    if (warp == NW) {
      // ------------------------------------------------------------ copies
      int issued = 0;
      for (int kt = 0; kt < nk; ++kt) {
        const int s = kt % ST;
        bool w = true;
        if (kt >= ST) w = mbar_wait(eb + 8u * s, (uint32_t)((kt / ST) - 1) & 1u, abortp);
        if (!__all_sync(0xffffffffu, w)) {
          ok = false;
          break;
        }
        if (lane == 0) mbar_expect_tx(fb + 8u * s, STAGE_TX);
        __syncwarp();
        const uint32_t as = smem_u32(As + s * A_STAGE), bs = smem_u32(Bs + s * B_STAGE);
        const int k0 = kt * BK;
        for (int c = lane; c < 2 * BK; c += 32) {
          const bool is_a = c < BK;
          const int k = k0 + (is_a ? c : c - BK);
          const int rows = is_a ? BM : BN;
          const int valid = k < K ? min(rows, is_a ? m_rem : n_rem) : 0;
          const uint32_t dst = is_a ? as + (uint32_t)(c * LDA_S * 8)
                                    : bs + (uint32_t)((c - BK) * LDB_S * 8);
          if (valid > 0)
            bulk_copy(dst, is_a ? A + (long long)k * lda : B + (long long)k * ldb,
                      (uint32_t)valid * 8u, fb + 8u * s);
          if (valid < rows)
            bulk_copy(dst + (uint32_t)valid * 8u, g_zero_row, (uint32_t)(rows - valid) * 8u,
                      fb + 8u * s);
        }
        ++issued;
      }
      // no copy may still be landing when the CTA exits
      if (lane == 0)
        for (int t = issued > ST ? issued - ST : 0; t < issued; ++t)
          if (!mbar_wait_all(fb + 8u * (t % ST), (uint32_t)(t / ST) & 1u)) ok = false;
      if (lane == 0 && (!ok || *abortp)) *err = 1;
      __syncwarp();
      return ok;
    }
    // -------------------------------------------------------------- DMMA
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j)
#pragma unroll
        for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp / WGN) * WM, wn0 = (warp % WGN) * WN;
    for (int kt = 0; kt < nk; ++kt) {
      const int s = kt % ST;
      if (!__all_sync(0xffffffffu, mbar_wait(fb + 8u * s, (uint32_t)(kt / ST) & 1u, abortp))) {
        ok = false;
        break;
      }
      const double* as = As + s * A_STAGE;
      const double* bs = Bs + s * B_STAGE;
#pragma unroll
      for (int kk = 0; kk < BK; kk += 8) {
        double a[MT][4], b[NT][2];
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          const double* p = as + (kk + t) * LDA_S + wm0 + i * 16 + g;
          a[i][0] = p[0];
          a[i][1] = p[8];
          a[i][2] = p[4 * LDA_S];
          a[i][3] = p[4 * LDA_S + 8];
        }
#pragma unroll
        for (int j = 0; j < NT; ++j) {
          const double* p = bs + (kk + t) * LDB_S + wn0 + j * 8 + g;
          b[j][0] = p[0];
          b[j][1] = p[4 * LDB_S];
        }
#pragma unroll
        for (int i = 0; i < MT; ++i)
#pragma unroll
          for (int j = 0; j < NT; ++j) mma_16x8x8(acc[i][j], a[i], b[j]);
      }
      // the stage's fragment loads (generic proxy) must be ordered before the
      // producer's next bulk copy into the slot (async proxy)
      asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(eb + 8u * s);
    }
    if (!ok && lane == 0) *err = 1;
    return ok;
  }

  // Calls f(row, col, value) for every accumulator element (consumer warps).
  template <class F>
  __device__ void for_each(F f) const {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;
    const int wm0 = (warp / WGN) * WM, wn0 = (warp % WGN) * WN;
#pragma unroll
    for (int i = 0; i < MT; ++i)
#pragma unroll
      for (int j = 0; j < NT; ++j) {
        const int r = wm0 + i * 16 + g, c = wn0 + j * 8 + 2 * t;
        f(r, c, acc[i][j][0]);
        f(r, c + 1, acc[i][j][1]);
        f(r + 8, c, acc[i][j][2]);
        f(r + 8, c + 1, acc[i][j][3]);
      }
  }
};

}  // namespace dmma
}  // namespace isdf_b200
