// FP64-accurate GEMM from INT8 slices on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, INT32 accumulators in TMEM).
//
// Each FP64 operand row (A) or column (B) is scaled by a power of two 2^e and
// split into S signed 8-bit slices, x = 2^e sum_t q_t 2^{-7(t+1)}, |q_t| <= 64.
// The product of two split numbers is a sum of integer slice products; every
// slice-pair GEMM accumulates exactly in INT32 (|q| <= 64, K <= 2^17), and the
// pairs with the same t + u = d share one TMEM accumulator:
//   C(m, n) = 2^{ea_m + eb_n} sum_{d < S} S_d(m, n) 2^{-7(d+2)}.
// Pairs with t + u >= S are dropped (the usual truncation of the scheme).
//
// CTA: 128 threads, output tile 128 x 64, S accumulators of 64 TMEM columns.
// Shared-memory operand tiles use the canonical K-major no-swizzle layout of
// the UMMA descriptors: 16-byte K chunks, rows of a chunk contiguous
// (LBO = distance between K chunks, SBO = 128 B between 8-row groups). Two
// stages: all threads cp.async the next K-tile while thread 0's MMAs run on
// the current one; tcgen05.commit arrives on the stage's mbarrier, and every
// wait on it is bounded (a timeout sets *err and the kernel skips ahead,
// still freeing its TMEM).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace isdf_b200 {
namespace ozaki {

constexpr int BM = 128, BN = 64, BKB = 64;  // tile rows, tile columns, K bytes per stage
constexpr int kTmemCols = 512;
constexpr long long kSpinLimit = 1ll << 26;

template <int S>
struct Cfg {
  static constexpr int A_PLANE = BM * BKB;  // bytes of one slice's A tile per stage
  static constexpr int B_PLANE = BN * BKB;
  static constexpr int STAGE = S * (A_PLANE + B_PLANE);
  static constexpr int SMEM = 2 * STAGE + 64;  // + mbarriers
  static_assert(S * BN <= kTmemCols, "TMEM columns");
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, no swizzle
}

// kind::i8, D = S32, A = B = signed 8-bit, both K-major, M = 128, N = 64.
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) |
                            ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
      mbar));
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity) {
  for (long long i = 0; i < kSpinLimit; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity));
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void cp16(uint32_t saddr, const void* g) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(saddr), "l"(g));
}

// Loads one stage: S A-planes (128 rows x 64 B) and S B-planes (64 rows x 64 B)
// into the chunked layout [plane][chunk 0..3][row][16 B].
template <int S>
__device__ __forceinline__ void load_stage(uint8_t* st, const int8_t* A, long long a_plane,
                                           int lda, const int8_t* B, long long b_plane, int ldb,
                                           int kbyte) {
  using C = Cfg<S>;
  const int tid = threadIdx.x;
  // A: S * 128 rows * 4 chunks = S * 512 copies
#pragma unroll
  for (int r = 0; r < S * 4; ++r) {
    const int e = tid + r * 128;
    const int plane = e >> 9, rem = e & 511, row = rem >> 2, chunk = rem & 3;
    const int8_t* g = A + plane * a_plane + (long long)row * lda + kbyte + chunk * 16;
    cp16(smem_u32(st + plane * C::A_PLANE + chunk * (BM * 16) + row * 16), g);
  }
  uint8_t* sb = st + S * C::A_PLANE;
#pragma unroll
  for (int r = 0; r < S * 2; ++r) {
    const int e = tid + r * 128;
    const int plane = e >> 8, rem = e & 255, row = rem >> 2, chunk = rem & 3;
    const int8_t* g = B + plane * b_plane + (long long)row * ldb + kbyte + chunk * 16;
    cp16(smem_u32(sb + plane * C::B_PLANE + chunk * (BN * 16) + row * 16), g);
  }
}

// EPI 0: C = value; 1: C = value^2; 2: C = C * value.
// KMODE 0: full K; 1: B(k, n) = 0 for k > n (upper); 2: B(k, n) = 0 for k < n (lower).
// A: planes of (rows padded to 128) x ldk bytes; B: planes of (cols padded to 64) x ldk bytes;
// the K extent kp is a multiple of BKB with zero slices past the true K.
template <int S, int EPI, int KMODE>
__global__ void __launch_bounds__(128, 1)
    k_ozaki_gemm(const int8_t* __restrict__ A, long long a_plane, int lda,
                 const int8_t* __restrict__ B, long long b_plane, int ldb,
                 const int* __restrict__ ea, const int* __restrict__ eb, int M, int N, int kp,
                 double* __restrict__ C, long long ldc, int* __restrict__ err) {
  using Cf = Cfg<S>;
  extern __shared__ __align__(1024) uint8_t smem[];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const long long m0 = (long long)blockIdx.y * BM;
  const int n0 = blockIdx.x * BN;
  uint8_t* stage[2] = {smem, smem + Cf::STAGE};
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + 2 * Cf::STAGE);
  const uint32_t bar0 = smem_u32(&bars[0]), bar1 = smem_u32(&bars[1]);

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar0));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;\n" ::"r"(bar1));
    asm volatile("fence.mbarrier_init.release.cluster;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = tmem_slot;

  const int8_t* Ab = A + m0 * lda;
  const int8_t* Bb = B + (long long)n0 * ldb;
  // K range of this tile (triangular B: KMODE 1 keeps k < n0 + BN, 2 keeps k >= n0)
  int kb = 0, ke = kp;
  if (KMODE == 1) ke = min(kp, ((n0 + BN + BKB - 1) / BKB) * BKB);
  if (KMODE == 2) kb = (n0 / BKB) * BKB;
  const int nk = (ke - kb) / BKB;
  bool ok = true;
  int last_bar = -1;
  uint32_t last_parity = 0;
  if (nk > 0) load_stage<S>(stage[0], Ab, a_plane, lda, Bb, b_plane, ldb, kb);
  asm volatile("cp.async.commit_group;\n");
  for (int t = 0; t < nk; ++t) {
    const int cur = t & 1;
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
    if (!__syncthreads_and(ok)) {
      ok = false;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const uint32_t sa = smem_u32(stage[cur]);
      const uint32_t sbb = sa + S * Cf::A_PLANE;
#pragma unroll
      for (int d = 0; d < S; ++d) {
#pragma unroll
        for (int ta = 0; ta <= d; ++ta) {
          const int ub = d - ta;
#pragma unroll
          for (int kk = 0; kk < BKB / 32; ++kk) {
            const uint64_t ad =
                umma_desc(sa + ta * Cf::A_PLANE + kk * 2 * (BM * 16), BM * 16, 128);
            const uint64_t bd =
                umma_desc(sbb + ub * Cf::B_PLANE + kk * 2 * (BN * 16), BN * 16, 128);
            const uint32_t acc = (t > 0 || ta > 0 || kk > 0) ? 1u : 0u;
            mma_i8(tmem + (uint32_t)(d * BN), ad, bd, acc);
          }
        }
      }
      mma_commit(cur ? bar1 : bar0);
    }
    last_bar = cur;
    last_parity = (uint32_t)((t >> 1) & 1);
    // before refilling the other buffer, its previous MMAs must have finished
    if (t + 1 < nk) {
      if (t >= 1) {
        const int prev = (t - 1) & 1;
        if (!mbar_wait(prev ? bar1 : bar0, ((t - 1) >> 1) & 1)) ok = false;
      }
      if (ok) load_stage<S>(stage[cur ^ 1], Ab, a_plane, lda, Bb, b_plane, ldb, kb + (t + 1) * BKB);
      asm volatile("cp.async.commit_group;\n");
    }
  }
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
  // tcgen05.commit tracks every earlier MMA of the thread: the last commit's
  // phase completes the accumulators. Waited even after a timeout (bounded),
  // so that no MMA is in flight when the TMEM is freed.
  if (last_bar >= 0 && !mbar_wait(last_bar ? bar1 : bar0, last_parity)) ok = false;
  ok = __syncthreads_and(ok);
  if (!ok && tid == 0) atomicExch(err, 1);
  asm volatile("tcgen05.fence::after_thread_sync;\n");

  if (ok) {
    // warp w owns TMEM lanes 32w..32w+31 = tile rows
    const int row = warp * 32 + lane;
    const long long m = m0 + row;
    const double sa = (m < M) ? ldexp(1.0, ea[m]) : 0.0;
    double out[BN];
#pragma unroll
    for (int j = 0; j < BN; ++j) out[j] = 0.0;
#pragma unroll
    for (int d = 0; d < S; ++d) {
      if (nk == 0) break;  // empty K range: the tile is zero
      const double w = ldexp(1.0, -7 * (d + 2));
#pragma unroll
      for (int c0 = 0; c0 < BN; c0 += 16) {
        uint32_t v[16];
        const uint32_t addr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(d * BN + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,"
            "%13,%14,%15}, [%16];\n"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
              "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
              "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(addr));
        asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
        for (int j = 0; j < 16; ++j) out[c0 + j] += (double)(int)v[j] * w;
      }
    }
    if (m < M) {
#pragma unroll
      for (int j = 0; j < BN; ++j) {
        const int n = n0 + j;
        if (n < N) {
          const double val = out[j] * sa * ldexp(1.0, eb[n]);
          double* p = C + m + (long long)n * ldc;
          if (EPI == 0) *p = val;
          else if (EPI == 1) *p = val * val;
          else *p = *p * val;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols));
}

}  // namespace ozaki
}  // namespace isdf_b200
