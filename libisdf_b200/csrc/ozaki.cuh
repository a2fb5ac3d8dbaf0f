// FP64-accurate GEMM from INT8 slices on the 5th-generation tensor cores
// (tcgen05.mma kind::i8, INT32 accumulators in TMEM).
//
// Each FP64 operand row (A) or column (B) is scaled by a power of two 2^e
// (|x| 2^-e <= 1/2) and split into S signed 8-bit digits in base 254,
//   x = 2^e sum_t q_t 254^{-(t+1)},  |q_t| <= 127,
// by q_t = rint(r * 254), r <- r * 254 - q_t (|r| stays <= 1/2, so no digit
// overflows int8, and every digit carries log2(254) = 7.99 bits). The product
// of two split numbers is a sum of integer digit products; every digit-pair
// GEMM accumulates exactly in INT32 (127^2 * K * 7 pairs < 2^31 for
// K <= kMaxK), and the pairs with the same t + u = d share one TMEM
// accumulator:
//   C(m, n) = 2^{ea_m + eb_n} sum_{d < S} S_d(m, n) 254^{-(d+2)}.
// Pairs with t + u >= S are dropped (the usual truncation of the scheme); the
// dropped part is below (S+1)/4 * 254^{-S} of 2^{ea+eb} K, 2^-47 at S = 6.
//
// CTA tile: 128 rows x 64 output columns, S accumulators of 64 TMEM columns
// (column block d holds S_d). The B tile of a stage stacks the S slices along
// N (row u*64 + j = slice u, column j), so that one A slice t meets all the B
// slices it pairs with in a single MMA of N = (S - t) * 64 columns (split at
// 256) whose accumulator starts at column block t: pair (t, u) lands in block
// t + u. That is 2S - 1 or fewer MMAs per K step instead of S(S+1)/2 narrow
// ones, and the shared-memory reads per MMA fall accordingly.
//
// Operands arrive pre-tiled (the slicing kernel writes them so): for each
// 128-row block of A and each 32-byte K block, the S slice tiles are one
// contiguous S x 4 KB run in the canonical K-major no-swizzle UMMA layout
// ([slice][16-byte K chunk][row][16 B]); for each 64-column block of B and K
// block, the stacked tile is one contiguous S x 2 KB run
// ([chunk][slice * 64 + column][16 B]). A pipeline stage is therefore two
// bulk copies (cp.async.bulk, no tensor map, no multicast) issued by one
// thread and completing on the stage's mbarrier by transaction count.
//
// Warp roles (320 threads, one persistent CTA per SM): warps 0-7 run the
// epilogue (warp w reads TMEM lanes 32 (w % 4) .. + 31 and half of the tile's
// columns, so that two warps share each lane quarter and the conversion and
// stores of a tile take half as long), one thread of warp 8 issues the MMAs
// and warp 8 owns the TMEM allocation, one thread of warp 9 issues the copies
// into an NSTAGE-deep ring that runs ahead across tiles. Each ring
// slot has a "full" mbarrier (expect-tx arrival plus the copies' bytes) and
// an "empty" mbarrier (tcgen05.commit after the slot's MMAs); acc_full /
// acc_empty hand the accumulators between the MMA thread and the epilogue,
// which releases them as soon as they are in registers and stores while the
// next tile's MMAs run. Every wait is bounded: a timeout sets a shared abort
// flag and *err, the other waiters give up on seeing the flag, and before
// the CTA exits the kernel still waits (bounded) for its issued copies and
// MMAs, freeing its TMEM last.
//
// UMMA descriptors: LBO = distance between the two K chunks, SBO = 128 B
// between 8-row groups. Tiles are rasterised in groups of 8 row blocks, so
// that the CTAs in flight share both their A rows and their B columns in L2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "mbarrier.cuh"

namespace isdf_b200 {
namespace ozaki {

constexpr int BM = 128, BN = 64, BKB = 32;  // tile rows, tile columns, K bytes per stage
constexpr int kTmemCols = 512;
constexpr int kEpiWarps = 8;  // two per TMEM lane quarter, each draining half the columns
constexpr int kThreads = (kEpiWarps + 2) * 32;
constexpr int kGroupM = 8;
constexpr int kSmemLimit = 232448;  // 227 KB per CTA
constexpr int kMaxK = 16384;        // 7 * 127^2 * kMaxK < 2^31
constexpr double kBase = 254.0;
constexpr int kNoExponent = (int)0x80808080;  // byte-fill sentinel: below every ilogb

template <int S>
struct Cfg {
  static constexpr int A_PLANE = BM * BKB;  // bytes of one slice's A tile per stage
  static constexpr int A_STAGE = S * A_PLANE;
  static constexpr int B_ROWS = S * BN;     // stacked B slices
  static constexpr int B_STAGE = B_ROWS * BKB;
  static constexpr int STAGE = A_STAGE + B_STAGE;
  static constexpr int NSTAGE_FIT = (kSmemLimit - 1024) / STAGE;
  static constexpr int NSTAGE = NSTAGE_FIT > 8 ? 8 : NSTAGE_FIT;
  static constexpr int BAR_OFF = NSTAGE * STAGE;
  static constexpr int SMEM = BAR_OFF + (2 * NSTAGE + 3) * 8 + 16;
  static_assert(S * BN <= kTmemCols, "TMEM columns");
  static_assert(NSTAGE >= 2, "shared memory");
  static_assert(SMEM <= kSmemLimit, "shared memory");
};

__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFF);
  d |= (uint64_t)((lbo >> 4) & 0x3FFF) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, no swizzle
}

// kind::i8, D = S32, A = B = signed 8-bit, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(n >> 3) << 17) |
         ((uint32_t)(BM >> 4) << 24);
}

__device__ __forceinline__ void mma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc,
                                       uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
      mbar));
}

// Byte offset of slice t, K chunk c (16 bytes), row r of the tile (block blk,
// K block kb) in the pre-tiled operand layouts above.
template <int S, int R, bool STACKED>
__host__ __device__ __forceinline__ long long tiled_offset(long long blk, int kb, int nkb, int t,
                                                           int c, int r) {
  const long long base = (blk * nkb + kb) * (long long)(S * R * BKB);
  return STACKED ? base + c * (S * R * 16) + (t * R + r) * 16
                 : base + t * (R * BKB) + c * (R * 16) + r * 16;
}

#define ISDF_TMEM_LD16(v, addr)                                                              \
  asm volatile(                                                                              \
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13," \
      "%14,%15}, [%16];\n"                                                                    \
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),  \
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),          \
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15])                                                \
      : "r"(addr))

// 2^e: the bit pattern of a normal power of two (e in [-1022, 1023]), else
// ldexp; the same value either way. The epilogue scales every element by two
// of them, and the library call would cost a large share of its time.
__device__ __forceinline__ double pow2(int e) {
  return (e >= -1022 && e <= 1023) ? __longlong_as_double((long long)(e + 1023) << 52)
                                   : ldexp(1.0, e);
}

// Tile id -> (first row, first column), grouped raster: kGroupM row blocks
// by all column blocks per group.
__device__ __forceinline__ void tile_origin(long long id, int num_m, int num_n, long long* m0,
                                            int* n0) {
  const long long per_group = (long long)kGroupM * num_n;
  const int grp = (int)(id / per_group);
  const int first_m = grp * kGroupM;
  const int gm = min(kGroupM, num_m - first_m);
  const int within = (int)(id - (long long)grp * per_group);
  *m0 = (long long)(first_m + within % gm) * BM;
  *n0 = (within / gm) * BN;
}

// K range of a tile in BKB blocks (triangular B: KMODE 1 keeps k < n0 + BN,
// KMODE 2 keeps k >= n0).
template <int KMODE>
__device__ __forceinline__ void tile_k_range(int n0, int kp, int* kb, int* nk) {
  int b = 0, e = kp;
  if (KMODE == 1) e = min(kp, ((n0 + BN + BKB - 1) / BKB) * BKB);
  if (KMODE == 2) b = (n0 / BKB) * BKB;
  *kb = b;
  *nk = e > b ? (e - b) / BKB : 0;
}

// EPI 0: C = value; 1: C = value^2; 2: C = C * value.
// KMODE 0: full K; 1: B(k, n) = 0 for k > n (upper); 2: B(k, n) = 0 for k < n (lower).
// A, B: pre-tiled slices (tiled_offset<S, 128, false> and <S, 64, true>) over
// ceil(M/128) row blocks and ceil(N/64) column blocks, kp / BKB K blocks, zero
// slices past the true K and the true M, N.
// rowmax (optional, initialised to kNoExponent): atomicMax of ilogb over each
// output row's nonzero values, i.e. the row exponent the next slicing needs.
//
// Persistent: gridDim.x CTAs (one per SM) walk the tiles blockIdx.x,
// blockIdx.x + gridDim.x, ... The copy thread runs ahead across tile
// boundaries; the epilogue warps drain the accumulators into registers,
// release them (acc_empty) and store while the MMA thread already works on
// the next tile.
template <int S, int EPI, int KMODE>
__global__ void __launch_bounds__(kThreads, 1)
    k_ozaki_gemm(const int8_t* __restrict__ A, const int8_t* __restrict__ B,
                 const int* __restrict__ ea, const int* __restrict__ eb, int M, int N, int kp,
                 double* __restrict__ C, long long ldc, int* __restrict__ rowmax,
                 int* __restrict__ err) {
  using Cf = Cfg<S>;
  constexpr int NST = Cf::NSTAGE;
  extern __shared__ __align__(128) uint8_t smem[];
  __shared__ uint32_t tmem_slot;
  __shared__ int abort_flag;
  volatile int* abortp = &abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int num_n = (N + BN - 1) / BN, num_m = (M + BM - 1) / BM;
  const long long tiles = (long long)num_m * num_n;
  const int nkb = kp / BKB;

  const uint32_t sbase = smem_u32(smem);
  const uint32_t bar_base = sbase + Cf::BAR_OFF;
  auto full_bar = [&](int i) { return bar_base + 8u * (uint32_t)i; };
  auto empty_bar = [&](int i) { return bar_base + 8u * (uint32_t)(NST + i); };
  const uint32_t acc_full = bar_base + 8u * (uint32_t)(2 * NST);
  const uint32_t acc_empty = acc_full + 8u;
  const uint32_t done_bar = acc_full + 16u;

  if (warp == kEpiWarps) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     smem_u32(&tmem_slot)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n");
  }
  if (tid == 0) {
    for (int i = 0; i < NST; ++i) {
      mbar_init(full_bar(i), 1);
      mbar_init(empty_bar(i), 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, kEpiWarps * 32);
    mbar_init(done_bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n");
  }
  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;\n");
  const uint32_t tmem = tmem_slot;

  if (warp == kEpiWarps + 1) {
    // ---------------------------------------------------------------- copies
    if (lane == 0) {
      long long g = 0;  // stages issued so far (all tiles)
      bool stop = false;
      for (long long id = blockIdx.x; id < tiles && !stop; id += gridDim.x) {
        long long m0;
        int n0, kb, nk;
        tile_origin(id, num_m, num_n, &m0, &n0);
        tile_k_range<KMODE>(n0, kp, &kb, &nk);
        const int8_t* Ab = A + tiled_offset<S, BM, false>(m0 / BM, kb / BKB, nkb, 0, 0, 0);
        const int8_t* Bb = B + tiled_offset<S, BN, true>(n0 / BN, kb / BKB, nkb, 0, 0, 0);
        for (int t = 0; t < nk; ++t) {
          const int slot = (int)(g % NST);
          if (g >= NST && !mbar_wait(empty_bar(slot), (uint32_t)((g / NST) - 1) & 1u, abortp)) {
            stop = true;
            break;
          }
          const uint32_t st = sbase + slot * Cf::STAGE;
          mbar_expect_tx(full_bar(slot), Cf::STAGE);
          bulk_copy(st, Ab + (long long)t * Cf::A_STAGE, Cf::A_STAGE, full_bar(slot));
          bulk_copy(st + Cf::A_STAGE, Bb + (long long)t * Cf::B_STAGE, Cf::B_STAGE,
                    full_bar(slot));
          ++g;
        }
      }
      // no copy may still be landing when the CTA exits: wait (bounded) for
      // the last stage issued into each slot
      for (long long t = g > NST ? g - NST : 0; t < g; ++t)
        if (!mbar_wait_all(full_bar((int)(t % NST)), (uint32_t)(t / NST) & 1u)) *abortp = 1;
    }
    __syncwarp();
  } else if (warp == kEpiWarps) {
    // ---------------------------------------------------------------- MMA issue
    if (lane == 0) {
      long long g = 0;
      int it = 0;
      bool stop = false;
      for (long long id = blockIdx.x; id < tiles; id += gridDim.x, ++it) {
        long long m0;
        int n0, kb, nk;
        tile_origin(id, num_m, num_n, &m0, &n0);
        tile_k_range<KMODE>(n0, kp, &kb, &nk);
        // the epilogue must have drained the previous tile's accumulators
        if (it > 0 && !mbar_wait(acc_empty, (uint32_t)(it - 1) & 1u, abortp)) stop = true;
        asm volatile("tcgen05.fence::after_thread_sync;\n");
        for (int t = 0; t < nk && !stop; ++t) {
          const int slot = (int)(g % NST);
          if (!mbar_wait(full_bar(slot), (uint32_t)(g / NST) & 1u, abortp)) {
            stop = true;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;\n");
          const uint32_t sa = sbase + slot * Cf::STAGE;
          const uint32_t sb = sa + S * Cf::A_PLANE;
#pragma unroll
          for (int ta = 0; ta < S; ++ta) {
            const uint64_t ad = umma_desc(sa + ta * Cf::A_PLANE, BM * 16, 128);
            const uint32_t acc = (t > 0 || ta > 0) ? 1u : 0u;
#pragma unroll
            for (int r0 = 0; r0 < (S - ta) * BN; r0 += 256) {
              const int n = (S - ta) * BN - r0 < 256 ? (S - ta) * BN - r0 : 256;
              const uint64_t bd = umma_desc(sb + r0 * 16, Cf::B_ROWS * 16, 128);
              mma_i8(tmem + (uint32_t)(ta * BN + r0), ad, bd, idesc_i8(n), acc);
            }
          }
          mma_commit(empty_bar(slot));
          ++g;
        }
        // this tile's accumulators (committed also after an abort, so that
        // the epilogue's wait for them ends)
        mma_commit(acc_full);
        if (stop) break;
      }
      // every MMA issued above has completed before the TMEM is freed
      mma_commit(done_bar);
      if (!mbar_wait_all(done_bar, 0)) *abortp = 1;
    }
    __syncwarp();
  } else {
    // ---------------------------------------------------------------- epilogue
    // warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows) and columns
    // [ (w / 4) CW, + CW )
    constexpr int CW = BN / (kEpiWarps / 4);
    const int q = warp & 3, c_lo = (warp >> 2) * CW;
    double w[S];  // 254^{-(d+2)}
    w[0] = 1.0 / (kBase * kBase);
#pragma unroll
    for (int d = 1; d < S; ++d) w[d] = w[d - 1] / kBase;
    int it = 0;
    for (long long id = blockIdx.x; id < tiles; id += gridDim.x, ++it) {
      long long m0;
      int n0, kb, nk;
      tile_origin(id, num_m, num_n, &m0, &n0);
      tile_k_range<KMODE>(n0, kp, &kb, &nk);
      bool ready = mbar_wait(acc_full, (uint32_t)it & 1u, abortp) && *abortp == 0;
      if (!__all_sync(0xffffffffu, ready)) break;  // warp-uniform: tcgen05.ld is collective
      asm volatile("tcgen05.fence::after_thread_sync;\n");
      const int row = q * 32 + lane;
      const long long m = m0 + row;
      const uint32_t lane_base = tmem + ((uint32_t)(q * 32) << 16);
      double out[CW];
#pragma unroll
      for (int j = 0; j < CW; ++j) out[j] = 0.0;
      if (nk > 0) {
        // 16 columns per TMEM round trip, two levels at a time; per column the
        // levels accumulate in order d = 0, 1, ...
#pragma unroll
        for (int c0 = 0; c0 < CW; c0 += 16) {
#pragma unroll
          for (int d = 0; d < S; d += 2) {
            uint32_t va[16], vb[16];
            ISDF_TMEM_LD16(va, lane_base + (uint32_t)(d * BN + c_lo + c0));
            if (d + 1 < S) ISDF_TMEM_LD16(vb, lane_base + (uint32_t)((d + 1) * BN + c_lo + c0));
            asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
#pragma unroll
            for (int j = 0; j < 16; ++j) {
              out[c0 + j] = __fma_rn((double)(int)va[j], w[d], out[c0 + j]);
              if (d + 1 < S)
                out[c0 + j] = __fma_rn((double)(int)vb[j], w[d + 1], out[c0 + j]);
            }
          }
        }
      }
      // accumulators drained: the MMA thread may start the next tile
      asm volatile("tcgen05.fence::before_thread_sync;\n");
      mbar_arrive(acc_empty);
      if (m < M) {
        const double sa = pow2(ea[m]);
        double amax = 0.0;
#pragma unroll
        for (int j = 0; j < CW; ++j) {
          const int n = n0 + c_lo + j;
          if (n < N) {
            const double val = out[j] * sa * pow2(eb[n]);
            double* p = C + m + (long long)n * ldc;
            double r;
            if (EPI == 0) r = val;
            else if (EPI == 1) r = val * val;
            else r = *p * val;
            *p = r;
            amax = fmax(amax, fabs(r));
          }
        }
        // the row's largest binade, for slicing this output as the next A operand
        if (rowmax && amax > 0.0) atomicMax(&rowmax[m], ilogb(amax));
      }
    }
  }

  asm volatile("tcgen05.fence::before_thread_sync;\n");
  __syncthreads();
  if (*abortp != 0 && tid == 0) atomicExch(err, 1);
  if (warp == kEpiWarps) {
    asm volatile("tcgen05.fence::after_thread_sync;\n");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kTmemCols));
  }
}

#undef ISDF_TMEM_LD16

}  // namespace ozaki
}  // namespace isdf_b200
