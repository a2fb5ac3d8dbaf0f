// QRCP interpolation-point selection on sm_100a.
//
// Reference: src/cpu/getpoints_QRCP.cpp:11-500 (CPU only; the reference's GPU
// entry point has no selector). Same algorithm:
//   numPre = IRound(sqrt(mu * f)), f = 1.5 in the reference   (:82-86)
//   G1, G2 = srand48(seed) Gaussian draws, orthonormal columns (:143-189)
//   A = psi_S1 G1, B = psi_S2 G2 (Ng x numPre)                (:201-207)
//   MG(i + j*numPre, r) = B(r, i) A(r, j); column norms        (:228-235)
//   keep columns with norm^2 > 1e-5 * max                      (:272-284)
//   column-pivoted QR of the kept columns; piv = MGIdx[pivots] (:440-457)
//
// B200 form. MG (numPre^2 x Ng: 19.5 GB at Si64 with f = 2.5) is never
// stored. Column-pivoted Householder QR picks, at every step, the column with
// the largest residual norm; that is the same sequence as pivoted Gram-Schmidt
// on the columns x_r = vec(B_r (x) A_r). Step k:
//   * pick the first column (in the current pivoted order) of maximal
//     residual norm, swap positions as the LAPACK routine does;
//   * q_k = x_pk orthogonalised against q_0..q_{k-1} (two passes), normalised;
//   * every residual norm is downdated with t_r = q_k . x_r, which is
//     t_r = sum_j A(r, j) (B_r Qm)_j, Qm(i, j) = q_k[i + j*numPre]: one
//     FP64 tensor-core tile GEMM over all columns with the row dot fused into
//     its epilogue, and the multiplicative downdate of LAPACK's dgeqpf,
//     nu <- nu sqrt(max(0, 1 - (t/nu)^2));
//   * where dgeqpf's cancellation test fires (LAPACK Working Note 176:
//     temp (nu / nu_ref)^2 <= sqrt(eps), eps = 2^-53), the downdated value is
//     not used: dgeqpf then recomputes the norm of the column's transformed
//     trailing part, i.e. of its residual after the k+1 projections; here
//     that residual is formed from the column's features (projected on
//     q_0..q_k twice) and its norm becomes both nu and the new reference nu_ref.
// Orthonormalising G by Householder QR instead of the reference's dgesvd
// changes G1, G2 by orthogonal factors: MG changes by an orthogonal matrix on
// its left, which leaves the column norms and the pivot sequence unchanged.
#include <mutex>
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "arena.h"
#include "common.cuh"
#include "dgemm.cuh"
#include "fit.h"
#include "readback.h"
#include "qrcp.h"
#include "solve.h"

namespace isdf_b200 {

namespace {

constexpr int kMaxPre = 128;  // numPre limit: one 128-wide tile holds every column of Qm

struct QrState {
  unsigned long long maxbits;  // max residual norm of the active columns (bit pattern)
  int minpos;                  // first position holding that maximum
  int done;
  int nrec;                    // columns flagged for a norm recompute in this step
  int ntot;
  int total_rec;               // norms recomputed over the whole selection
  int pad;
};

// dgeqpf's recompute threshold sqrt(eps), eps = dlamch('Epsilon') = 2^-53.
__device__ __forceinline__ double tol3z() { return sqrt(1.1102230246251565e-16); }

// The downdate of one active column's residual norm with t = q_k . x_c, as
// dgeqpf does it. Returns false (and lists the column) where the cancellation
// test fires: that column's norm is recomputed exactly after this kernel.
__device__ __forceinline__ bool downdate_norm(int c, double t, double* __restrict__ nu,
                                              const double* __restrict__ nu0, QrState* st,
                                              int* __restrict__ rec_list) {
  const double v = nu[c];
  if (v == 0.0) return true;
  const double ratio = fabs(t) / v;
  const double temp = fmax(1.0 - ratio * ratio, 0.0);
  const double rel = v / nu0[c];
  if (temp * rel * rel <= tol3z()) {
    rec_list[atomicAdd(&st->nrec, 1)] = c;
    return false;
  }
  nu[c] = v * sqrt(temp);
  return true;
}

// ------------------------------------------------------------- norms, filter
// Squared MG column norm per grid point, summed j-outer, i-inner with
// explicit rounding as the reference's loop (getpoints_QRCP.cpp:228-235).
__global__ void k_mg_norm(const double* __restrict__ A, const double* __restrict__ B, long long n,
                          int p, double* __restrict__ norm2, QrState* st) {
  double mx = 0.0;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < n;
       r += (long long)gridDim.x * blockDim.x) {
    double s = 0.0;
    for (int j = 0; j < p; ++j) {
      const double a = A[r + (long long)j * n];
      for (int i = 0; i < p; ++i) {
        const double mg = rmul(B[r + (long long)i * n], a);
        s = radd(s, rmul(mg, mg));
      }
    }
    norm2[r] = s;
    mx = fmax(mx, s);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.0)
    atomicMax(&st->maxbits, (unsigned long long)__double_as_longlong(mx));
}

__global__ void __launch_bounds__(256) k_keep_count(const double* __restrict__ norm2, long long n,
                                                    const QrState* st, int* tile_cnt) {
  const double thr = rmul(__longlong_as_double((long long)st->maxbits), 1e-5);
  __shared__ int wc[8];
  const long long base = (long long)blockIdx.x * 1024;
  int c = 0;
  for (int k = 0; k < 4; ++k) {
    const long long i = base + k * 256 + threadIdx.x;
    if (i < n && norm2[i] > thr) ++c;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) wc[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; ++w) t += wc[w];
    tile_cnt[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_scan_tiles(int* cnt, int ntiles, int* total) {
  __shared__ int part[1024];
  const int per = (ntiles + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, ntiles);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    const int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    const int v = cnt[i];
    cnt[i] = run;
    run += v;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

__global__ void __launch_bounds__(256) k_keep_scatter(const double* __restrict__ norm2, long long n,
                                                      const QrState* st, const int* tile_off,
                                                      int* __restrict__ idx) {
  const double thr = rmul(__longlong_as_double((long long)st->maxbits), 1e-5);
  __shared__ int wc[8][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const long long base = (long long)blockIdx.x * 1024;
  unsigned bal[4];
  for (int k = 0; k < 4; ++k) {
    const long long i = base + k * 256 + threadIdx.x;
    bal[k] = __ballot_sync(0xffffffffu, i < n && norm2[i] > thr);
    if (lane == 0) wc[wid][k] = __popc(bal[k]);
  }
  __syncthreads();
  const int off = tile_off[blockIdx.x];
  for (int k = 0; k < 4; ++k) {
    int before = 0;
    for (int kk = 0; kk < k; ++kk)
      for (int w = 0; w < 8; ++w) before += wc[w][kk];
    for (int w = 0; w < wid; ++w) before += wc[w][k];
    if (bal[k] & (1u << lane))
      idx[off + before + __popc(bal[k] & ((1u << lane) - 1u))] = (int)(base + k * 256 + threadIdx.x);
  }
}

// Compacted operands Ac, Bc (ntot x p, column-major with an even leading
// dimension ld = ntot rounded up, the padding row zero, so that every column
// starts on a 16-byte boundary), residual norms, order.
__global__ void k_compact(const double* __restrict__ A, const double* __restrict__ B, long long n,
                          int p, const int* __restrict__ idx, const double* __restrict__ norm2,
                          QrState* st, double* __restrict__ Ac, double* __restrict__ Bc,
                          double* __restrict__ nu, double* __restrict__ nu0, int* __restrict__ pos,
                          int* __restrict__ perm, unsigned char* __restrict__ active) {
  const int ntot = st->ntot;
  const long long ld = ntot + (ntot & 1);
  if ((ntot & 1) && blockIdx.x == 0 && threadIdx.x == 0)
    for (int j = 0; j < p; ++j) Ac[ntot + j * ld] = Bc[ntot + j * ld] = 0.0;
  double mx = 0.0;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ntot; c += gridDim.x * blockDim.x) {
    const long long r = idx[c];
    for (int j = 0; j < p; ++j) {
      Ac[c + j * ld] = A[r + (long long)j * n];
      Bc[c + j * ld] = B[r + (long long)j * n];
    }
    const double v = sqrt(norm2[r]);
    nu[c] = v;
    nu0[c] = v;
    pos[c] = c;
    perm[c] = c;
    active[c] = 1;
    mx = fmax(mx, v);
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.0)
    atomicMax(&st->maxbits, (unsigned long long)__double_as_longlong(mx));
}

__global__ void k_reset_max(QrState* st) {
  st->maxbits = 0ull;
  st->minpos = INT_MAX;
}

// ------------------------------------------------------------- one pivot step
// First position (in the pivoted order) holding the maximal residual norm, as
// LAPACK's idamax over the remaining columns picks it.
__global__ void k_argpos(const double* __restrict__ nu, const int* __restrict__ pos,
                         const unsigned char* __restrict__ active, int ntot, QrState* st) {
  if (st->done) return;
  const double mx = __longlong_as_double((long long)st->maxbits);
  int best = INT_MAX;
  for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < ntot; c += gridDim.x * blockDim.x)
    if (active[c] && nu[c] == mx) best = min(best, pos[c]);
  for (int o = 16; o > 0; o >>= 1) best = min(best, __shfl_xor_sync(0xffffffffu, best, o));
  if ((threadIdx.x & 31) == 0 && best != INT_MAX) atomicMin(&st->minpos, best);
}

// Pivot bookkeeping (one thread) and the pivot's feature vector
// x[i + j*p] = B(c, i) * A(c, j).
__global__ void k_pick(int k, int p, int ld, const double* __restrict__ Ac,
                       const double* __restrict__ Bc, int* __restrict__ pos,
                       int* __restrict__ perm, unsigned char* __restrict__ active,
                       int* __restrict__ sel, QrState* st, double* __restrict__ x) {
  __shared__ int col;
  if (threadIdx.x == 0) {
    col = -1;
    const double mx = __longlong_as_double((long long)st->maxbits);
    if (!st->done && mx > 0.0 && st->minpos != INT_MAX) {
      const int q = st->minpos;
      const int c = perm[q];
      const int ck = perm[k];
      perm[k] = c;
      perm[q] = ck;
      pos[ck] = q;
      pos[c] = k;
      active[c] = 0;
      sel[k] = c;
      col = c;
    } else {
      st->done = 1;
    }
    st->maxbits = 0ull;
    st->minpos = INT_MAX;
    st->nrec = 0;
  }
  __syncthreads();
  if (col < 0) return;
  const int m = p * p;
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const int i = e % p, j = e / p;
    x[e] = Bc[col + (long long)i * ld] * Ac[col + (long long)j * ld];
  }
}

// cdot[l] = Q[:, l] . x for l < k: one block per l (a strided partial per
// thread, then a fixed-order tree), so the sums do not depend on scheduling.
__global__ void __launch_bounds__(256) k_qt_x(const double* __restrict__ Q, int m, int k,
                                              const double* __restrict__ x, const QrState* st,
                                              double* __restrict__ cdot) {
  if (st->done) return;
  const int l = blockIdx.x;
  if (l >= k) return;
  __shared__ double red[8];
  const double* q = Q + (long long)l * m;
  double s = 0.0;
#pragma unroll 4
  for (int i = threadIdx.x; i < m; i += 256) s = fma(q[i], x[i], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = red[0];
    for (int w = 1; w < 8; ++w) v += red[w];
    cdot[l] = v;
  }
}

// x -= Q[:, 0:k] cdot: a block takes 32 consecutive rows (one per lane), its
// 32 warps the columns l = w (mod 32), and the 32 partials are added in warp
// order (enough loads in flight per SM to stream Q from L2).
__global__ void __launch_bounds__(1024) k_x_minus_qc(const double* __restrict__ Q, int m, int k,
                                                     const double* __restrict__ cdot,
                                                     const QrState* st, double* __restrict__ x) {
  if (st->done) return;
  __shared__ double red[32][33];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int i = blockIdx.x * 32 + lane;
  double s = 0.0;
  if (i < m) {
#pragma unroll 4
    for (int l = w; l < k; l += 32) s = fma(Q[i + (long long)l * m], cdot[l], s);
  }
  red[w][lane] = s;
  __syncthreads();
  if (w == 0 && i < m) {
    double v = red[0][lane];
    for (int u = 1; u < 32; ++u) v += red[u][lane];
    x[i] -= v;
  }
}

// q_k = x / |x| into Q[:, k] and into Qm (depth-major: Qm[i*p + j] = q[i + j*p]).
__global__ void __launch_bounds__(1024) k_normalise(int k, int p, const double* __restrict__ x,
                                                    QrState* st, double* __restrict__ Q,
                                                    double* __restrict__ Qm) {
  if (st->done) return;
  const int m = p * p;
  __shared__ double red[32];
  double s = 0.0;
  for (int e = threadIdx.x; e < m; e += blockDim.x) s = fma(x[e], x[e], s);
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) red[0] = v;
  }
  __syncthreads();
  const double nrm = sqrt(red[0]);
  if (!(nrm > 0.0)) {
    if (threadIdx.x == 0) st->done = 1;
    return;
  }
  const double inv = 1.0 / nrm;
  for (int e = threadIdx.x; e < m; e += blockDim.x) {
    const double q = x[e] * inv;
    Q[(long long)k * m + e] = q;
    const int i = e % p, j = e / p;
    Qm[i * p + j] = q;
  }
}

// Residual-norm downdate of every active column with t_c = q_k . x_c, and the
// maximum of the new norms for the next step.
using CoreU = dmma::Core<128, 128>;
template <int VEC>
__global__ void __launch_bounds__(256) k_update(const double* __restrict__ Ac,
                                                const double* __restrict__ Bc, int ntot, int ld,
                                                int p,
                                                const double* __restrict__ Qm,
                                                const unsigned char* __restrict__ active,
                                                double* __restrict__ nu,
                                                double* __restrict__ nu0, QrState* st,
                                                int* __restrict__ rec_list) {
  if (st->done) return;
  extern __shared__ double smem[];
  const int m0 = blockIdx.x * CoreU::BM;
  const int m_rem = min(CoreU::BM, ntot - m0);
  CoreU core;
  core.zero();
  core.run<VEC>(smem, Bc + m0, ld, Qm, p, m_rem, p, 0, p);
  // row dot with A, reduced over the 4 lanes of a quad and the 4 column warps
  double* red = smem;  // [4][128], the pipeline buffers are free again
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm0 = (warp >> 2) * CoreU::WM, wn0 = (warp & 3) * CoreU::WN;
#pragma unroll
  for (int i = 0; i < CoreU::MT; ++i) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int r = wm0 + i * 16 + g + 8 * h;
      double s = 0.0;
      if (r < m_rem) {
#pragma unroll
        for (int j = 0; j < CoreU::NT; ++j) {
          const int c = wn0 + j * 8 + 2 * t;
          if (c < p) s = fma(Ac[(m0 + r) + (long long)c * ld], core.acc[i][j][2 * h], s);
          if (c + 1 < p) s = fma(Ac[(m0 + r) + (long long)(c + 1) * ld], core.acc[i][j][2 * h + 1], s);
        }
      }
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      if (t == 0) red[(warp & 3) * CoreU::BM + r] = s;
    }
  }
  __syncthreads();
  double mx = 0.0;
  if (threadIdx.x < CoreU::BM && (int)threadIdx.x < m_rem) {
    const int c = m0 + threadIdx.x;
    if (active[c]) {
      const double tdot = red[threadIdx.x] + red[CoreU::BM + threadIdx.x] +
                          red[2 * CoreU::BM + threadIdx.x] + red[3 * CoreU::BM + threadIdx.x];
      if (downdate_norm(c, tdot, nu, nu0, st, rec_list)) mx = nu[c];
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if ((threadIdx.x & 31) == 0 && mx > 0.0)
    atomicMax(&st->maxbits, (unsigned long long)__double_as_longlong(mx));
}

// The same downdate on the warp-specialised tile (16-byte aligned Bc and Qm,
// p even; the even leading dimension lets the last odd row copy its zero
// padding partner): 64 rows x BN columns, BN = p rounded up to a multiple of
// 8 (the columns past p copied as zeros), four DMMA warps of 16 full rows
// each, so the row dot with A closes inside a quad of lanes. BN tracks p
// instead of a fixed 128-wide tile: at most 7 padding columns take
// tensor-core work.
template <int BN>
using UpdTile = dmma::WsTile<64, BN, 4, 1, 16, 3>;
// three CTAs per SM while the accumulators leave room (136 registers)
template <int BN>
struct UpdMinBlocks {
  static constexpr int value = BN <= 96 ? 3 : 2;
};

template <int BN, int MINB>
__global__ void __launch_bounds__(UpdTile<BN>::THREADS, MINB)
    k_update_ws(const double* __restrict__ Ac, const double* __restrict__ Bc, int ntot, int ld,
                int p,
                const double* __restrict__ Qm, const unsigned char* __restrict__ active,
                double* __restrict__ nu, double* __restrict__ nu0, QrState* st,
                int* __restrict__ rec_list, int* err) {
  using T = UpdTile<BN>;
  if (st->done) return;
  extern __shared__ __align__(128) double smem[];
  const int m0 = blockIdx.x * T::BM;
  const int m_rem = min(T::BM, ntot - m0);
  T tile;
  if (!tile.run(smem, Bc + m0, ld, (m_rem + 1) & ~1, Qm, p, p, p, err)) return;
  if (T::producer()) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  double mx = 0.0;
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int r = warp * 16 + g + 8 * h;
    double s = 0.0;
    if (r < m_rem) {
#pragma unroll
      for (int j = 0; j < T::NT; ++j) {
        const int c = j * 8 + 2 * t;
        if (c < p) s = fma(Ac[(m0 + r) + (long long)c * ld], tile.acc[0][j][2 * h], s);
        if (c + 1 < p) s = fma(Ac[(m0 + r) + (long long)(c + 1) * ld], tile.acc[0][j][2 * h + 1], s);
      }
    }
    s += __shfl_xor_sync(0xffffffffu, s, 1);
    s += __shfl_xor_sync(0xffffffffu, s, 2);
    if (t == 0 && r < m_rem) {
      const int c = m0 + r;
      if (active[c] && downdate_norm(c, s, nu, nu0, st, rec_list)) mx = fmax(mx, nu[c]);
    }
  }
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0 && mx > 0.0)
    atomicMax(&st->maxbits, (unsigned long long)__double_as_longlong(mx));
}

// Exact residual norms of the columns the downdate flagged in this step
// (dgeqpf's recompute). One CTA per flagged column at a time: the column's
// features x[i + j*p] = B(c, i) A(c, j) go to shared memory, are projected
// on q_0..q_k twice (classical Gram-Schmidt: all k+1 dots, one warp per q_l
// with a fixed lane order, then the update, one thread per feature summing
// over l in order), and the residual's norm becomes nu[c] and the new
// reference nu0[c]. cbuf: gridDim.x x k1 doubles of scratch for the dots.
constexpr int kRecomputeGrid = 148;
__global__ void __launch_bounds__(256) k_recompute(const double* __restrict__ Ac,
                                                   const double* __restrict__ Bc, int ld, int p,
                                                   const double* __restrict__ Q, int m, int k1,
                                                   const int* __restrict__ rec_list,
                                                   double* __restrict__ nu,
                                                   double* __restrict__ nu0, QrState* st,
                                                   double* __restrict__ cbuf) {
  extern __shared__ double x[];  // m features
  __shared__ double red[8];
  if (st->done) return;
  const int nrec = st->nrec;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* c = cbuf + (size_t)blockIdx.x * k1;
  for (int f = blockIdx.x; f < nrec; f += gridDim.x) {
    const int col = rec_list[f];
    for (int e = threadIdx.x; e < m; e += 256) {
      const int i = e % p, j = e / p;
      x[e] = Bc[col + (long long)i * ld] * Ac[col + (long long)j * ld];
    }
    __syncthreads();
    for (int pass = 0; pass < 2; ++pass) {
      for (int l = warp; l < k1; l += 8) {
        const double* q = Q + (long long)l * m;
        double s = 0.0;
        for (int i = lane; i < m; i += 32) s = fma(q[i], x[i], s);
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) c[l] = s;
      }
      __syncthreads();
      for (int i = threadIdx.x; i < m; i += 256) {
        double s = 0.0;
        for (int l = 0; l < k1; ++l) s = fma(Q[(long long)l * m + i], c[l], s);
        x[i] -= s;
      }
      __syncthreads();
    }
    double s = 0.0;
    for (int i = threadIdx.x; i < m; i += 256) s = fma(x[i], x[i], s);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) red[warp] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += red[w];
      const double v = sqrt(t);
      nu[col] = v;
      nu0[col] = v;
      if (v > 0.0) atomicMax(&st->maxbits, (unsigned long long)__double_as_longlong(v));
      atomicAdd(&st->total_rec, 1);
    }
    __syncthreads();
  }
}

// Householder QR of the K x p draws (host, FP64): returns p orthonormal columns
// spanning the same space, row-major (K x p) for the depth-major GEMM operand.
std::vector<double> orthonormal_rows(const std::vector<double>& g_colmajor, int K, int p) {
  std::vector<double> a = g_colmajor;  // column-major K x p
  std::vector<double> tau(p, 0.0);
  for (int j = 0; j < p; ++j) {
    double nrm = 0.0;
    for (int i = j; i < K; ++i) nrm += a[i + (size_t)j * K] * a[i + (size_t)j * K];
    nrm = std::sqrt(nrm);
    const double a0 = a[j + (size_t)j * K];
    const double beta = a0 >= 0 ? -nrm : nrm;
    if (nrm == 0.0) continue;
    const double v0 = a0 - beta;
    for (int i = j + 1; i < K; ++i) a[i + (size_t)j * K] /= v0;
    tau[j] = (beta - a0) / beta;
    a[j + (size_t)j * K] = beta;
    for (int c = j + 1; c < p; ++c) {
      double s = a[j + (size_t)c * K];
      for (int i = j + 1; i < K; ++i) s += a[i + (size_t)j * K] * a[i + (size_t)c * K];
      s *= tau[j];
      a[j + (size_t)c * K] -= s;
      for (int i = j + 1; i < K; ++i) a[i + (size_t)c * K] -= s * a[i + (size_t)j * K];
    }
  }
  // Q = H_0 ... H_{p-1} I[:, 0:p]
  std::vector<double> q((size_t)K * p, 0.0);
  for (int j = 0; j < p; ++j) q[j + (size_t)j * K] = 1.0;
  for (int j = p - 1; j >= 0; --j) {
    for (int c = 0; c < p; ++c) {
      double s = q[j + (size_t)c * K];
      for (int i = j + 1; i < K; ++i) s += a[i + (size_t)j * K] * q[i + (size_t)c * K];
      s *= tau[j];
      q[j + (size_t)c * K] -= s;
      for (int i = j + 1; i < K; ++i) q[i + (size_t)c * K] -= s * a[i + (size_t)j * K];
    }
  }
  std::vector<double> rows((size_t)K * p);
  for (int i = 0; i < K; ++i)
    for (int j = 0; j < p; ++j) rows[(size_t)i * p + j] = q[i + (size_t)j * K];
  return rows;
}

// srand48 Gaussian draws as include/common/utility.hpp:455-471: column-major.
std::vector<double> gaussian_draws(int m, int n) {
  std::vector<double> g((size_t)m * n);
  const double pi = 3.14159265358979323846;
  for (auto& v : g) {
    const double a = drand48(), b = drand48();
    v = std::sqrt(-2.0 * std::log(a)) * std::cos(2.0 * pi * b);
  }
  return g;
}

struct QrBuffers {
  double *A, *B, *norm2, *Ac, *Bc, *nu, *nu0, *Q, *Qm, *x, *cdot, *G1, *G2, *rec_dots;
  int *idx, *pos, *perm, *sel, *tile_cnt, *rec_list;
  unsigned char* active;
  QrState* st;
  int* err;  // a bounded pipeline wait of the update ran out
};

QrBuffers carve(Arena& a, long long n, int p, int k1, int k2, int kmax) {
  QrBuffers b;
  const int m = p * p;
  const int ntiles = (int)((n + 1023) / 1024);
  b.A = a.take<double>((size_t)n * p);
  b.B = a.take<double>((size_t)n * p);
  b.norm2 = a.take<double>((size_t)n);
  b.Ac = a.take<double>((size_t)(n + 1) * p);  // leading dimension up to n + 1 (even)
  b.Bc = a.take<double>((size_t)(n + 1) * p);
  b.nu = a.take<double>((size_t)n);
  b.nu0 = a.take<double>((size_t)n);
  b.Q = a.take<double>((size_t)m * kmax);
  b.Qm = a.take<double>((size_t)m);
  b.x = a.take<double>((size_t)m);
  b.cdot = a.take<double>((size_t)kmax);
  b.G1 = a.take<double>((size_t)k1 * p);
  b.G2 = a.take<double>((size_t)k2 * p);
  b.idx = a.take<int>((size_t)n);
  b.pos = a.take<int>((size_t)n);
  b.perm = a.take<int>((size_t)n);
  b.sel = a.take<int>((size_t)kmax);
  b.tile_cnt = a.take<int>((size_t)ntiles);
  b.rec_list = a.take<int>((size_t)n);
  b.rec_dots = a.take<double>((size_t)kRecomputeGrid * kmax);
  b.active = a.take<unsigned char>((size_t)n);
  b.st = a.take<QrState>(1);
  b.err = a.take<int>(1);
  return b;
}

int set_update_attrs() {
  std::lock_guard<std::mutex> attr_lock(attr_mutex());
  static bool done[64] = {};
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done[dev]) return ISDF_OK;
  ISDF_CUDA(cudaFuncSetAttribute(k_update<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)CoreU::SMEM_BYTES));
  ISDF_CUDA(cudaFuncSetAttribute(k_recompute, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(double) * kMaxPre * kMaxPre)));
#define ISDF_UPD_ATTR(BN)                                                                  \
  ISDF_CUDA(cudaFuncSetAttribute(k_update_ws<BN, UpdMinBlocks<BN>::value>,                   \
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,                \
                                 (int)UpdTile<BN>::SMEM_BYTES))
  ISDF_UPD_ATTR(16);
  ISDF_UPD_ATTR(24);
  ISDF_UPD_ATTR(32);
  ISDF_UPD_ATTR(40);
  ISDF_UPD_ATTR(48);
  ISDF_UPD_ATTR(56);
  ISDF_UPD_ATTR(64);
  ISDF_UPD_ATTR(72);
  ISDF_UPD_ATTR(80);
  ISDF_UPD_ATTR(88);
  ISDF_UPD_ATTR(96);
  ISDF_UPD_ATTR(104);
  ISDF_UPD_ATTR(112);
  ISDF_UPD_ATTR(120);
  ISDF_UPD_ATTR(128);
#undef ISDF_UPD_ATTR
  if (dev >= 0 && dev < 64) done[dev] = true;
  return ISDF_OK;
}

template <int BN>
void launch_update_bn(const QrBuffers& b, int ntot, int ld, int p, cudaStream_t s) {
  using T = UpdTile<BN>;
  const unsigned grid = (unsigned)((ntot + T::BM - 1) / T::BM);
  k_update_ws<BN, UpdMinBlocks<BN>::value><<<grid, T::THREADS, T::SMEM_BYTES, s>>>(
      b.Ac, b.Bc, ntot, ld, p, b.Qm, b.active, b.nu, b.nu0, b.st, b.rec_list, b.err);
}

// The downdate on the narrowest warp-specialised tile that holds p columns
// (p rounded up to a multiple of 8).
void launch_update_ws(const QrBuffers& b, int ntot, int ld, int p, cudaStream_t s) {
  switch ((p + 7) / 8) {
    case 0: case 1: case 2: launch_update_bn<16>(b, ntot, ld, p, s); break;
    case 3: launch_update_bn<24>(b, ntot, ld, p, s); break;
    case 4: launch_update_bn<32>(b, ntot, ld, p, s); break;
    case 5: launch_update_bn<40>(b, ntot, ld, p, s); break;
    case 6: launch_update_bn<48>(b, ntot, ld, p, s); break;
    case 7: launch_update_bn<56>(b, ntot, ld, p, s); break;
    case 8: launch_update_bn<64>(b, ntot, ld, p, s); break;
    case 9: launch_update_bn<72>(b, ntot, ld, p, s); break;
    case 10: launch_update_bn<80>(b, ntot, ld, p, s); break;
    case 11: launch_update_bn<88>(b, ntot, ld, p, s); break;
    case 12: launch_update_bn<96>(b, ntot, ld, p, s); break;
    case 13: launch_update_bn<104>(b, ntot, ld, p, s); break;
    case 14: launch_update_bn<112>(b, ntot, ld, p, s); break;
    case 15: launch_update_bn<120>(b, ntot, ld, p, s); break;
    default: launch_update_bn<128>(b, ntot, ld, p, s); break;
  }
}

}  // namespace

int qrcp_num_pre(int mu, double factor) { return iround(std::sqrt(mu * factor)); }

size_t qrcp_workspace_bytes(long long ng, int nstate, int mu, double factor) {
  const int p = qrcp_num_pre(mu, factor);
  Arena a;
  a.counting = true;
  carve(a, ng, p, nstate, nstate, std::min(mu, p * p));
  return a.off;
}

int qrcp_select(const QrcpArgs& args, Arena& arena, cudaStream_t s, QrcpResult* res) {
  const long long n = args.ng;
  const int p = qrcp_num_pre(args.mu, args.factor);
  const int k1 = args.nv1 + args.nc1, k2 = args.nv2 + args.nc2;
  if (p > args.nstate)
    return record_error(ISDF_ERR_ARG,
                        "numMu is too large for interpolative separable density fitting!");
  if ((long long)p * p > n)
    return record_error(ISDF_ERR_ARG, "numPre*numPre > ntot. The number of grid points is perhaps too small!");
  if (p > k1 || p > k2)
    return record_error(ISDF_ERR_UNSUPPORTED, "QRCP: numPre exceeds a state window");
  if (p > kMaxPre) return record_error(ISDF_ERR_UNSUPPORTED, "QRCP: numPre above 128");
  if (n > 0x7fffffffLL) return record_error(ISDF_ERR_UNSUPPORTED, "QRCP: Ng >= 2^31");
  const int m = p * p;
  const int kmax_cap = std::min(args.mu, m);
  QrBuffers b = carve(arena, n, p, k1, k2, kmax_cap);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "QRCP: workspace too small");
  ISDF_TRY(set_update_attrs());
  int launches = 0;

  // sketch (host): srand48(seed), G1 then G2, orthonormal columns
  srand48((long)args.seed);
  std::vector<double> g1 = gaussian_draws(k1, p);
  std::vector<double> g2 = gaussian_draws(k2, p);
  std::vector<double> q1 = orthonormal_rows(g1, k1, p);
  std::vector<double> q2 = orthonormal_rows(g2, k2, p);
  ISDF_CUDA(cudaMemcpyAsync(b.G1, q1.data(), sizeof(double) * q1.size(), cudaMemcpyHostToDevice, s));
  ISDF_CUDA(cudaMemcpyAsync(b.G2, q2.data(), sizeof(double) * q2.size(), cudaMemcpyHostToDevice, s));
  ISDF_CUDA(cudaMemsetAsync(b.st, 0, sizeof(QrState), s));
  ISDF_CUDA(cudaMemsetAsync(b.err, 0, sizeof(int), s));

  // A = psi_S1 G1, B = psi_S2 G2
  ISDF_TRY(dgemm_store((int)n, p, k1, args.d_psi + (long long)(args.nocc - args.nv1) * n, n, b.G1,
                       p, b.A, n, s));
  ISDF_TRY(dgemm_store((int)n, p, k2, args.d_psi + (long long)(args.nocc - args.nv2) * n, n, b.G2,
                       p, b.B, n, s));
  launches += 2;

  // norms, filter, compaction
  const int ntiles = (int)((n + 1023) / 1024);
  k_mg_norm<<<kNumSMs * 8, 256, 0, s>>>(b.A, b.B, n, p, b.norm2, b.st);
  k_keep_count<<<ntiles, 256, 0, s>>>(b.norm2, n, b.st, b.tile_cnt);
  k_scan_tiles<<<1, 1024, 0, s>>>(b.tile_cnt, ntiles, &b.st->ntot);
  k_keep_scatter<<<ntiles, 256, 0, s>>>(b.norm2, n, b.st, b.tile_cnt, b.idx);
  k_reset_max<<<1, 1, 0, s>>>(b.st);
  k_compact<<<kNumSMs * 4, 256, 0, s>>>(b.A, b.B, n, p, b.idx, b.norm2, b.st, b.Ac, b.Bc, b.nu,
                                        b.nu0, b.pos, b.perm, b.active);
  launches += 6;
  ISDF_CHECK_LAUNCH();
  QrState hst;
  ISDF_TRY(read_back(&hst, b.st, sizeof(QrState), s));
  const int ntot = hst.ntot;
  const int kmax = std::min(kmax_cap, ntot);
  res->ntot_mg = ntot;

  // pivoted Gram-Schmidt over the kept columns
  const int ld = ntot + (ntot & 1);  // Ac / Bc leading dimension (k_compact)
  const unsigned ugrid = (unsigned)((ntot + CoreU::BM - 1) / CoreU::BM);
  const bool uv2 = ((reinterpret_cast<size_t>(b.Bc) | reinterpret_cast<size_t>(b.Qm)) & 15) == 0 &&
                   p % 2 == 0;
  const unsigned agrid = (unsigned)std::min(kNumSMs * 8, (ntot + 255) / 256);
  for (int k = 0; k < kmax; ++k) {
    k_argpos<<<agrid, 256, 0, s>>>(b.nu, b.pos, b.active, ntot, b.st);
    k_pick<<<1, 1024, 0, s>>>(k, p, ld, b.Ac, b.Bc, b.pos, b.perm, b.active, b.sel, b.st, b.x);
    launches += 2;
    if (k > 0) {
      for (int pass = 0; pass < 2; ++pass) {
        k_qt_x<<<k, 256, 0, s>>>(b.Q, m, k, b.x, b.st, b.cdot);
        k_x_minus_qc<<<(m + 31) / 32, 1024, 0, s>>>(b.Q, m, k, b.cdot, b.st, b.x);
        launches += 2;
      }
    }
    k_normalise<<<1, 1024, 0, s>>>(k, p, b.x, b.st, b.Q, b.Qm);
    if (uv2)  // 16-byte aligned rows: the warp-specialised tile
      launch_update_ws(b, ntot, ld, p, s);
    else
      k_update<1><<<ugrid, 256, CoreU::SMEM_BYTES, s>>>(b.Ac, b.Bc, ntot, ld, p, b.Qm, b.active, b.nu,
                                                        b.nu0, b.st, b.rec_list);
    k_recompute<<<kRecomputeGrid, 256, sizeof(double) * m, s>>>(b.Ac, b.Bc, ld, p, b.Q, m, k + 1,
                                                                b.rec_list, b.nu, b.nu0, b.st,
                                                                b.rec_dots);
    launches += 3;
    if ((k & 255) == 255) ISDF_CHECK_LAUNCH();
  }
  ISDF_CHECK_LAUNCH();

  // piv = MGIdx[pivots], then the remaining kept columns in pivoted order, then 0
  std::vector<int> idx(ntot), perm(ntot), sel(kmax);
  ISDF_TRY(read_back(&hst, b.st, sizeof(QrState), s));
  int err = 0;
  ISDF_TRY(read_back(&err, b.err, sizeof(int), s));
  if (err) return record_error(ISDF_ERR_TIMEOUT, "QRCP: an update pipeline wait timed out");
  ISDF_TRY(read_back(idx.data(), b.idx, sizeof(int) * ntot, s));
  ISDF_TRY(read_back(perm.data(), b.perm, sizeof(int) * ntot, s));
  if (kmax > 0) ISDF_TRY(read_back(sel.data(), b.sel, sizeof(int) * kmax, s));
  std::memset(args.piv, 0, sizeof(int) * (size_t)n);
  for (int j = 0; j < ntot; ++j) args.piv[j] = idx[perm[j]];
  res->steps = kmax;
  res->num_pre = p;
  res->recomputes = hst.total_rec;
  res->done_early = hst.done;
  res->launches = launches + (readback_mailbox() ? (kmax > 0 ? 6 : 5) : 0);
  return ISDF_OK;
}

}  // namespace isdf_b200
