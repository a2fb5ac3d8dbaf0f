// Density-weighted K-means interpolation-point selection on sm_100a.
//
// Reproduces the reference's CPU KMEAN (src/common/utility.cpp:631-988) bit
// for bit at one rank: every FP64 operation is an explicitly rounded add /
// sub / mul / div (no FMA contraction, like the reference's SSE2 x86-64
// build), the centroid sums are folded in point-index order per cluster, and
// every argmin keeps the first minimum. The reference's own GPU kernels
// (src/cuda/cuda_utils.cu:124-234,368-428) materialise an Npt x mu distance
// matrix and FMA-contract the distance; here the distance matrix is never
// stored and the arithmetic follows the CPU path.
//
// Device data layout (SoA, one entry per K-means point p in [0, Ng)):
//   pidx[p]   grid index of point p: the kept points ascending, then the
//             zero tail that aliases grid point 0 (utility.cpp:648,659,707);
//   px,py,pz  coordinates by the formula of utility.cpp:711-713;
//   pw        weight w[pidx[p]];
//   label[p]  nearest centroid.
// Centroids: double4 (x, y, z, 0) in cen[], rk on the device in st->rk.
#include <mutex>
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "arena.h"
#include "comm.h"
#include "common.cuh"
#include "solve.h"
#include "kmeans.h"
#include "readback.h"

namespace isdf_b200 {

namespace {

constexpr int kTile = 2048;      // points per counting-sort tile (one walking warp each)
constexpr int kFinalChunk = 4096;  // points per partial argmin chunk
constexpr int kIterChunk = 8;    // Lloyd iterations launched between host checks
constexpr int kMaxCellsPerDim = 20;  // centroid cell grid of the pruned assignment
constexpr int kMaxCells = kMaxCellsPerDim * kMaxCellsPerDim * kMaxCellsPerDim;

struct KmState {
  int s;        // Lloyd iterations completed
  int flag;     // labels changed in the last assignment
  int changed;  // accumulator for the running assignment
  int done;
  int rk;       // current number of centroids
  int npt;      // kept points
  int any_empty;
  int reset_bounds;  // centroid indices moved (empty-cluster compaction): bounds invalid
  unsigned long long maxw_bits;
  unsigned long long maxshift_bits;  // largest centroid move of this iteration (bit pattern)
  unsigned long long searches;       // assignments that ran the cell search (all iterations)
};

// ---------------------------------------------------------------- weight
// w(r) = 0 + (sum_{S2} psi^2) * (sum_{S1} psi^2), each sum a sequential fold
// over the states in increasing order (getpoints_Kmeans_MPI.cpp:37-45).
// One thread per grid point; a warp reads 32 consecutive doubles of a column.
__global__ void __launch_bounds__(256) k_weight(const double* __restrict__ psi, long long ng,
                                                int s2lo, int s2hi, int s1lo, int s1hi, int same,
                                                double* __restrict__ w) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long r = (long long)blockIdx.x * blockDim.x + threadIdx.x; r < ng; r += stride) {
    const double* p = psi + r;
    double si = 0.0;
#pragma unroll 8
    for (int i = s2lo; i < s2hi; ++i) {
      double v = __ldg(p + (long long)i * ng);
      si = radd(si, rmul(v, v));
    }
    double sj = si;
    if (!same) {
      sj = 0.0;
#pragma unroll 8
      for (int j = s1lo; j < s1hi; ++j) {
        double v = __ldg(p + (long long)j * ng);
        sj = radd(sj, rmul(v, v));
      }
    }
    w[r] = radd(0.0, rmul(si, sj));
  }
}

// ---------------------------------------------------------------- filter
// maxW = max(0, max_r w(r)) (findMax starts at 0.0). Non-negative doubles
// order like their bit patterns, so an integer atomicMax is exact.
__global__ void k_maxw(const double* __restrict__ w, long long n, KmState* st) {
  double m = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    m = fmax(m, w[i]);
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0 && m > 0.0)
    atomicMax(&st->maxw_bits, (unsigned long long)__double_as_longlong(m));
}

__device__ __forceinline__ bool kept(double wv, double thr) { return wv > thr; }

// Per-tile count of kept points (tile = blockDim.x * 4 points).
__global__ void __launch_bounds__(256) k_filter_count(const double* __restrict__ w, long long n,
                                                      const KmState* st, int* tile_cnt) {
  const double thr = rmul(1e-8, __longlong_as_double((long long)st->maxw_bits));
  __shared__ int warp_cnt[8];
  long long base = (long long)blockIdx.x * 1024;
  int c = 0;
  for (int k = 0; k < 4; ++k) {
    long long i = base + k * 256 + threadIdx.x;
    if (i < n && kept(w[i], thr)) ++c;
  }
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if ((threadIdx.x & 31) == 0) warp_cnt[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int k = 0; k < 8; ++k) t += warp_cnt[k];
    tile_cnt[blockIdx.x] = t;
  }
}

// Exclusive scan of ntiles counts in one block; writes npt.
__global__ void __launch_bounds__(1024) k_scan_small(int* cnt, int ntiles, int* total) {
  __shared__ int part[1024];
  const int per = (ntiles + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, ntiles);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += cnt[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    int v = cnt[i];
    cnt[i] = run;
    run += v;
  }
  if (threadIdx.x == 1023) *total = part[1023];
}

// Order-preserving compaction of the kept grid indices into pidx[0..npt);
// pidx[npt..n) was zeroed before (the reference's zero-initialised tail).
__global__ void __launch_bounds__(256) k_filter_scatter(const double* __restrict__ w, long long n,
                                                        const KmState* st, const int* tile_off,
                                                        int* __restrict__ pidx) {
  const double thr = rmul(1e-8, __longlong_as_double((long long)st->maxw_bits));
  __shared__ int warp_cnt[8][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  long long base = (long long)blockIdx.x * 1024;
  unsigned ballots[4];
  for (int k = 0; k < 4; ++k) {
    long long i = base + k * 256 + threadIdx.x;
    bool f = i < n && kept(w[i], thr);
    ballots[k] = __ballot_sync(0xffffffffu, f);
    if (lane == 0) warp_cnt[wid][k] = __popc(ballots[k]);
  }
  __syncthreads();
  // order of elements: k-major, then warp, then lane
  int off = tile_off[blockIdx.x];
  for (int k = 0; k < 4; ++k) {
    int before = 0;
    for (int kk = 0; kk < k; ++kk)
      for (int ww = 0; ww < 8; ++ww) before += warp_cnt[ww][kk];
    for (int ww = 0; ww < wid; ++ww) before += warp_cnt[ww][k];
    long long i = base + k * 256 + threadIdx.x;
    if (ballots[k] & (1u << lane)) {
      int r = __popc(ballots[k] & ((1u << lane) - 1u));
      pidx[off + before + r] = (int)i;
    }
  }
}

// Coordinates of grid point t by the formula of utility.cpp:711-713 (and
// :758-760 for centroids), each operation rounded as the reference's build.
__device__ __forceinline__ void grid_coords(int t, int nx, int ny, double dx0, double dx1,
                                            double dx2, double* gx_, double* gy_,
                                            double* gz_) {
  const double gx = rmul((double)(t % nx), dx0);
  const double gy = rmul(rdiv(rsub((double)(t % (nx * ny)), rdiv(gx, dx0)), (double)nx), dx1);
  const double gz =
      rmul(rdiv(rsub(rsub((double)t, rdiv(gx, dx0)), rmul(rdiv(gy, dx1), (double)nx)),
                (double)(nx * ny)),
           dx2);
  *gx_ = gx;
  *gy_ = gy;
  *gz_ = gz;
}

// Point coordinates and weights (utility.cpp:707-713); the centroids start
// at the first rk kept points (utility.cpp:750-762), i.e. points 0..rk-1.
__global__ void k_points(const int* __restrict__ pidx, const double* __restrict__ w, int n,
                         int nx, int ny, double dx0, double dx1, double dx2,
                         double* __restrict__ px, double* __restrict__ py,
                         double* __restrict__ pz, double* __restrict__ pw, int rk,
                         double4* __restrict__ cen) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
    int t = pidx[p];
    double gx, gy, gz;
    grid_coords(t, nx, ny, dx0, dx1, dx2, &gx, &gy, &gz);
    px[p] = gx;
    py[p] = gy;
    pz[p] = gz;
    pw[p] = w[t];
    if (p < rk) cen[p] = make_double4(gx, gy, gz, 0.0);
  }
}

// Warm start (utility.cpp:725-749): w at the previous pivots, for the
// filter test the reference applies to them.
__global__ void k_gather_w(const double* __restrict__ w, const int* __restrict__ idx, int cnt,
                           double* __restrict__ out) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < cnt; j += gridDim.x * blockDim.x)
    out[j] = w[idx[j]];
}

// Warm start: centroid j starts at grid point cinit[j].
__global__ void k_warm_centroids(const int* __restrict__ cinit, int rk, int nx, int ny,
                                 double dx0, double dx1, double dx2,
                                 double4* __restrict__ cen) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < rk; j += gridDim.x * blockDim.x) {
    double gx, gy, gz;
    grid_coords(cinit[j], nx, ny, dx0, dx1, dx2, &gx, &gy, &gz);
    cen[j] = make_double4(gx, gy, gz, 0.0);
  }
}

// ---------------------------------------------------------------- assign
// d = ((dx*dx + dy*dy) + dz*dz) with dx = point - centroid (pdist2,
// utility.cpp:598-615); label = first centroid reaching the minimum
// (findMin Dim=1, utility.cpp:579-595).
constexpr int kAssignThreads = 256;

// ---------------------------------------------------------------- pruned assign
// Exact spatial pruning: centroids are binned into a uniform nc^3 cell grid
// over the box; a point visits cells in Chebyshev rings around its own cell
// and skips a cell only when the squared distance from the point to the
// cell's box, shrunk by a relative 2e-14 safety factor (well above the
// rounding of both the box bound and the distance formula), is strictly
// greater than the best distance found. Every skipped centroid would have
// computed a strictly larger distance, so the result - the first centroid in
// index order reaching the minimum computed distance, compared as (d, index)
// pairs - is the brute-force result bit for bit.
struct CellGrid {
  int nc;
  double h[3];
  double tol;
};

// Thread -> point map of the assignment. Brick mode: each warp takes a
// 4 x 4 x 2 brick of grid points instead of 32 points along the kept-point
// list, so that its lanes search nearly the same cells; a grid point that
// the weight filter dropped leaves its lane idle (g2p[g] = -1), and the
// zero-tail points p >= npt (copies of grid point 0) follow the bricks one
// per thread. Linear mode: thread t takes point t. Either way every point is
// assigned once and the result does not depend on the map.
// A rank of a sharded selection assigns only its points [p_lo, p_hi): its
// kept points lie in a z range of bricks (launched from brick thread t0 on),
// its zero-tail points follow them.
struct AssignMap {
  int brick;  // 0: linear
  int nx, ny, nz;
  int nbx, nby;    // bricks along x and y
  long long nbt;   // brick threads launched: bricks x 32
  long long t0;    // first brick thread
  int npt, n;
  int p_lo, p_hi;  // the points this launch assigns
  const int* g2p;  // grid index -> kept-point index (or -1); nullptr: identity
};

__device__ __forceinline__ int assign_point(long long t, const AssignMap& am) {
  if (!am.brick) {
    const long long p = am.p_lo + t;
    return p < am.p_hi ? (int)p : -1;
  }
  if (t >= am.nbt) {
    const long long p = (long long)max(am.npt, am.p_lo) + (t - am.nbt);
    return p < am.p_hi ? (int)p : -1;
  }
  t += am.t0;
  const long long b = t >> 5;
  const int l = (int)(t & 31);
  const int bx = (int)(b % am.nbx);
  const long long r = b / am.nbx;
  const int by = (int)(r % am.nby), bz = (int)(r / am.nby);
  const int ix = bx * 4 + (l & 3), iy = by * 4 + ((l >> 2) & 3), iz = bz * 2 + (l >> 4);
  if (ix >= am.nx || iy >= am.ny || iz >= am.nz) return -1;
  const int g = ix + am.nx * (iy + am.ny * iz);
  const int p = am.g2p ? am.g2p[g] : g;
  return (p >= am.p_lo && p < am.p_hi) ? p : -1;
}

// Inverse of the kept-point list: g2p[pidx[p]] = p for p < npt (the rest -1).
__global__ void k_grid_to_point(const int* __restrict__ pidx, int npt, int* __restrict__ g2p) {
  for (int p = blockIdx.x * blockDim.x + threadIdx.x; p < npt; p += gridDim.x * blockDim.x)
    g2p[pidx[p]] = p;
}

// One block: cell of each centroid, counting sort into cell order.
// In-place inclusive scan of a[0..n) by a block of 1024 threads: every
// thread sums a contiguous chunk, the chunk totals are scanned across the
// warp and the block, and each thread rewrites its chunk.
__device__ void block_inclusive_scan(int* a, int n, int* warp_tot) {
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int per = (n + 1023) / 1024;
  const int b0 = min(n, tid * per), b1 = min(n, b0 + per);
  int sum = 0;
  for (int i = b0; i < b1; ++i) sum += a[i];
  int v = sum;
  for (int o = 1; o < 32; o <<= 1) {
    const int u = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += u;
  }
  if (lane == 31) warp_tot[w] = v;
  __syncthreads();
  if (w == 0) {
    int t = warp_tot[lane];
    for (int o = 1; o < 32; o <<= 1) {
      const int u = __shfl_up_sync(0xffffffffu, t, o);
      if (lane >= o) t += u;
    }
    warp_tot[lane] = t;
  }
  __syncthreads();
  int run = v - sum + (w > 0 ? warp_tot[w - 1] : 0);
  for (int i = b0; i < b1; ++i) {
    run += a[i];
    a[i] = run;
  }
  __syncthreads();
}

// Centroids into the cell grid (cell_start, cell_cen).
__global__ void __launch_bounds__(1024) k_build_cells(const double4* __restrict__ cen,
                                                      const KmState* st, CellGrid g,
                                                      int* __restrict__ cell_start,
                                                      double4* __restrict__ cell_cen,
                                                      int* __restrict__ cell_of) {
  if (st->done) return;
  extern __shared__ int sc[];  // ncells + 1 counters
  __shared__ int warp_tot[32];
  const int rk = st->rk;
  const int nc = g.nc, ncells = nc * nc * nc;
  for (int c = threadIdx.x; c <= ncells; c += blockDim.x) sc[c] = 0;
  __syncthreads();
  for (int j = threadIdx.x; j < rk; j += blockDim.x) {
    const double4 c = cen[j];
    const int ci = min(nc - 1, max(0, (int)floor(c.x / g.h[0])));
    const int cj = min(nc - 1, max(0, (int)floor(c.y / g.h[1])));
    const int ck = min(nc - 1, max(0, (int)floor(c.z / g.h[2])));
    const int id = ci + nc * (cj + nc * ck);
    cell_of[j] = id;
    atomicAdd(&sc[id + 1], 1);
  }
  __syncthreads();
  block_inclusive_scan(sc + 1, ncells, warp_tot);
  for (int c = threadIdx.x; c <= ncells; c += blockDim.x) cell_start[c] = sc[c];
  __syncthreads();
  // placement inside a cell is arbitrary: the search compares (d, index) pairs
  for (int j = threadIdx.x; j < rk; j += blockDim.x) {
    const int slot = atomicAdd(&sc[cell_of[j]], 1);
    const double4 c = cen[j];
    cell_cen[slot] = make_double4(c.x, c.y, c.z, (double)j);
  }
}

// Squared distance in the reference's rounding (pdist2, utility.cpp:598-615).
__device__ __forceinline__ double ref_dist2(double x, double y, double z, const double4& c) {
  const double d1 = rsub(x, c.x), d2 = rsub(y, c.y), d3 = rsub(z, c.z);
  return radd(radd(rmul(d1, d1), rmul(d2, d2)), rmul(d3, d3));
}

// Distance bounds (Hamerly): bnd[p] = (u, l), u >= the true distance from p
// to its assigned centroid, l <= the true distance to every other centroid.
// Moving centroids move them by at most shift[label] and the largest shift.
// When u (1 + 1e-12) < l, the assigned centroid is strictly nearest with a
// margin far above the relative error of the rounded squared distances
// (~1e-15), so the reference's argmin (first minimum of the rounded
// distances) is the assigned label and the search is skipped. Otherwise the
// exact ring search runs and the bounds are rebuilt from it: u from the
// best distance, l from the second best seen, the box bounds of skipped
// cells and the ring at which the search stopped.
constexpr double kBoundMargin = 1.0 + 1e-12;
constexpr double kRoundUp = 1.0 + 1e-13;
constexpr double kRoundDown = 1.0 - 1e-13;

// Exact ring search for the nearest centroid of (x, y, z) (first minimum of
// the reference's rounded distances), seeded with centroid `old` when it is
// valid; writes the point's distance bounds and returns the label.
__device__ __forceinline__ int ring_search(double x, double y, double z, int old, int rk,
                                           const double4* __restrict__ cen,
                                           const int* __restrict__ cell_start,
                                           const double4* __restrict__ cell_cen,
                                           const CellGrid& g, double2* bnd_p) {
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  double best = inf;
  int bj = 0x7fffffff;
  if (old >= 0 && old < rk) {  // any centroid is a valid start
    best = ref_dist2(x, y, z, cen[old]);
    bj = old;
  }
  const int pi = min(g.nc - 1, max(0, (int)floor(x / g.h[0])));
  const int pj = min(g.nc - 1, max(0, (int)floor(y / g.h[1])));
  const int pk = min(g.nc - 1, max(0, (int)floor(z / g.h[2])));
  double second = inf;  // second-best squared distance seen
  double floor2 = inf;  // lower bound (squared) on every centroid not seen
  const double hmin = fmin(g.h[0], fmin(g.h[1], g.h[2]));
  const double shrink = 1.0 - 2e-14;
  for (int r = 0; r <= g.nc; ++r) {
    if (r >= 2) {
      const double lb = (r - 1) * hmin - g.tol;
      if (lb > 0.0 && lb * lb * shrink > best) {
        floor2 = fmin(floor2, lb * lb * shrink);
        break;
      }
    }
    for (int dk = -r; dk <= r; ++dk) {
      const int ck = pk + dk;
      if (ck < 0 || ck >= g.nc) continue;
      for (int dj = -r; dj <= r; ++dj) {
        const int cj = pj + dj;
        if (cj < 0 || cj >= g.nc) continue;
        for (int di = -r; di <= r; ++di) {
          if (max(abs(di), max(abs(dj), abs(dk))) != r) continue;
          const int ci = pi + di;
          if (ci < 0 || ci >= g.nc) continue;
          // box lower bound (box widened by tol)
          const double bx = fmax(0.0, fmax(ci * g.h[0] - g.tol - x, x - (ci + 1) * g.h[0] - g.tol));
          const double by = fmax(0.0, fmax(cj * g.h[1] - g.tol - y, y - (cj + 1) * g.h[1] - g.tol));
          const double bz = fmax(0.0, fmax(ck * g.h[2] - g.tol - z, z - (ck + 1) * g.h[2] - g.tol));
          const double lb = bx * bx + by * by + bz * bz;
          if (lb * shrink > best) {
            floor2 = fmin(floor2, lb * shrink);
            continue;
          }
          const int id = ci + g.nc * (cj + g.nc * ck);
          const int e = cell_start[id + 1];
          for (int q = cell_start[id]; q < e; ++q) {
            const double4 c = cell_cen[q];
            const double d = ref_dist2(x, y, z, c);
            const int j = (int)c.w;
            if (d < best || (d == best && j < bj)) {
              if (j != bj) second = best;
              best = d;
              bj = j;
            } else if (j != bj) {
              second = fmin(second, d);
            }
          }
        }
      }
    }
  }
  *bnd_p = make_double2(__dmul_ru(__dsqrt_ru(best), kRoundUp),
                        __dmul_rd(__dsqrt_rd(fmin(second, floor2)), kRoundDown));
  return bj;
}

// Per point, once per selection (the points do not move): its cell and the
// distances from it to the outside of the 3^3 and 5^3 cell blocks around it
// (rounded down, less the binning tolerance; infinite where a block reaches
// the domain's faces), which the distance-bound test reads instead of
// recomputing three divisions and twelve face distances every iteration.
__global__ void k_point_cells(const double* __restrict__ px, const double* __restrict__ py,
                              const double* __restrict__ pz, int n, CellGrid g,
                              int* __restrict__ pcell, double2* __restrict__ pd12) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const double x = px[p], y = py[p], z = pz[p];
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  const int pi = min(g.nc - 1, max(0, (int)floor(x / g.h[0])));
  const int pj = min(g.nc - 1, max(0, (int)floor(y / g.h[1])));
  const int pk = min(g.nc - 1, max(0, (int)floor(z / g.h[2])));
  double D1 = inf, D2 = inf;
  if (pi >= 2) D1 = fmin(D1, x - (pi - 1) * g.h[0]);
  if (pi + 2 <= g.nc - 1) D1 = fmin(D1, (pi + 2) * g.h[0] - x);
  if (pj >= 2) D1 = fmin(D1, y - (pj - 1) * g.h[1]);
  if (pj + 2 <= g.nc - 1) D1 = fmin(D1, (pj + 2) * g.h[1] - y);
  if (pk >= 2) D1 = fmin(D1, z - (pk - 1) * g.h[2]);
  if (pk + 2 <= g.nc - 1) D1 = fmin(D1, (pk + 2) * g.h[2] - z);
  if (pi >= 3) D2 = fmin(D2, x - (pi - 2) * g.h[0]);
  if (pi + 3 <= g.nc - 1) D2 = fmin(D2, (pi + 3) * g.h[0] - x);
  if (pj >= 3) D2 = fmin(D2, y - (pj - 2) * g.h[1]);
  if (pj + 3 <= g.nc - 1) D2 = fmin(D2, (pj + 3) * g.h[1] - y);
  if (pk >= 3) D2 = fmin(D2, z - (pk - 2) * g.h[2]);
  if (pk + 3 <= g.nc - 1) D2 = fmin(D2, (pk + 3) * g.h[2] - z);
  pcell[p] = pi + g.nc * (pj + g.nc * pk);
  pd12[p] = make_double2(D1 * kRoundDown - g.tol, D2 * kRoundDown - g.tol);
}

// Warp-coherent search. A warp's points are a 4 x 4 x 2 brick of the grid
// (or 32 consecutive points), so the points of a warp that fail the bound
// test share their candidates: with U the largest of their seed distances
// (squared distance to the old label, which bounds each one's nearest), every
// centroid that can be nearest to one of them lies in a cell whose box is
// within sqrt(U) of the points' bounding box. The warp stages those cells'
// centroids in shared memory once and every searching lane runs the same loop
// over them, comparing (d, index) pairs as the ring search does: the label is
// the ring search's bit for bit. Centroids not staged are more than sqrt(U)
// from every point of the box, which gives the lower bound. Lanes without a
// seed (the first assignment), more than 216 cells or more than 160 candidates take the
// ring search instead.
constexpr int kWarpCand = 160;   // centroids staged per warp
constexpr int kWarpCells = 216;  // cells a warp may scan

__device__ __forceinline__ double warp_max(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}
__device__ __forceinline__ double warp_min(double v) {
  for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__global__ void __launch_bounds__(kAssignThreads) k_assign_warp(
    const double* __restrict__ px, const double* __restrict__ py, const double* __restrict__ pz,
    int n, const double4* __restrict__ cen, const int* __restrict__ cell_start,
    const double4* __restrict__ cell_cen, CellGrid g, AssignMap am, KmState* st,
    int* __restrict__ label, int count, double2* __restrict__ bnd,
    const double* __restrict__ shift, const float* __restrict__ nbshift,
    const int* __restrict__ pcell, const double2* __restrict__ pd12) {
  if (st->done) return;
  __shared__ double4 cand[kAssignThreads / 32][kWarpCand];
  const int rk = st->rk;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int p = assign_point((long long)blockIdx.x * blockDim.x + threadIdx.x, am);
  bool need = false;
  int old = -1;
  if (p >= 0 && p < n) {
    old = count ? label[p] : -1;
    need = true;
    if (old >= 0 && old < rk && count && !st->reset_bounds) {
      const double2 b = bnd[p];
      // Every other centroid moved closer by at most its shift: at most
      // the 3^3-block maximum inside the 27 cells around p, the 5^3-block
      // maximum in the ring beyond (which started at least D1 = dd.x away),
      // the global maximum further out (at least D2 = dd.y away); no bound
      // across the domain's faces.
      const double gmax = __longlong_as_double((long long)st->maxshift_bits);
      const int cell = pcell[p];
      const double near1 = (double)nbshift[cell], near2 = (double)nbshift[kMaxCells + cell];
      const double2 dd = pd12[p];
      double lo = __dsub_rd(b.y, near1);
      lo = fmin(lo, __dsub_rd(fmax(b.y, dd.x), near2));
      lo = fmin(lo, __dsub_rd(fmax(b.y, dd.y), gmax));
      lo = fmax(0.0, lo);
      double up = __dadd_ru(b.x, shift[old]);
      if (!(up * kBoundMargin < lo))
        up = __dmul_ru(__dsqrt_ru(ref_dist2(px[p], py[p], pz[p], cen[old])), kRoundUp);
      if (up * kBoundMargin < lo) {  // the label stays
        bnd[p] = make_double2(up, lo);
        need = false;
      }
    }
  }
  const unsigned mask = __ballot_sync(0xffffffffu, need);
  if (!mask) return;
  const double inf = __longlong_as_double(0x7ff0000000000000LL);
  double x = 0.0, y = 0.0, z = 0.0, best = inf;
  int bj = 0x7fffffff;
  if (need) {
    x = px[p];
    y = py[p];
    z = pz[p];
    if (old >= 0 && old < rk) {
      best = ref_dist2(x, y, z, cen[old]);
      bj = old;
    }
  }
  const double shrink = 1.0 - 2e-14;
  bool ok = __all_sync(0xffffffffu, !need || bj != 0x7fffffff);
  const double U = warp_max(need ? best : 0.0);
  const double x0 = warp_min(need ? x : inf), x1 = warp_max(need ? x : -inf);
  const double y0 = warp_min(need ? y : inf), y1 = warp_max(need ? y : -inf);
  const double z0 = warp_min(need ? z : inf), z1 = warp_max(need ? z : -inf);
  int total = 0;
  if (ok) {
    const double R = __dmul_ru(__dsqrt_ru(U), kRoundUp) + g.tol;
    const int nc = g.nc;
    const int i0 = min(nc - 1, max(0, (int)floor((x0 - R) / g.h[0])));
    const int i1 = min(nc - 1, max(0, (int)floor((x1 + R) / g.h[0])));
    const int j0 = min(nc - 1, max(0, (int)floor((y0 - R) / g.h[1])));
    const int j1 = min(nc - 1, max(0, (int)floor((y1 + R) / g.h[1])));
    const int k0 = min(nc - 1, max(0, (int)floor((z0 - R) / g.h[2])));
    const int k1 = min(nc - 1, max(0, (int)floor((z1 + R) / g.h[2])));
    const int ni = i1 - i0 + 1, nj = j1 - j0 + 1;
    const int ncell = ni * nj * (k1 - k0 + 1);
    if (ncell > kWarpCells) ok = false;
    for (int base = 0; ok && base < ncell; base += 32) {
      const int c = base + lane;
      int cnt = 0, first = 0;
      if (c < ncell) {
        const int ci = i0 + c % ni, cj = j0 + (c / ni) % nj, ck = k0 + c / (ni * nj);
        // distance from the points' box to the cell's box (widened by tol)
        const double bx = fmax(0.0, fmax(ci * g.h[0] - g.tol - x1, x0 - (ci + 1) * g.h[0] - g.tol));
        const double by = fmax(0.0, fmax(cj * g.h[1] - g.tol - y1, y0 - (cj + 1) * g.h[1] - g.tol));
        const double bz = fmax(0.0, fmax(ck * g.h[2] - g.tol - z1, z0 - (ck + 1) * g.h[2] - g.tol));
        const double lb = bx * bx + by * by + bz * bz;
        if (!(lb * shrink > U)) {
          const int id = ci + nc * (cj + nc * ck);
          first = cell_start[id];
          cnt = cell_start[id + 1] - first;
        }
      }
      int off = cnt;  // inclusive scan over the warp
      for (int o = 1; o < 32; o <<= 1) {
        const int v = __shfl_up_sync(0xffffffffu, off, o);
        if (lane >= o) off += v;
      }
      const int here = __shfl_sync(0xffffffffu, off, 31);
      if (total + here > kWarpCand) {
        ok = false;
        break;
      }
      for (int q = 0; q < cnt; ++q) cand[wid][total + off - cnt + q] = cell_cen[first + q];
      total += here;
    }
  }
  __syncwarp();
  int changed = 0;
  if (need) {
    int lab;
    if (ok) {
      double second = inf;
      for (int q = 0; q < total; ++q) {
        const double4 c = cand[wid][q];
        const double d = ref_dist2(x, y, z, c);
        const int j = (int)c.w;
        if (d < best || (d == best && j < bj)) {
          if (j != bj) second = best;
          best = d;
          bj = j;
        } else if (j != bj) {
          second = fmin(second, d);
        }
      }
      // every centroid not staged is more than sqrt(U) from the point
      const double floor2 = U * shrink;
      bnd[p] = make_double2(__dmul_ru(__dsqrt_ru(best), kRoundUp),
                            __dmul_rd(__dsqrt_rd(fmin(second, floor2)), kRoundDown));
      lab = bj;
    } else {
      lab = ring_search(x, y, z, old, rk, cen, cell_start, cell_cen, g, &bnd[p]);
    }
    if (count && old != lab) ++changed;
    label[p] = lab;
  }
  for (int o = 16; o > 0; o >>= 1) changed += __shfl_xor_sync(0xffffffffu, changed, o);
  if (lane == 0) {
    if (count && changed) atomicAdd(&st->changed, changed);
    atomicAdd(&st->searches, (unsigned long long)__popc(mask));
  }
}

// ---------------------------------------------------------------- control
__global__ void k_iter_begin(KmState* st, double max_f, int max_iter) {
  if (st->done) return;
  if (!((double)st->flag > max_f && st->s < max_iter)) {
    st->done = 1;
    return;
  }
  st->changed = 0;
  st->any_empty = 0;
  st->reset_bounds = 0;
  st->maxshift_bits = 0;
}

// set_flag = 0 in a sharded selection, whose flag is the ranks' total (k_shard_begin).
__global__ void k_iter_end(KmState* st, int set_flag) {
  if (st->done) return;
  if (set_flag) st->flag = st->changed;
  st->s += 1;
}

// ---------------------------------------------------------------- update
// Stable counting sort of the points by label (tiles of kTile points), then
// one warp per cluster folds w, w*x, w*y, w*z over the members in increasing
// point index: the exact sequence of additions of utility.cpp:816-822.
__global__ void __launch_bounds__(256) k_hist(const int* __restrict__ label, int n,
                                              const KmState* st, int* __restrict__ hist) {
  if (st->done) return;
  extern __shared__ int sh[];
  const int rk = st->rk;
  for (int l = threadIdx.x; l < rk; l += blockDim.x) sh[l] = 0;
  __syncthreads();
  const int base = blockIdx.x * kTile;
  const int end = min(base + kTile, n);
  for (int p = base + threadIdx.x; p < end; p += blockDim.x) atomicAdd(&sh[label[p]], 1);
  __syncthreads();
  int* row = hist + (size_t)blockIdx.x * rk;
  for (int l = threadIdx.x; l < rk; l += blockDim.x) row[l] = sh[l];
}

// Per label: exclusive scan over tiles (in place) and the member count. A
// block holds 32 labels (one per lane) and kScanWarps warps, each over a
// contiguous range of tiles: the warps' range sums, their exclusive prefix in
// shared memory, then each warp rewrites its range from that prefix. One
// thread per label walking all tiles left the scan bound by the latency of
// its ~ntiles/16 dependent load batches.
constexpr int kScanWarps = 16;

__global__ void __launch_bounds__(32 * kScanWarps) k_hist_scan(int* __restrict__ hist, int ntiles,
                                                               const KmState* st,
                                                               int* __restrict__ members) {
  if (st->done) return;
  const int rk = st->rk;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int l = blockIdx.x * 32 + lane;
  const int per = (ntiles + kScanWarps - 1) / kScanWarps;
  const int t0 = w * per, t1 = min(t0 + per, ntiles);
  __shared__ int part[kScanWarps][32];
  constexpr int kB = 8;  // loads batched ahead of the additions and stores
  int sum = 0;
  if (l < rk) {
    for (int t = t0; t < t1; t += kB) {
      int v[kB];
#pragma unroll
      for (int u = 0; u < kB; ++u) v[u] = t + u < t1 ? hist[(size_t)(t + u) * rk + l] : 0;
#pragma unroll
      for (int u = 0; u < kB; ++u) sum += v[u];
    }
  }
  part[w][lane] = sum;
  __syncthreads();
  if (l >= rk) return;
  int run = 0;
  for (int q = 0; q < w; ++q) run += part[q][lane];
  for (int t = t0; t < t1; t += kB) {
    int v[kB];
#pragma unroll
    for (int u = 0; u < kB; ++u) v[u] = t + u < t1 ? hist[(size_t)(t + u) * rk + l] : 0;
#pragma unroll
    for (int u = 0; u < kB; ++u) {
      if (t + u < t1) hist[(size_t)(t + u) * rk + l] = run;
      run += v[u];
    }
  }
  // the last warp's prefix covers every tile (its own range may be empty)
  if (w == kScanWarps - 1) members[l] = run;
}

// Exclusive scan of the member counts (one block): start[l].
__global__ void __launch_bounds__(1024) k_label_start(const int* __restrict__ members,
                                                      const KmState* st, int* __restrict__ start) {
  if (st->done) return;
  __shared__ int part[1024];
  const int rk = st->rk;
  const int per = (rk + 1023) / 1024;
  const int lo = threadIdx.x * per, hi = min(lo + per, rk);
  int s = 0;
  for (int i = lo; i < hi; ++i) s += members[i];
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {
    int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int run = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = lo; i < hi; ++i) {
    start[i] = run;
    run += members[i];
  }
}

// One tile per block: 128 threads stage the tile's labels in shared memory,
// then one warp walks them in order and gives every point its stable position
// (peers with equal labels share one running offset), written over its label.
// All 128 threads then move the points there: what lands is the point's
// (w x, w y, w z, w), so that the per-cluster fold reads its members
// contiguously. The walk has no global loads in its dependent chain; the
// point loads of the move are independent of one another.
__global__ void __launch_bounds__(128) k_scatter(const int* __restrict__ label, int n,
                                                 const KmState* st, const int* __restrict__ hist,
                                                 const int* __restrict__ start,
                                                 const double* __restrict__ px,
                                                 const double* __restrict__ py,
                                                 const double* __restrict__ pz,
                                                 const double* __restrict__ pw,
                                                 double4* __restrict__ sorted) {
  if (st->done) return;
  extern __shared__ int sm_scatter[];
  const int rk = st->rk;
  int* run = sm_scatter;
  int* lab = sm_scatter + rk;  // the tile's labels, then the points' positions
  const int* row = hist + (size_t)blockIdx.x * rk;
  for (int l = threadIdx.x; l < rk; l += 128) run[l] = start[l] + row[l];
  const int base = blockIdx.x * kTile;
  const int cnt = min(kTile, n - base);
  for (int k = threadIdx.x; k < cnt; k += 128) lab[k] = label[base + k];
  __syncthreads();
  if (threadIdx.x < 32) {
    const int lane = threadIdx.x;
    for (int c = 0; c < cnt; c += 32) {
      const int k = c + lane;
      const bool ok = k < cnt;
      const int l = ok ? lab[k] : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, l);
      const int b = ok ? run[l] : 0;
      __syncwarp();
      if (ok) {
        lab[k] = b + __popc(peers & ((1u << lane) - 1u));
        if (lane == __ffs(peers) - 1) run[l] = b + __popc(peers);
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < cnt; k += 128) {
    const int p = base + k;
    const double w = pw[p];
    sorted[lab[k]] = make_double4(rmul(w, px[p]), rmul(w, py[p]), rmul(w, pz[p]), w);
  }
}

// m successive round-to-nearest additions acc <- fl(acc + c), acc >= 0,
// c >= 0, with the exact result of the sequential loop. While acc stays in
// one binade [2^e, 2^(e+1)) every addition adds the same number of ulps
// (c rounded to the ulp grid), unless c's remainder is exactly half an ulp
// (a tie, which depends on acc's parity): those steps, binade crossings and
// subnormal accumulators are taken one at a time; the rest are jumped.
__device__ double repeat_add(double acc, double c, long long m) {
  const double two53 = 9007199254740992.0;
  while (m > 0) {
    if (c == 0.0) return radd(acc, 0.0);
    if (!(acc >= 2.2250738585072014e-308) || c >= ldexp(1.0, ilogb(acc))) {
      acc = radd(acc, c);
      --m;
      continue;
    }
    const int e = ilogb(acc);
    const double u = ldexp(1.0, e - 52);  // ulp of acc
    const double cu = c / u;              // exact: u is a power of two
    const double q = floor(cu);
    const double r = cu - q;
    if (r == 0.5) {
      acc = radd(acc, c);
      --m;
      continue;
    }
    const double qp = q + (r > 0.5 ? 1.0 : 0.0);  // ulps added per step
    if (qp == 0.0) return acc;  // c rounds away now and at every larger exponent
    const double a = acc / u;   // integer in [2^52, 2^53)
    const double room = two53 - q - 2.0 - a;
    if (room < 0.0) {
      acc = radd(acc, c);
      --m;
      continue;
    }
    long long k = (long long)floor(room / qp) + 1;
    if (k > m) k = m;
    acc = __dmul_rn(__dadd_rn(a, __dmul_rn((double)k, qp)), u);  // all exact
    m -= k;
  }
  return acc;
}

// One warp per cluster: sequential fold over the members (in index order).
// The zero-tail points p >= npt are identical copies of grid point 0 (weight
// w[0], coordinates (0, 0, 0)) and come last in their cluster's member list,
// so their part of the fold is a repeated addition of one value. The members'
// (w x, w y, w z, w) are read contiguously, kSegBatches batches of 32 ahead
// of the fold, so that the load latency hides behind the dependent additions.
constexpr int kSegBatches = 4;

__device__ __forceinline__ void seg_load(const double4* __restrict__ v, int q, int m, int lane,
                                         double4 (&out)[kSegBatches]) {
#pragma unroll
  for (int j = 0; j < kSegBatches; ++j) {
    const int i = q + j * 32 + lane;
    out[j] = i < m ? v[i] : make_double4(0.0, 0.0, 0.0, 0.0);
  }
}

// n, npt: the points folded and how many of them are kept points (the rest
// is zero tail); flag_empty: record an empty cluster in st (off when the sums
// are one rank's partial sums).
__global__ void __launch_bounds__(256) k_segsum(const double4* __restrict__ sorted,
                                                const int* __restrict__ start,
                                                const int* __restrict__ members,
                                                const double* __restrict__ px,
                                                const double* __restrict__ py,
                                                const double* __restrict__ pz,
                                                const double* __restrict__ pw,
                                                const int* __restrict__ label, int n, int npt,
                                                int flag_empty, KmState* st,
                                                double4* __restrict__ sums) {
  if (st->done) return;
  const int rk = st->rk;
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= rk) return;
  const double4* v = sorted + start[c];
  int m = members[c];
  long long tail = 0;
  if (npt < n && label[npt] == c) {
    tail = n - npt;
    m -= (int)tail;
  }
  // lanes 0..3 each fold one component (w x, w y, w z, w) from the warp's
  // shared-memory copy of the batch: one load and one dependent addition per
  // member instead of four broadcasts and four additions
  __shared__ double4 stage[8][32 * kSegBatches];
  double4* st_w = stage[threadIdx.x >> 5];
  double acc = 0.0;
  double4 cur[kSegBatches], nxt[kSegBatches];
  seg_load(v, 0, m, lane, cur);
  for (int q = 0; q < m; q += 32 * kSegBatches) {
#pragma unroll
    for (int j = 0; j < kSegBatches; ++j) st_w[j * 32 + lane] = cur[j];
    __syncwarp();
    if (q + 32 * kSegBatches < m) seg_load(v, q + 32 * kSegBatches, m, lane, nxt);
    const int cnt = min(32 * kSegBatches, m - q);
    if (lane < 4) {
      const double* comp = reinterpret_cast<const double*>(st_w) + lane;
      int e = 0;
      for (; e + 8 <= cnt; e += 8) {
#pragma unroll
        for (int u = 0; u < 8; ++u) acc = radd(acc, comp[(e + u) * 4]);
      }
      for (; e < cnt; ++e) acc = radd(acc, comp[e * 4]);
    }
    __syncwarp();
#pragma unroll
    for (int j = 0; j < kSegBatches; ++j) cur[j] = nxt[j];
  }
  double ax = __shfl_sync(0xffffffffu, acc, 0);
  double ay = __shfl_sync(0xffffffffu, acc, 1);
  double az = __shfl_sync(0xffffffffu, acc, 2);
  double aw = __shfl_sync(0xffffffffu, acc, 3);
  if (lane == 0) {
    if (tail) {
      const double w0 = pw[npt];
      aw = repeat_add(aw, w0, tail);
      ax = repeat_add(ax, rmul(w0, px[npt]), tail);
      ay = repeat_add(ay, rmul(w0, py[npt]), tail);
      az = repeat_add(az, rmul(w0, pz[npt]), tail);
    }
    sums[c] = make_double4(ax, ay, az, aw);
    if (flag_empty && aw == 0.0) st->any_empty = 1;
  }
}

// New centroids = sums / count; an empty cluster takes the last centroid's
// sums and rk shrinks (utility.cpp:831-853).
// The update also records how far every centroid moved (rounded upward), the
// largest move, and for every cell of the grid the largest move of a centroid
// that sat in its 3 x 3 x 3 neighbourhood before the update (cell_of still
// holds the previous positions' cells here).
__global__ void __launch_bounds__(1024) k_centroids(double4* __restrict__ sums, KmState* st,
                                                    double4* __restrict__ cen,
                                                    double* __restrict__ shift,
                                                    const int* __restrict__ cell_of, CellGrid g,
                                                    float* __restrict__ nbshift) {
  if (st->done) return;
  int rk = st->rk;
  if (!st->any_empty) {
    extern __shared__ unsigned cmax[];  // 3 x ncells: the cells' maxima, then two pass buffers
    const int nc = g.nc, ncells = nc * nc * nc;
    unsigned* tmp = cmax + ncells;
    for (int c = threadIdx.x; c < ncells; c += blockDim.x) cmax[c] = 0u;
    __syncthreads();
    // the largest move: one atomic per warp (the moves are >= 0, so their bit
    // patterns order as the values do)
    unsigned long long mx = 0ull;
    for (int i = threadIdx.x; i < rk; i += blockDim.x) {
      double4 s = sums[i];
      const double4 o = cen[i];
      const double4 c = make_double4(rdiv(s.x, s.w), rdiv(s.y, s.w), rdiv(s.z, s.w), 0.0);
      cen[i] = c;
      // upper bound on the distance the centroid moved (rounded upward)
      const double dx = fabs(c.x - o.x), dy = fabs(c.y - o.y), dz = fabs(c.z - o.z);
      const double d2 = __dadd_ru(__dadd_ru(__dmul_ru(dx, dx), __dmul_ru(dy, dy)), __dmul_ru(dz, dz));
      const double sh = __dmul_ru(__dsqrt_ru(d2), 1.0 + 1e-13);
      shift[i] = sh;
      mx = max(mx, (unsigned long long)__double_as_longlong(sh));
      atomicMax(&cmax[cell_of[i]], __float_as_uint(__double2float_ru(sh)));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0 && mx) atomicMax(&st->maxshift_bits, mx);
    __syncthreads();
    // 3^3 and 5^3 neighbourhood maxima as separable passes (x, y, z)
    unsigned* t2 = tmp + ncells;
    for (int rad = 1; rad <= 2; ++rad) {
      for (int c = threadIdx.x; c < ncells; c += blockDim.x) {
        const int ci = c % nc;
        unsigned m = 0u;
        for (int d = max(-rad, -ci); d <= min(rad, nc - 1 - ci); ++d) m = max(m, cmax[c + d]);
        tmp[c] = m;
      }
      __syncthreads();
      for (int c = threadIdx.x; c < ncells; c += blockDim.x) {
        const int cj = (c / nc) % nc;
        unsigned m = 0u;
        for (int d = max(-rad, -cj); d <= min(rad, nc - 1 - cj); ++d) m = max(m, tmp[c + d * nc]);
        t2[c] = m;
      }
      __syncthreads();
      float* out = rad == 1 ? nbshift : nbshift + kMaxCells;
      for (int c = threadIdx.x; c < ncells; c += blockDim.x) {
        const int ck = c / (nc * nc);
        unsigned m = 0u;
        for (int d = max(-rad, -ck); d <= min(rad, nc - 1 - ck); ++d)
          m = max(m, t2[c + d * nc * nc]);
        out[c] = __uint_as_float(m);
      }
      __syncthreads();
    }
    return;
  }
  if (threadIdx.x != 0) return;
  st->reset_bounds = 1;
  for (int i = 0; i < rk; i++) {
    double4 s = sums[i];
    if (s.w != 0.0) {
      sums[i] = make_double4(rdiv(s.x, s.w), rdiv(s.y, s.w), rdiv(s.z, s.w), s.w);
    } else {
      rk--;
      sums[i] = sums[rk];
      i--;
    }
  }
  for (int i = 0; i < rk; i++) {
    double4 s = sums[i];
    cen[i] = make_double4(s.x, s.y, s.z, 0.0);
  }
  st->rk = rk;
}

// ---------------------------------------------------------------- final
// Nearest point to every centroid: first minimum over points
// (std::min_element, utility.cpp:926-945). Partial minima per point chunk,
// then an in-order reduction over the chunks.
__global__ void __launch_bounds__(128) k_final_partial(const double* __restrict__ px,
                                                       const double* __restrict__ py,
                                                       const double* __restrict__ pz, int n,
                                                       const double4* __restrict__ cen,
                                                       const KmState* st,
                                                       double* __restrict__ part_d,
                                                       int* __restrict__ part_i) {
  const int rk = st->rk;
  const int j = blockIdx.x * 128 + threadIdx.x;
  const int chunk = blockIdx.y;
  __shared__ double sx[512], sy[512], sz[512];
  double cx = 0, cy = 0, cz = 0;
  if (j < rk) {
    double4 c = cen[j];
    cx = c.x;
    cy = c.y;
    cz = c.z;
  }
  double best = __longlong_as_double(0x7ff0000000000000LL);
  int bi = 0x7fffffff;
  const int base = chunk * kFinalChunk;
  const int end = min(base + kFinalChunk, n);
  for (int p0 = base; p0 < end; p0 += 512) {
    const int m = min(512, end - p0);
    __syncthreads();
    for (int k = threadIdx.x; k < m; k += 128) {
      sx[k] = px[p0 + k];
      sy[k] = py[p0 + k];
      sz[k] = pz[p0 + k];
    }
    __syncthreads();
    for (int k = 0; k < m; ++k) {
      double d1 = rsub(sx[k], cx), d2 = rsub(sy[k], cy), d3 = rsub(sz[k], cz);
      double d = radd(radd(rmul(d1, d1), rmul(d2, d2)), rmul(d3, d3));
      if (d < best) {
        best = d;
        bi = p0 + k;
      }
    }
  }
  if (j < rk) {
    part_d[(size_t)chunk * rk + j] = best;
    part_i[(size_t)chunk * rk + j] = bi;
  }
}

__global__ void k_final_reduce(const double* __restrict__ part_d, const int* __restrict__ part_i,
                               int nchunks, const KmState* st, const int* __restrict__ pidx,
                               int* __restrict__ sel) {
  const int rk = st->rk;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= rk) return;
  double best = __longlong_as_double(0x7ff0000000000000LL);
  int bi = 0;
  for (int c = 0; c < nchunks; ++c) {
    double d = part_d[(size_t)c * rk + j];
    if (d < best) {
      best = d;
      bi = part_i[(size_t)c * rk + j];
    }
  }
  sel[j] = pidx[bi];
}

// ---------------------------------------------------------------- sharded
// A rank's record per Lloyd iteration: entry 0 carries the labels its last
// assignment changed (.x), entries 1..rk its partial centroid sums.
__global__ void k_shard_header(const KmState* st, double4* __restrict__ send) {
  send[0] = make_double4((double)st->changed, 0.0, 0.0, 0.0);
}

// The loop test of utility.cpp:812 on the ranks' total of changed labels
// (the reference's MPI_Reduce + MPI_Bcast of flag, utility.cpp:908-917),
// then the per-iteration resets of k_iter_begin.
__global__ void k_shard_begin(KmState* st, const double4* __restrict__ recv, int ranks, int stride,
                              double max_f, int max_iter) {
  if (st->done) return;
  if (st->s > 0) {
    long long f = 0;
    for (int q = 0; q < ranks; ++q) f += (long long)recv[(size_t)q * stride].x;
    st->flag = (int)f;
  }
  if (!((double)st->flag > max_f && st->s < max_iter)) {
    st->done = 1;
    return;
  }
  st->changed = 0;
  st->any_empty = 0;
  st->reset_bounds = 0;
  st->maxshift_bits = 0;
}

__device__ __forceinline__ double4 add4(const double4& a, const double4& b) {
  return make_double4(radd(a.x, b.x), radd(a.y, b.y), radd(a.z, b.z), radd(a.w, b.w));
}

// The ranks' partial sums combined in binomial-tree order (at step s = 1, 2,
// 4, ..., rank q takes in rank q + s: the reduce of utility.cpp:825-826 as
// MPICH's binomial algorithm runs it), evaluated rank by rank with a stack of
// completed subtrees: (r0 + r1) + (r2 + r3) for 4 ranks, (r0 + r1) + r2 for 3.
__global__ void k_shard_sums(KmState* st, const double4* __restrict__ recv, int ranks, int stride,
                             double4* __restrict__ sums) {
  if (st->done) return;
  const int rk = st->rk;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= rk) return;
  double4 val[8];
  int lev[8];
  int top = 0;
  for (int q = 0; q < ranks; ++q) {
    double4 v = recv[(size_t)q * stride + 1 + c];
    int l = 0;
    while (top > 0 && lev[top - 1] == l) {
      v = add4(val[top - 1], v);
      --top;
      ++l;
    }
    val[top] = v;
    lev[top] = l;
    ++top;
  }
  double4 acc = val[top - 1];
  for (int i = top - 2; i >= 0; --i) acc = add4(val[i], acc);
  sums[c] = acc;
  if (acc.w == 0.0) st->any_empty = 1;
}

// One rank's nearest point per centroid: the first minimum over its points
// (findMin, utility.cpp:926-945), as (distance, grid index).
__global__ void k_final_local(const double* __restrict__ part_d, const int* __restrict__ part_i,
                              int nchunks, const KmState* st, const int* __restrict__ pidx,
                              double2* __restrict__ out) {
  const int rk = st->rk;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= rk) return;
  double best = __longlong_as_double(0x7ff0000000000000LL);
  int bi = 0;
  for (int c = 0; c < nchunks; ++c) {
    double d = part_d[(size_t)c * rk + j];
    if (d < best) {
      best = d;
      bi = part_i[(size_t)c * rk + j];
    }
  }
  out[j] = make_double2(best, (double)pidx[bi]);
}

// MPI_MINLOC over the ranks (utility.cpp:946-969): the smallest distance,
// ties to the smaller grid index.
__global__ void k_minloc(const double2* __restrict__ recv, int ranks, int stride,
                         const KmState* st, int* __restrict__ sel) {
  const int rk = st->rk;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= rk) return;
  double2 best = recv[j];
  for (int q = 1; q < ranks; ++q) {
    const double2 v = recv[(size_t)q * stride + j];
    if (v.x < best.x || (v.x == best.x && v.y < best.y)) best = v;
  }
  sel[j] = (int)best.y;
}

// Dynamic shared memory above 48 KB needs an opt-in per kernel and device.
int set_kmeans_smem_attrs() {
  std::lock_guard<std::mutex> attr_lock(attr_mutex());
  static bool done[64] = {};
  int dev = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  if (dev >= 0 && dev < 64 && done[dev]) return ISDF_OK;
  ISDF_CUDA(cudaFuncSetAttribute(k_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int) * kKmeansMaxMu)));
  ISDF_CUDA(cudaFuncSetAttribute(k_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(sizeof(int) * (kKmeansMaxMu + kTile))));
  ISDF_CUDA(cudaFuncSetAttribute(k_centroids, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(3 * sizeof(unsigned) * kMaxCells)));
  if (dev >= 0 && dev < 64) done[dev] = true;
  return ISDF_OK;
}

struct KmBuffers {
  int* pidx;
  double *px, *py, *pz, *pw;
  int* label;
  double4* sorted;  // (w x, w y, w z, w) in cluster order
  int* hist;
  int* members;
  int* start;
  int* tile_cnt;
  double4* cen;
  double4* sums;
  double2* bnd;    // per point (upper, lower) distance bounds
  double* shift;   // per centroid: distance moved in the last update
  int* g2p;        // grid index -> kept-point index
  float* nbshift;  // per cell: largest move of a centroid in its 27-cell neighbourhood
  double* part_d;
  int* part_i;
  int* sel;
  KmState* st;
  int* cell_start;
  double4* cell_cen;
  int* pcell;        // per point: its cell
  double2* pd12;     // per point: distances to the outside of its 3^3 / 5^3 cell blocks
  int* cell_of;
};

KmBuffers carve(Arena& a, int n, int mu) {
  KmBuffers b;
  const int ntiles = (n + kTile - 1) / kTile;
  const int nfilter = (n + 1023) / 1024;
  const int nchunks = (n + kFinalChunk - 1) / kFinalChunk;
  b.pidx = a.take<int>(n);
  b.px = a.take<double>(n);
  b.py = a.take<double>(n);
  b.pz = a.take<double>(n);
  b.pw = a.take<double>(n);
  b.label = a.take<int>(n);
  b.sorted = a.take<double4>(n);
  b.hist = a.take<int>((size_t)ntiles * mu);
  b.members = a.take<int>(mu);
  b.start = a.take<int>(mu);
  b.tile_cnt = a.take<int>(nfilter);
  b.cen = a.take<double4>(mu);
  b.sums = a.take<double4>(mu);
  b.bnd = a.take<double2>(n);
  b.shift = a.take<double>(mu);
  b.g2p = a.take<int>(n);
  b.nbshift = a.take<float>(2 * (size_t)kMaxCells);  // 3^3 and 5^3 neighbourhoods
  b.part_d = a.take<double>((size_t)nchunks * mu);
  b.part_i = a.take<int>((size_t)nchunks * mu);
  b.sel = a.take<int>(mu);
  b.st = a.take<KmState>(1);
  b.cell_start = a.take<int>((size_t)kMaxCells + 1);
  b.cell_cen = a.take<double4>(mu);
  b.cell_of = a.take<int>(mu);
  b.pcell = a.take<int>(n);
  b.pd12 = a.take<double2>(n);
  return b;
}

// Exchange buffers of a sharded selection.
struct ShardBuffers {
  double4* send;  // (mu + 1): changed count, partial sums
  double4* recv;  // ranks x (mu + 1)
  double2* fsend;  // mu: nearest point per centroid
  double2* frecv;  // ranks x mu
};

ShardBuffers carve_shard(Arena& a, int mu, int ranks) {
  ShardBuffers b;
  b.send = a.take<double4>((size_t)mu + 1);
  b.recv = a.take<double4>((size_t)ranks * (mu + 1));
  b.fsend = a.take<double2>((size_t)mu);
  b.frecv = a.take<double2>((size_t)ranks * mu);
  return b;
}

}  // namespace

size_t kmeans_workspace_bytes(long long ng, int mu) {
  Arena a;
  a.counting = true;
  carve(a, (int)ng, mu);
  return a.off;
}

size_t kmeans_shard_workspace_bytes(long long ng, int mu, int ranks) {
  Arena a;
  a.counting = true;
  carve(a, (int)ng, mu);
  carve_shard(a, mu, ranks);
  return a.off;
}

int kmeans_weight(const double* d_psi, long long ng, int nocc, int nv1, int nc1, int nv2, int nc2,
                  double* d_w, cudaStream_t stream) {
  const int same = (nv1 == nv2 && nc1 == nc2);
  unsigned grid = grid_for(ng, 256);
  if (grid > (unsigned)kNumSMs * 16) grid = kNumSMs * 16;
  k_weight<<<grid, 256, 0, stream>>>(d_psi, ng, nocc - nv2, nocc + nc2, nocc - nv1, nocc + nc1,
                                     same, d_w);
  ISDF_CHECK_LAUNCH();
  return ISDF_OK;
}

// libstdc++'s std::random_shuffle(first, last) loop, driven by std::rand(),
// which the reference calls on its npt < mu branch (utility.cpp:679); draw()
// stands in for std::rand().
template <class Draw>
static void shuffle_like_libstdcxx(int* first, int* last, Draw draw) {
  if (first == last) return;
  for (int* i = first + 1; i != last; ++i) {
    int* j = first + draw() % ((i - first) + 1);
    if (i != j) std::swap(*i, *j);
  }
}
static void shuffle_like_libstdcxx(int* first, int* last) {
  shuffle_like_libstdcxx(first, last, [] { return std::rand(); });
}

// The sequence std::rand() gives after std::srand(seed), from glibc's own
// generator on a private state (initstate_r / random_r, the generator behind
// rand()), so that ranks sharing one process do not share their draws.
struct SeededRand {
  random_data data;
  char state[128];
  explicit SeededRand(unsigned seed) {
    std::memset(&data, 0, sizeof(data));
    std::memset(state, 0, sizeof(state));
    initstate_r(seed, state, sizeof(state), &data);
  }
  int operator()() {
    int32_t r = 0;
    random_r(&data, &r);
    return (int)r;
  }
};

int kmeans_select(const KmeansArgs& args, Arena& arena, cudaStream_t stream, KmeansResult* res,
                  Transport* shard) {
  const int n = (int)args.ng;
  const int mu = args.mu;
  if (n <= 0 || mu <= 0 || mu > kKmeansMaxMu) return record_error(ISDF_ERR_ARG, "kmeans: bad n/mu");
  if (args.ng > 0x7fffffffLL) return record_error(ISDF_ERR_UNSUPPORTED, "kmeans: Ng >= 2^31");
  const int ranks = shard ? shard->size : 1;
  if (ranks > kKmeansMaxRanks || ranks > n)
    return record_error(ISDF_ERR_UNSUPPORTED, "kmeans: more ranks than supported or points");
  KmBuffers b = carve(arena, n, mu);
  ShardBuffers sb{};
  if (shard) sb = carve_shard(arena, mu, ranks);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "kmeans: workspace too small");
  // this rank's points of the n-long list (utility.cpp:682-689); all of them at one rank
  const int lo = shard ? (int)block_start(n, ranks, shard->rank) : 0;
  const int cnt = shard ? (int)block_count(n, ranks, shard->rank) : n;
  const int ntiles = (n + kTile - 1) / kTile;
  const int nfilter = (n + 1023) / 1024;
  const int nchunks = (n + kFinalChunk - 1) / kFinalChunk;
  // a rank of a sharded selection draws from its own generator (below)
  if (args.rand_seed >= 0 && !shard) std::srand((unsigned)args.rand_seed);
  // warm start: the caller's previous pivots, read before piv is rewritten
  std::vector<int> prev;
  if (args.warm && n > 1 && args.piv[0] != args.piv[1]) {
    prev.assign(args.piv, args.piv + mu);
    for (int v : prev)
      if (v < 0 || v >= n) return record_error(ISDF_ERR_ARG, "kmeans: warm-start pivot outside the grid");
  }
  res->warm_pivots = -1;

  // filter: maxW, kept-point compaction, zero tail
  ISDF_CUDA(cudaMemsetAsync(b.st, 0, sizeof(KmState), stream));
  ISDF_CUDA(cudaMemsetAsync(b.pidx, 0, sizeof(int) * (size_t)n, stream));
  k_maxw<<<kNumSMs * 4, 256, 0, stream>>>(args.d_w, n, b.st);
  k_filter_count<<<nfilter, 256, 0, stream>>>(args.d_w, n, b.st, b.tile_cnt);
  k_scan_small<<<1, 1024, 0, stream>>>(b.tile_cnt, nfilter, &b.st->npt);
  k_filter_scatter<<<nfilter, 256, 0, stream>>>(args.d_w, n, b.st, b.tile_cnt, b.pidx);
  ISDF_CHECK_LAUNCH();
  KmState hst;
  ISDF_TRY(read_back(&hst, b.st, sizeof(KmState), stream));
  const int npt = hst.npt;
  res->npt = npt;
  std::memset(args.piv, 0, sizeof(int) * (size_t)n);

  if (npt < mu) {
    // utility.cpp:667-681: piv from the kept list, then a shuffled tail.
    std::vector<int> index(n, 0);
    ISDF_TRY(read_back(index.data(), b.pidx, sizeof(int) * (size_t)npt, stream));
    int k0 = 0, k1 = 0;
    for (int i = 0; i < npt; i++) {
      if (i == index[k0]) {
        args.piv[k0] = i;
        k0 = std::min(k0 + 1, mu - 1);
      } else {
        args.piv[npt + k1] = i;
        k1++;
      }
    }
    if (shard) {
      // every rank process of the reference starts from libc's initial
      // state (seed 1) unless the caller seeds it
      SeededRand draw(args.rand_seed >= 0 ? (unsigned)args.rand_seed : 1u);
      shuffle_like_libstdcxx(args.piv + npt, args.piv + n, [&] { return draw(); });
    } else {
      shuffle_like_libstdcxx(args.piv + npt, args.piv + n);
    }
    res->rk_eff = mu;
    res->iters = -1;
    res->launches = 4 + (readback_mailbox() ? 2 : 0);
    return ISDF_OK;
  }

  const double dx0 = args.length[0] / args.num_grid[0];
  const double dx1 = args.length[1] / args.num_grid[1];
  const double dx2 = args.length[2] / args.num_grid[2];
  std::vector<int> cinit;
  if (!prev.empty()) {
    // utility.cpp:725-749: the previous pivots whose weight passes the
    // filter, in their order, then the first kept points not among them
    // (at most mu kept points are examined: each one either joins or is
    // one of the kept previous pivots)
    ISDF_CUDA(cudaMemcpyAsync(b.sel, prev.data(), sizeof(int) * (size_t)mu,
                              cudaMemcpyHostToDevice, stream));
    k_gather_w<<<grid_for(mu, 256), 256, 0, stream>>>(args.d_w, b.sel, mu, b.part_d);
    ISDF_CHECK_LAUNCH();
    std::vector<double> wprev(mu);
    std::vector<int> head(mu);
    ISDF_TRY(read_back(wprev.data(), b.part_d, sizeof(double) * (size_t)mu, stream));
    ISDF_TRY(read_back(head.data(), b.pidx, sizeof(int) * (size_t)mu, stream));
    double maxw;
    std::memcpy(&maxw, &hst.maxw_bits, sizeof(double));
    const double thr = 1e-8 * maxw;
    cinit.reserve(mu);
    for (int i = 0; i < mu; ++i)
      if (wprev[i] > thr) cinit.push_back(prev[i]);
    res->warm_pivots = (int)cinit.size();
    std::vector<char> in((size_t)n, 0);
    for (int c : cinit) in[c] = 1;
    for (int k = 0; (int)cinit.size() < mu && k < mu; ++k)
      if (!in[head[k]]) cinit.push_back(head[k]);
    ISDF_CUDA(cudaMemcpyAsync(b.sel, cinit.data(), sizeof(int) * (size_t)mu,
                              cudaMemcpyHostToDevice, stream));
  }
  k_points<<<grid_for(n, 256), 256, 0, stream>>>(b.pidx, args.d_w, n, args.num_grid[0],
                                                 args.num_grid[1], dx0, dx1, dx2, b.px, b.py,
                                                 b.pz, b.pw, mu, b.cen);
  if (!prev.empty())
    k_warm_centroids<<<grid_for(mu, 256), 256, 0, stream>>>(b.sel, mu, args.num_grid[0],
                                                            args.num_grid[1], dx0, dx1, dx2,
                                                            b.cen);
  {
    KmState init{};
    init.flag = n;
    init.rk = mu;
    init.npt = npt;
    init.maxw_bits = hst.maxw_bits;
    ISDF_CUDA(cudaMemcpyAsync(b.st, &init, sizeof(KmState), cudaMemcpyHostToDevice, stream));
  }
  CellGrid cg;
  {
    int nc = (int)std::lround(std::cbrt(mu / 1.5));
    nc = std::max(1, std::min(nc, kMaxCellsPerDim));
    cg.nc = nc;
    double lmax = 0.0;
    for (int i = 0; i < 3; ++i) {
      cg.h[i] = args.length[i] / nc;
      lmax = std::max(lmax, std::fabs(args.length[i]));
    }
    cg.tol = 1e-9 * lmax;
  }
  const size_t cell_smem = sizeof(int) * ((size_t)cg.nc * cg.nc * cg.nc + 1);
  AssignMap am{};
  am.nx = args.num_grid[0];
  am.ny = args.num_grid[1];
  am.nz = args.num_grid[2];
  am.nbx = (am.nx + 3) / 4;
  am.nby = (am.ny + 3) / 4;
  am.nbt = (long long)am.nbx * am.nby * ((am.nz + 1) / 2) * 32;
  am.t0 = 0;
  am.npt = npt;
  am.n = n;
  am.p_lo = lo;
  am.p_hi = lo + cnt;
  am.brick = ((long long)am.nx * am.ny * am.nz == n && am.nbt + n < 0x7fffffffLL);
  am.g2p = nullptr;
  if (am.brick && npt < n) {
    ISDF_CUDA(cudaMemsetAsync(b.g2p, 0xff, sizeof(int) * (size_t)n, stream));
    k_grid_to_point<<<grid_for(npt, 256), 256, 0, stream>>>(b.pidx, npt, b.g2p);
    am.g2p = b.g2p;
  }
  const int kept_hi = std::min(lo + cnt, npt);  // this rank's kept points: [lo, kept_hi)
  const int tail_loc = std::max(0, lo + cnt - std::max(npt, lo));
  if (am.brick && shard) {
    // the bricks of the z planes that hold this rank's kept points
    if (lo < kept_hi) {
      int ends[2];
      ISDF_TRY(read_back(&ends[0], b.pidx + lo, sizeof(int), stream));
      ISDF_TRY(read_back(&ends[1], b.pidx + kept_hi - 1, sizeof(int), stream));
      const long long plane = (long long)am.nx * am.ny;
      const long long bz0 = ends[0] / plane / 2, bz1 = ends[1] / plane / 2;
      const long long per_bz = (long long)am.nbx * am.nby * 32;
      am.t0 = bz0 * per_bz;
      am.nbt = (bz1 - bz0 + 1) * per_bz;
    } else {
      am.nbt = 0;
    }
  }
  const unsigned pgrid = am.brick ? grid_for(am.nbt + tail_loc, kAssignThreads)
                                  : grid_for(cnt, kAssignThreads);
  k_point_cells<<<grid_for(n, 256), 256, 0, stream>>>(b.px, b.py, b.pz, n, cg, b.pcell, b.pd12);
  k_build_cells<<<1, 1024, cell_smem, stream>>>(b.cen, b.st, cg, b.cell_start, b.cell_cen,
                                                b.cell_of);
  k_assign_warp<<<pgrid, kAssignThreads, 0, stream>>>(b.px, b.py, b.pz, n, b.cen, b.cell_start,
                                                      b.cell_cen, cg, am, b.st, b.label, 0,
                                                      b.bnd, b.shift, b.nbshift, b.pcell,
                                                      b.pd12);
  ISDF_CHECK_LAUNCH();

  const size_t cmax_smem = 3 * sizeof(unsigned) * ((size_t)cg.nc * cg.nc * cg.nc);
  const double max_f = 1e-5 * n;  // KmeansTolerance * n (utility.cpp:812)
  const size_t hist_smem = sizeof(int) * (size_t)mu;
  const size_t scatter_smem = sizeof(int) * ((size_t)mu + kTile);
  ISDF_TRY(set_kmeans_smem_attrs());
  int chunks = 0;
  const int max_chunks = args.max_iter / kIterChunk + 2;
  // One chunk = kIterChunk Lloyd iterations (10 launches each; every kernel
  // returns at once when the loop has stopped). The chunk is captured once
  // into a CUDA graph and replayed, which removes the per-launch host cost
  // that dominates small solves; direct launches are the fallback when the
  // stream cannot be captured.
  auto launch_chunk = [&]() {
    for (int it = 0; it < kIterChunk; ++it) {
      k_iter_begin<<<1, 1, 0, stream>>>(b.st, max_f, args.max_iter);
      k_hist<<<ntiles, 256, hist_smem, stream>>>(b.label, n, b.st, b.hist);
      k_hist_scan<<<(mu + 31) / 32, 32 * kScanWarps, 0, stream>>>(b.hist, ntiles, b.st, b.members);
      k_label_start<<<1, 1024, 0, stream>>>(b.members, b.st, b.start);
      k_scatter<<<ntiles, 128, scatter_smem, stream>>>(b.label, n, b.st, b.hist, b.start, b.px,
                                                       b.py, b.pz, b.pw, b.sorted);
      k_segsum<<<grid_for(mu, 8), 256, 0, stream>>>(b.sorted, b.start, b.members, b.px, b.py,
                                                    b.pz, b.pw, b.label, n, npt, 1, b.st, b.sums);
      k_centroids<<<1, 1024, cmax_smem, stream>>>(b.sums, b.st, b.cen, b.shift, b.cell_of, cg,
                                                  b.nbshift);
      k_build_cells<<<1, 1024, cell_smem, stream>>>(b.cen, b.st, cg, b.cell_start, b.cell_cen,
                                                    b.cell_of);
      k_assign_warp<<<pgrid, kAssignThreads, 0, stream>>>(b.px, b.py, b.pz, n, b.cen,
                                                          b.cell_start, b.cell_cen, cg, am, b.st,
                                                          b.label, 1, b.bnd, b.shift, b.nbshift,
                                                          b.pcell, b.pd12);
      k_iter_end<<<1, 1, 0, stream>>>(b.st, 1);
    }
  };
  // Sharded: the rank folds its own points [lo, lo + cnt) (utility.cpp:813-822),
  // the ranks exchange their partial sums and changed-label counts (one
  // all-gather per iteration, utility.cpp:825-826,908-917), and every rank
  // combines them in the same order, so that all ranks hold the same
  // centroids without a broadcast. Its collectives keep the chunk out of a
  // CUDA graph.
  const int ntl = (cnt + kTile - 1) / kTile;
  const int npt_loc = std::max(0, std::min(npt - lo, cnt));
  const size_t rec_bytes = sizeof(double4) * ((size_t)mu + 1);
  std::vector<size_t> rcounts(ranks, rec_bytes), rdispls(ranks);
  for (int q = 0; q < ranks; ++q) rdispls[q] = (size_t)q * rec_bytes;
  auto launch_chunk_sharded = [&]() -> int {
    for (int it = 0; it < kIterChunk; ++it) {
      k_hist<<<ntl, 256, hist_smem, stream>>>(b.label + lo, cnt, b.st, b.hist);
      k_hist_scan<<<(mu + 31) / 32, 32 * kScanWarps, 0, stream>>>(b.hist, ntl, b.st, b.members);
      k_label_start<<<1, 1024, 0, stream>>>(b.members, b.st, b.start);
      k_scatter<<<ntl, 128, scatter_smem, stream>>>(b.label + lo, cnt, b.st, b.hist, b.start,
                                                    b.px + lo, b.py + lo, b.pz + lo, b.pw + lo,
                                                    b.sorted);
      k_segsum<<<grid_for(mu, 8), 256, 0, stream>>>(b.sorted, b.start, b.members, b.px + lo,
                                                    b.py + lo, b.pz + lo, b.pw + lo, b.label + lo,
                                                    cnt, npt_loc, 0, b.st, sb.send + 1);
      k_shard_header<<<1, 1, 0, stream>>>(b.st, sb.send);
      ISDF_CHECK_LAUNCH();
      ISDF_TRY(shard->allgatherv(sb.send, rec_bytes, sb.recv, rcounts.data(), rdispls.data(),
                                 stream));
      k_shard_begin<<<1, 1, 0, stream>>>(b.st, sb.recv, ranks, mu + 1, max_f, args.max_iter);
      k_shard_sums<<<grid_for(mu, 128), 128, 0, stream>>>(b.st, sb.recv, ranks, mu + 1, b.sums);
      k_centroids<<<1, 1024, cmax_smem, stream>>>(b.sums, b.st, b.cen, b.shift, b.cell_of, cg,
                                                  b.nbshift);
      k_build_cells<<<1, 1024, cell_smem, stream>>>(b.cen, b.st, cg, b.cell_start, b.cell_cen,
                                                    b.cell_of);
      k_assign_warp<<<pgrid, kAssignThreads, 0, stream>>>(b.px, b.py, b.pz, n, b.cen,
                                                          b.cell_start, b.cell_cen, cg, am, b.st,
                                                          b.label, 1, b.bnd, b.shift, b.nbshift,
                                                          b.pcell, b.pd12);
      k_iter_end<<<1, 1, 0, stream>>>(b.st, 0);
      ISDF_CHECK_LAUNCH();
    }
    return ISDF_OK;
  };
  cudaGraphExec_t exec = nullptr;
  if (!shard) {
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
      launch_chunk();
      if (cudaStreamEndCapture(stream, &graph) == cudaSuccess && graph) {
        if (cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
        cudaGraphDestroy(graph);
      }
    }
    (void)cudaGetLastError();  // a refused capture leaves an error to clear
  }
  struct ExecGuard {
    cudaGraphExec_t e;
    ~ExecGuard() {
      if (e) cudaGraphExecDestroy(e);
    }
  } guard{exec};
  for (;;) {
    if (shard) ISDF_TRY(launch_chunk_sharded());
    else if (exec) ISDF_CUDA(cudaGraphLaunch(exec, stream));
    else launch_chunk();
    ISDF_CHECK_LAUNCH();
    ISDF_TRY(read_back(&hst, b.st, sizeof(KmState), stream));
    if (hst.done) break;
    if (++chunks > max_chunks) return record_error(ISDF_ERR_CUDA, "kmeans: loop did not stop");
  }
  res->iters = hst.s;
  res->search_frac = (double)hst.searches / ((double)cnt * (hst.s + 1));
  // + the state, per-chunk and selection reads through the mapped mailbox
  res->launches =
      4 + 4 + (am.g2p ? 1 : 0) + (chunks + 1) * kIterChunk * (shard ? 12 : 10) + 2 +
      (readback_mailbox() ? chunks + 3 : 0);
  const int rk = hst.rk;

  if (!shard) {
    dim3 fgrid((unsigned)((rk + 127) / 128), (unsigned)nchunks);
    k_final_partial<<<fgrid, 128, 0, stream>>>(b.px, b.py, b.pz, n, b.cen, b.st, b.part_d,
                                               b.part_i);
    k_final_reduce<<<grid_for(rk, 128), 128, 0, stream>>>(b.part_d, b.part_i, nchunks, b.st,
                                                          b.pidx, b.sel);
  } else {
    // each rank's first minimum over its points, then MINLOC over the ranks
    const int nch = (cnt + kFinalChunk - 1) / kFinalChunk;
    dim3 fgrid((unsigned)((rk + 127) / 128), (unsigned)nch);
    k_final_partial<<<fgrid, 128, 0, stream>>>(b.px + lo, b.py + lo, b.pz + lo, cnt, b.cen, b.st,
                                               b.part_d, b.part_i);
    k_final_local<<<grid_for(rk, 128), 128, 0, stream>>>(b.part_d, b.part_i, nch, b.st,
                                                         b.pidx + lo, sb.fsend);
    ISDF_CHECK_LAUNCH();
    const size_t fb = sizeof(double2) * (size_t)mu;
    std::vector<size_t> fc(ranks, fb), fd(ranks);
    for (int q = 0; q < ranks; ++q) fd[q] = (size_t)q * fb;
    ISDF_TRY(shard->allgatherv(sb.fsend, fb, sb.frecv, fc.data(), fd.data(), stream));
    k_minloc<<<grid_for(rk, 128), 128, 0, stream>>>(sb.frecv, ranks, mu, b.st, b.sel);
  }
  ISDF_CHECK_LAUNCH();
  std::vector<int> sel(rk);
  ISDF_TRY(read_back(sel.data(), b.sel, sizeof(int) * (size_t)rk, stream));
  // unique (utility.cpp:617-629) and piv (utility.cpp:973-983)
  std::sort(sel.begin(), sel.end());
  sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
  const int rk_eff = (int)sel.size();
  int k0 = 0, k1 = 0;
  for (int i = 0; i < n; i++) {
    if (i == sel[k0]) {
      args.piv[k0] = i;
      k0 = std::min(k0 + 1, rk_eff - 1);
    } else {
      args.piv[rk_eff + k1] = i;
      k1++;
    }
  }
  res->rk_eff = rk_eff;
  return ISDF_OK;
}

// ===================================================================== batched small selections
// Several small K-means selections in one cooperative launch (the serving
// loop's batches of small requests): a group of G CTAs runs one request's
// whole Lloyd loop - assignment, stable counting sort by label, sequential
// per-cluster folds, centroid update with the empty-cluster compaction, the
// change count and the final nearest point per centroid - with software group
// barriers between the phases, so a batch of B requests costs one launch
// instead of ~10 launches per iteration per request. The arithmetic and every
// order of summation are the single-request path's (and the reference's,
// utility.cpp:813-945): piv is the same bit for bit. The assignment is a
// brute-force scan over the centroids held in shared memory, which suits the
// small systems this path serves (mu <= 512).
namespace {

constexpr int kBatchThreads = 256;
constexpr int kBatchWarps = kBatchThreads / 32;

struct KmBatchJob {
  const double *px, *py, *pz, *pw;
  const int* pidx;
  int* label;
  double4* sorted;
  double4* cen;
  double4* sums;
  int* hist;   // per sub-block label counts, then each sub-block's first slot per label
  int* tot;    // members per cluster
  int* sel;    // grid index of the nearest point per centroid
  int n, npt, mu, max_iter;
  double max_f;
  int rk, iters, err, any_empty;
  int changed[2];
  unsigned bar_count, bar_gen;
};

// All CTAs of one request's group meet here. Bounded: a CTA that waits
// longer than ~1 s sets err and returns false, and so does every CTA that
// sees err afterwards, so a failing group ends instead of hanging.
__device__ bool group_barrier(KmBatchJob* J, int G) {
  __shared__ int ok_s;
  __syncthreads();
  if (threadIdx.x == 0) {
    int ok = 1;
    __threadfence();
    const unsigned gen = *(volatile unsigned*)&J->bar_gen;
    if (atomicAdd(&J->bar_count, 1u) == (unsigned)G - 1) {
      J->bar_count = 0;
      __threadfence();
      atomicAdd(&J->bar_gen, 1u);
    } else {
      long long spins = 0;
      while (*(volatile unsigned*)&J->bar_gen == gen) {
        if (++spins > (1LL << 24)) {
          atomicExch(&J->err, 1);
          ok = 0;
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    ok_s = ok && *(volatile int*)&J->err == 0;
  }
  __syncthreads();
  return ok_s != 0;
}

// Loads of data that other CTAs of the launch wrote: through L2 (L1 is not
// coherent across SMs within a kernel).
__device__ __forceinline__ double4 ldcg4(const double4* p) {
  const double* d = reinterpret_cast<const double*>(p);
  return make_double4(__ldcg(d), __ldcg(d + 1), __ldcg(d + 2), __ldcg(d + 3));
}

// Exclusive scan of v[0..m) (m <= kKmeansBatchMaxMu) into out, one block.
__device__ void block_scan(const int* v, int m, int* out) {
  __shared__ int part[kBatchThreads];
  const int per = (m + kBatchThreads - 1) / kBatchThreads;
  const int lo = min(m, (int)threadIdx.x * per), hi = min(m, lo + per);
  int t = 0;
  for (int i = lo; i < hi; ++i) t += __ldcg(v + i);
  part[threadIdx.x] = t;
  __syncthreads();
  if (threadIdx.x == 0) {
    int run = 0;
    for (int i = 0; i < kBatchThreads; ++i) {
      const int x = part[i];
      part[i] = run;
      run += x;
    }
  }
  __syncthreads();
  int run = part[threadIdx.x];
  for (int i = lo; i < hi; ++i) {
    out[i] = run;
    run += __ldcg(v + i);
  }
  __syncthreads();
}

__global__ void __launch_bounds__(kBatchThreads) k_kmeans_batch(KmBatchJob* jobs, int G) {
  KmBatchJob* J = jobs + blockIdx.x / G;
  const int c = blockIdx.x % G;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __shared__ double cx[kKmeansBatchMaxMu], cy[kKmeansBatchMaxMu], cz[kKmeansBatchMaxMu];
  __shared__ int run[kBatchWarps][kKmeansBatchMaxMu];
  __shared__ int sstart[kKmeansBatchMaxMu];
  __shared__ int red[kBatchWarps];
  const int n = J->n, npt = J->npt;
  const int nsub = G * kBatchWarps;
  const int per = (n + nsub - 1) / nsub;
  const int sb = c * kBatchWarps + warp;
  const int sb_lo = min(n, sb * per), sb_hi = min(n, sb_lo + per);
  const int cta_lo = min(n, c * kBatchWarps * per), cta_hi = min(n, cta_lo + kBatchWarps * per);
  volatile KmBatchJob* VJ = J;

  auto load_cen = [&](int rk) {
    for (int i = threadIdx.x; i < rk; i += kBatchThreads) {
      const double4 q = ldcg4(J->cen + i);
      cx[i] = q.x;
      cy[i] = q.y;
      cz[i] = q.z;
    }
    __syncthreads();
  };
  // labels of this CTA's points (first minimum, pdist2's rounding); returns
  // the number of labels that changed (valid in thread 0)
  auto assign = [&](int rk) -> int {
    int ch = 0;
    for (int p = cta_lo + threadIdx.x; p < cta_hi; p += kBatchThreads) {
      const double x = J->px[p], y = J->py[p], z = J->pz[p];
      double best = ref_dist2(x, y, z, make_double4(cx[0], cy[0], cz[0], 0.0));
      int bj = 0;
      for (int j = 1; j < rk; ++j) {
        const double d = ref_dist2(x, y, z, make_double4(cx[j], cy[j], cz[j], 0.0));
        if (d < best) {
          best = d;
          bj = j;
        }
      }
      if (__ldcg(J->label + p) != bj) ++ch;
      J->label[p] = bj;
    }
    for (int o = 16; o > 0; o >>= 1) ch += __shfl_xor_sync(0xffffffffu, ch, o);
    if (lane == 0) red[warp] = ch;
    __syncthreads();
    int t = 0;
    if (threadIdx.x == 0)
      for (int w = 0; w < kBatchWarps; ++w) t += red[w];
    __syncthreads();
    return t;
  };

  int rk = J->mu;
  load_cen(rk);
  assign(rk);
  if (!group_barrier(J, G)) return;
  int flag = n, s = 0;
  while ((double)flag > J->max_f && s < J->max_iter) {
    const int par = s & 1;
    // 1. label counts per sub-block (one warp each)
    for (int k = lane; k < rk; k += 32) run[warp][k] = 0;
    __syncwarp();
    for (int p = sb_lo + lane; p < sb_hi; p += 32) atomicAdd(&run[warp][__ldcg(J->label + p)], 1);
    __syncwarp();
    for (int k = lane; k < rk; k += 32) J->hist[(size_t)sb * kKmeansBatchMaxMu + k] = run[warp][k];
    if (!group_barrier(J, G)) return;
    // 2. per cluster, each sub-block's offset within the cluster and the
    // cluster's size (every CTA has read last iteration's change count)
    if (c == 0 && threadIdx.x == 0) {
      VJ->changed[par ^ 1] = 0;
      VJ->any_empty = 0;
    }
    for (int k = c + G * threadIdx.x; k < rk; k += G * kBatchThreads) {
      int acc = 0;
      for (int q = 0; q < nsub; ++q) {
        int* h = J->hist + (size_t)q * kKmeansBatchMaxMu + k;
        const int v = __ldcg(h);
        *h = acc;
        acc += v;
      }
      J->tot[k] = acc;
    }
    if (!group_barrier(J, G)) return;
    // 3. stable scatter of (w x, w y, w z, w) into cluster order
    block_scan(J->tot, rk, sstart);
    for (int k = lane; k < rk; k += 32)
      run[warp][k] = sstart[k] + __ldcg(J->hist + (size_t)sb * kKmeansBatchMaxMu + k);
    __syncwarp();
    for (int base = sb_lo; base < sb_hi; base += 32) {
      const int p = base + lane;
      const bool ok = p < sb_hi;
      const int l = ok ? __ldcg(J->label + p) : -1;
      const unsigned peers = __match_any_sync(0xffffffffu, l);
      const int b = ok ? run[warp][l] : 0;
      __syncwarp();
      if (ok) {
        const double w = J->pw[p];
        const int r = __popc(peers & ((1u << lane) - 1u));
        J->sorted[b + r] = make_double4(rmul(w, J->px[p]), rmul(w, J->py[p]), rmul(w, J->pz[p]), w);
        if (lane == __ffs(peers) - 1) run[warp][l] = b + __popc(peers);
      }
      __syncwarp();
    }
    if (!group_barrier(J, G)) return;
    // 4. per cluster and component, the sequential fold in point order; the
    // zero tail (copies of grid point 0, last in their cluster) by repeat_add
    const int tail_label = npt < n ? __ldcg(J->label + npt) : -1;
    for (int kq = c * kBatchThreads + threadIdx.x; kq < 4 * rk; kq += G * kBatchThreads) {
      const int k = kq >> 2, q = kq & 3;
      int m = __ldcg(J->tot + k);
      long long tail = 0;
      if (k == tail_label) {
        tail = n - npt;
        m -= (int)tail;
      }
      const double* v = reinterpret_cast<const double*>(J->sorted + sstart[k]) + q;
      double acc = 0.0;
      for (int e = 0; e < m; ++e) acc = radd(acc, __ldcg(v + (size_t)e * 4));
      if (tail) {
        const double w0 = J->pw[npt];
        const double val = q == 3 ? w0 : rmul(w0, q == 0 ? J->px[npt] : q == 1 ? J->py[npt] : J->pz[npt]);
        acc = repeat_add(acc, val, tail);
      }
      reinterpret_cast<double*>(J->sums + k)[q] = acc;
      if (q == 3 && acc == 0.0) VJ->any_empty = 1;
    }
    if (!group_barrier(J, G)) return;
    // 5. new centroids = sums / count; an empty cluster takes the last one's
    // sums and rk shrinks (utility.cpp:831-853), in order, by one thread
    if (c == 0) {
      if (!VJ->any_empty) {
        for (int i = threadIdx.x; i < rk; i += kBatchThreads) {
          const double4 q = ldcg4(J->sums + i);
          J->cen[i] = make_double4(rdiv(q.x, q.w), rdiv(q.y, q.w), rdiv(q.z, q.w), 0.0);
        }
      } else if (threadIdx.x == 0) {
        int r = rk;
        for (int i = 0; i < r; i++) {
          const double4 q = ldcg4(J->sums + i);
          if (q.w != 0.0) {
            J->sums[i] = make_double4(rdiv(q.x, q.w), rdiv(q.y, q.w), rdiv(q.z, q.w), q.w);
          } else {
            r--;
            J->sums[i] = ldcg4(J->sums + r);
            i--;
          }
        }
        for (int i = 0; i < r; i++) {
          const double4 q = ldcg4(J->sums + i);
          J->cen[i] = make_double4(q.x, q.y, q.z, 0.0);
        }
        VJ->rk = r;
      }
    }
    if (!group_barrier(J, G)) return;
    // 6. reassignment and the change count
    rk = VJ->rk;
    load_cen(rk);
    const int ch = assign(rk);
    if (threadIdx.x == 0 && ch) atomicAdd(&J->changed[par], ch);
    if (!group_barrier(J, G)) return;
    flag = VJ->changed[par];
    ++s;
  }
  // nearest point to every centroid (first minimum over points), one warp each
  load_cen(rk);
  for (int j = c * kBatchWarps + warp; j < rk; j += nsub) {
    const double4 q = make_double4(cx[j], cy[j], cz[j], 0.0);
    double best = __longlong_as_double(0x7ff0000000000000LL);
    int bi = 0x7fffffff;
    for (int p = lane; p < n; p += 32) {
      const double d = ref_dist2(J->px[p], J->py[p], J->pz[p], q);
      if (d < best) {
        best = d;
        bi = p;
      }
    }
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob < best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    if (lane == 0) J->sel[j] = J->pidx[bi];
  }
  if (c == 0 && threadIdx.x == 0) VJ->iters = s;
}

struct BatchBuffers {
  int* pidx;
  double *px, *py, *pz, *pw;
  int* label;
  double4 *sorted, *cen, *sums;
  int *hist, *tot, *sel, *tile_cnt;
  KmState* st;
};

BatchBuffers carve_batch(Arena& a, int n, int G) {
  BatchBuffers b;
  const int nfilter = (n + 1023) / 1024;
  b.pidx = a.take<int>(n);
  b.px = a.take<double>(n);
  b.py = a.take<double>(n);
  b.pz = a.take<double>(n);
  b.pw = a.take<double>(n);
  b.label = a.take<int>(n);
  b.sorted = a.take<double4>(n);
  b.cen = a.take<double4>(kKmeansBatchMaxMu);
  b.sums = a.take<double4>(kKmeansBatchMaxMu);
  b.hist = a.take<int>((size_t)G * kBatchWarps * kKmeansBatchMaxMu);
  b.tot = a.take<int>(kKmeansBatchMaxMu);
  b.sel = a.take<int>(kKmeansBatchMaxMu);
  b.tile_cnt = a.take<int>(nfilter);
  b.st = a.take<KmState>(1);
  return b;
}

constexpr int kBatchMaxGroup = 16;  // CTAs per request

int batch_group(long long n) {
  long long g = (n + 4095) / 4096;
  return (int)std::max(1LL, std::min((long long)kBatchMaxGroup, g));
}

}  // namespace

// piv = [distinct selected points ascending | the rest ascending]
// (unique, utility.cpp:617-629, and utility.cpp:973-983); returns rk_eff.
static int piv_from_selection(std::vector<int>& sel, int n, int* piv) {
  std::sort(sel.begin(), sel.end());
  sel.erase(std::unique(sel.begin(), sel.end()), sel.end());
  const int rk_eff = (int)sel.size();
  int k0 = 0, k1 = 0;
  for (int i = 0; i < n; i++) {
    if (i == sel[k0]) {
      piv[k0] = i;
      k0 = std::min(k0 + 1, rk_eff - 1);
    } else {
      piv[rk_eff + k1] = i;
      k1++;
    }
  }
  return rk_eff;
}

size_t kmeans_batch_workspace_bytes(long long ng, int mu) {
  (void)mu;
  Arena a;
  a.counting = true;
  // the histogram sized for the largest group: a batch runs every request
  // with the largest group any of its requests needs
  carve_batch(a, (int)ng, kBatchMaxGroup);
  a.take<KmBatchJob>(1);
  return a.off + 512;
}

int kmeans_select_batch(const KmeansArgs* args, int count, Arena& arena, cudaStream_t stream,
                        KmeansResult* res) {
  if (count <= 0) return ISDF_OK;
  int G = 1;
  for (int r = 0; r < count; ++r) {
    const KmeansArgs& a = args[r];
    if (a.ng <= 1 || a.ng > kKmeansBatchMaxNg || a.mu <= 0 || a.mu > kKmeansBatchMaxMu ||
        a.mu > a.ng || a.max_iter < 0 || a.warm)
      return record_error(ISDF_ERR_UNSUPPORTED, "kmeans batch: request outside the batched sizes");
    G = std::max(G, batch_group(a.ng));
  }
  std::vector<BatchBuffers> bufs(count);
  for (int r = 0; r < count; ++r) bufs[r] = carve_batch(arena, (int)args[r].ng, G);
  KmBatchJob* d_jobs = arena.take<KmBatchJob>((size_t)count);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "kmeans batch: workspace too small");
  // filter: maxW, kept-point compaction, zero tail (per request)
  for (int r = 0; r < count; ++r) {
    const int n = (int)args[r].ng;
    const int nfilter = (n + 1023) / 1024;
    const BatchBuffers& b = bufs[r];
    ISDF_CUDA(cudaMemsetAsync(b.st, 0, sizeof(KmState), stream));
    ISDF_CUDA(cudaMemsetAsync(b.pidx, 0, sizeof(int) * (size_t)n, stream));
    k_maxw<<<kNumSMs * 4, 256, 0, stream>>>(args[r].d_w, n, b.st);
    k_filter_count<<<nfilter, 256, 0, stream>>>(args[r].d_w, n, b.st, b.tile_cnt);
    k_scan_small<<<1, 1024, 0, stream>>>(b.tile_cnt, nfilter, &b.st->npt);
    k_filter_scatter<<<nfilter, 256, 0, stream>>>(args[r].d_w, n, b.st, b.tile_cnt, b.pidx);
  }
  ISDF_CHECK_LAUNCH();
  std::vector<KmBatchJob> jobs;
  std::vector<int> slot;  // request of each batched job
  for (int r = 0; r < count; ++r) {
    const KmeansArgs& a = args[r];
    const int n = (int)a.ng, mu = a.mu;
    const BatchBuffers& b = bufs[r];
    KmState hst;
    ISDF_TRY(read_back(&hst, b.st, sizeof(KmState), stream));
    res[r] = KmeansResult();
    res[r].npt = hst.npt;
    if (a.rand_seed >= 0) std::srand((unsigned)a.rand_seed);
    std::memset(a.piv, 0, sizeof(int) * (size_t)n);
    if (hst.npt < mu) {
      // utility.cpp:667-681: piv from the kept list, then a shuffled tail
      std::vector<int> index(n, 0);
      ISDF_TRY(read_back(index.data(), b.pidx, sizeof(int) * (size_t)hst.npt, stream));
      int k0 = 0, k1 = 0;
      for (int i = 0; i < hst.npt; i++) {
        if (i == index[k0]) {
          a.piv[k0] = i;
          k0 = std::min(k0 + 1, mu - 1);
        } else {
          a.piv[hst.npt + k1] = i;
          k1++;
        }
      }
      shuffle_like_libstdcxx(a.piv + hst.npt, a.piv + n);
      res[r].rk_eff = mu;
      res[r].iters = -1;
      continue;
    }
    const double dx0 = a.length[0] / a.num_grid[0];
    const double dx1 = a.length[1] / a.num_grid[1];
    const double dx2 = a.length[2] / a.num_grid[2];
    k_points<<<grid_for(n, 256), 256, 0, stream>>>(b.pidx, a.d_w, n, a.num_grid[0], a.num_grid[1],
                                                   dx0, dx1, dx2, b.px, b.py, b.pz, b.pw, mu,
                                                   b.cen);
    ISDF_CUDA(cudaMemsetAsync(b.label, 0xff, sizeof(int) * (size_t)n, stream));
    KmBatchJob j;
    std::memset(&j, 0, sizeof(j));
    j.px = b.px;
    j.py = b.py;
    j.pz = b.pz;
    j.pw = b.pw;
    j.pidx = b.pidx;
    j.label = b.label;
    j.sorted = b.sorted;
    j.cen = b.cen;
    j.sums = b.sums;
    j.hist = b.hist;
    j.tot = b.tot;
    j.sel = b.sel;
    j.n = n;
    j.npt = hst.npt;
    j.mu = mu;
    j.max_iter = a.max_iter;
    j.max_f = 1e-5 * n;  // KmeansTolerance * n (utility.cpp:812)
    j.rk = mu;
    jobs.push_back(j);
    slot.push_back(r);
  }
  ISDF_CHECK_LAUNCH();
  if (jobs.empty()) return ISDF_OK;
  // every CTA of the launch must be resident at once (the group barriers)
  int dev = 0, per_sm = 0, coop = 0;
  ISDF_CUDA(cudaGetDevice(&dev));
  ISDF_CUDA(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return record_error(ISDF_ERR_UNSUPPORTED, "kmeans batch: no cooperative launch");
  int nsm = 0;
  ISDF_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
  ISDF_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_kmeans_batch, kBatchThreads, 0));
  const int max_jobs = std::max(1, per_sm * nsm / G);
  ISDF_CUDA(cudaMemcpyAsync(d_jobs, jobs.data(), sizeof(KmBatchJob) * jobs.size(),
                            cudaMemcpyHostToDevice, stream));
  for (size_t j0 = 0; j0 < jobs.size(); j0 += (size_t)max_jobs) {
    const int nj = (int)std::min<size_t>((size_t)max_jobs, jobs.size() - j0);
    KmBatchJob* dj = d_jobs + j0;
    int g = G;
    void* kargs[] = {(void*)&dj, (void*)&g};
    ISDF_CUDA(cudaLaunchCooperativeKernel((const void*)k_kmeans_batch, dim3((unsigned)(nj * G)),
                                          dim3(kBatchThreads), kargs, 0, stream));
  }
  std::vector<KmBatchJob> out(jobs.size());
  ISDF_TRY(read_back(out.data(), d_jobs, sizeof(KmBatchJob) * jobs.size(), stream));
  for (size_t j = 0; j < jobs.size(); ++j) {
    const int r = slot[j];
    if (out[j].err) return record_error(ISDF_ERR_TIMEOUT, "kmeans batch: a group barrier timed out");
    std::vector<int> sel(out[j].rk);
    ISDF_TRY(read_back(sel.data(), bufs[r].sel, sizeof(int) * sel.size(), stream));
    res[r].iters = out[j].iters;
    res[r].rk_eff = piv_from_selection(sel, (int)args[r].ng, args[r].piv);
    res[r].launches = 8 + (int)((jobs.size() + max_jobs - 1) / max_jobs);
  }
  return ISDF_OK;
}

}  // namespace isdf_b200
