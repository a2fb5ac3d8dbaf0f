// ISDF check on sm_100a: pair-density fit error and truncated-Coulomb error.
//
// Reference: src/common/checkcode.cpp:54-313 with src/common/fourier.cpp
// (host FFTW, full complex spectra). Same quantities:
//   fit error  = ||rho - theta C||_F / ||rho||_F, rho_ij(r) = psi_k(r) psi_j(r)
//   (ij|V|kl)  = Re sum_G conj(rho_ij(G)) V(G) rho_kl(G), forward FFTs scaled
//                by vol/Ng, V(G) = 4 pi R^2 (G = 0) or 8 pi/G^2 (1 - cos(G R)), R = 5
//   ISDF form  = C^T Re(zeta^H V zeta) C, zeta = FFT(theta columns)
//   Coulomb error = ||(ij|V|kl) - C^T A C||_F / ||(ij|V|kl)||_F.
// B200 form: cuFFT D2Z batched 3-D transforms (half spectra). For real
// functions the full-grid sum equals the half-spectrum sum with weight 2 on
// every x-frequency that is not self-conjugate, so with
//   Y(pair, k) = sqrt(w_k V_k) * (vol/Ng) * [Re F_k | Im F_k]
// (ij|V|kl) = Y Y^T, a real GEMM on the FP64 tensor cores; likewise for zeta.
// The fit error GEMM theta C fuses the rho recomputation and the two squared
// sums into its epilogue.
#include <cufft.h>

#include <cmath>
#include <mutex>
#include <vector>

#include "arena.h"
#include "check.h"
#include "common.cuh"
#include "dgemm.cuh"
#include "readback.h"
#include "fit.h"
#include "solve.h"

namespace isdf_b200 {

namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kRadius = 5.0;  // checkcode.cpp:168
using CoreC = dmma::Core<128, 128>;

// rho columns [p0, p0 + b): rho[r + i*ng] = psi(r, lo1 + k) psi(r, lo2 + j)
__global__ void k_rho(const double* __restrict__ psi, long long ng, int lo1, int lo2, int n2,
                      int p0, int b, double* __restrict__ rho) {
  const long long total = ng * b;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e % ng;
    const int pair = p0 + (int)(e / ng);
    const int k = pair / n2, j = pair % n2;
    rho[e] = psi[r + (long long)(lo1 + k) * ng] * psi[r + (long long)(lo2 + j) * ng];
  }
}

// sqrt(w V) * vol/Ng on the half spectrum (x fastest, nx/2+1 entries).
__global__ void k_weights(int nx, int ny, int nz, double lx, double ly, double lz, double fac,
                          double* __restrict__ sw) {
  const int hx = nx / 2 + 1;
  const long long nh = (long long)hx * ny * nz;
  for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < nh;
       h += (long long)gridDim.x * blockDim.x) {
    const int ix = (int)(h % hx), iy = (int)((h / hx) % ny), iz = (int)(h / ((long long)hx * ny));
    const double kx = ix * 2.0 * kPi / lx;
    const double ky = (iy <= ny / 2 ? iy : iy - ny) * 2.0 * kPi / ly;
    const double kz = (iz <= nz / 2 ? iz : iz - nz) * 2.0 * kPi / lz;
    const double gkk = (kx * kx + ky * ky + kz * kz) / 2.0;
    const double v = gkk < 1e-8 ? 4.0 * kPi * kRadius * kRadius
                                : 8.0 * kPi / (2.0 * gkk) * (1 - cos(sqrt(2.0 * gkk) * kRadius));
    const double w = (ix == 0 || (nx % 2 == 0 && ix == nx / 2)) ? 1.0 : 2.0;
    sw[h] = sqrt(w * v) * fac;
  }
}

// Y[(col0 + i) + k * ldy] for k < 2 nh from the batch of half spectra.
__global__ void k_spectra_to_rows(const cufftDoubleComplex* __restrict__ f, long long nh, int b,
                                  const double* __restrict__ sw, int col0, long long ldy,
                                  double* __restrict__ Y) {
  const long long total = nh * b;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e % b);
    const long long h = e / b;
    const cufftDoubleComplex z = f[h + (long long)i * nh];
    Y[(col0 + i) + h * ldy] = sw[h] * z.x;
    Y[(col0 + i) + (h + nh) * ldy] = sw[h] * z.y;
  }
}

// C_rm[mu * npair + pair] = psi(piv_mu, lo1 + k) psi(piv_mu, lo2 + j)
__global__ void k_cmat(const double* __restrict__ psi, long long ng, const int* __restrict__ piv,
                       int rk, int lo1, int lo2, int n2, int npair, double* __restrict__ C) {
  const long long total = (long long)rk * npair;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int mu = (int)(e / npair), pair = (int)(e % npair);
    const long long r = piv[mu];
    C[e] = psi[r + (long long)(lo1 + pair / n2) * ng] * psi[r + (long long)(lo2 + pair % n2) * ng];
  }
}

// Sampled pairs: rho columns [p0, p0 + b) of the listed pairs, pair index
// (k - lo1) * n2 + (j - lo2) as checkcode.cpp:62-73 numbers them.
__global__ void k_rho_list(const double* __restrict__ psi, long long ng, int lo1, int lo2, int n2,
                           const int* __restrict__ pairs, int p0, int b,
                           double* __restrict__ rho) {
  const long long total = ng * b;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long r = e % ng;
    const int pair = pairs[p0 + (int)(e / ng)];
    rho[e] = psi[r + (long long)(lo1 + pair / n2) * ng] * psi[r + (long long)(lo2 + pair % n2) * ng];
  }
}

// Depth-major C of the listed pairs: Cb[mu * b + i] = psi(piv_mu, k_i) psi(piv_mu, j_i).
__global__ void k_cmat_list(const double* __restrict__ psi, long long ng,
                            const int* __restrict__ piv, int rk, int lo1, int lo2, int n2,
                            const int* __restrict__ pairs, int p0, int b,
                            double* __restrict__ Cb) {
  const long long total = (long long)rk * b;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int mu = (int)(e / b), i = (int)(e % b);
    const int pair = pairs[p0 + i];
    const long long r = piv[mu];
    Cb[e] = psi[r + (long long)(lo1 + pair / n2) * ng] * psi[r + (long long)(lo2 + pair % n2) * ng];
  }
}

// theta C tile with ||rho - theta C||^2 and ||rho||^2 of the tile in partials.
__global__ void __launch_bounds__(256) k_fit_err(const double* __restrict__ theta, long long ng,
                                                 int rk, const double* __restrict__ C, int npair,
                                                 const double* __restrict__ psi, int lo1, int lo2,
                                                 int n2, double2* __restrict__ partial) {
  extern __shared__ double smem[];
  const int n0 = blockIdx.x * CoreC::BN;
  const long long m0 = (long long)blockIdx.y * CoreC::BM;
  const int m_rem = (int)(ng - m0 < CoreC::BM ? ng - m0 : CoreC::BM);
  CoreC core;
  core.zero();
  core.run<1>(smem, theta + m0, ng, C + n0, npair, m_rem, npair - n0, 0, rk);
  double e2 = 0.0, r2 = 0.0;
  core.for_each([&](int r, int c, double v) {
    if (r < m_rem && n0 + c < npair) {
      const int pair = n0 + c;
      const long long g = m0 + r;
      const double rho = psi[g + (long long)(lo1 + pair / n2) * ng] *
                         psi[g + (long long)(lo2 + pair % n2) * ng];
      e2 += (rho - v) * (rho - v);
      r2 += rho * rho;
    }
  });
  for (int o = 16; o > 0; o >>= 1) {
    e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    r2 += __shfl_xor_sync(0xffffffffu, r2, o);
  }
  __shared__ double2 wsum[8];
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = make_double2(e2, r2);
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < 8; ++w) {
      a += wsum[w].x;
      b += wsum[w].y;
    }
    partial[blockIdx.y * gridDim.x + blockIdx.x] = make_double2(a, b);
  }
}

// ||X - Y||^2 and ||X||^2 over n entries, per-block partials.
__global__ void k_diff_norms(const double* __restrict__ X, const double* __restrict__ Y,
                             long long n, double2* __restrict__ partial) {
  double e2 = 0.0, x2 = 0.0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double d = X[i] - Y[i];
    e2 += d * d;
    x2 += X[i] * X[i];
  }
  for (int o = 16; o > 0; o >>= 1) {
    e2 += __shfl_xor_sync(0xffffffffu, e2, o);
    x2 += __shfl_xor_sync(0xffffffffu, x2, o);
  }
  __shared__ double2 ws[32];
  if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = make_double2(e2, x2);
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
      a += ws[w].x;
      b += ws[w].y;
    }
    partial[blockIdx.x] = make_double2(a, b);
  }
}

struct CheckBuffers {
  double *rho, *sw, *Y, *Yz, *C, *ijkl, *aux, *Tt, *cac;
  cufftDoubleComplex* spec;
  int* piv;
  double2* part;
};

constexpr int kBatch = 128;
constexpr int kDiffBlocks = 296;

CheckBuffers carve(Arena& a, long long ng, long long nh, int npair, int rk, int nfit_tiles) {
  CheckBuffers b;
  b.rho = a.take<double>((size_t)ng * kBatch);
  b.spec = a.take<cufftDoubleComplex>((size_t)nh * kBatch);
  b.sw = a.take<double>((size_t)nh);
  b.Y = a.take<double>((size_t)npair * 2 * nh);
  b.Yz = a.take<double>((size_t)rk * 2 * nh);
  b.C = a.take<double>((size_t)rk * npair);
  b.ijkl = a.take<double>((size_t)npair * npair);
  b.aux = a.take<double>((size_t)rk * rk);
  b.Tt = a.take<double>((size_t)npair * rk);
  b.cac = a.take<double>((size_t)npair * npair);
  b.piv = a.take<int>((size_t)rk);
  b.part = a.take<double2>((size_t)(nfit_tiles > kDiffBlocks ? nfit_tiles : kDiffBlocks));
  return b;
}

int fit_tiles(long long ng, int npair) {
  return (int)(((npair + CoreC::BN - 1) / CoreC::BN) * ((ng + CoreC::BM - 1) / CoreC::BM));
}

struct Plan {
  cufftHandle h = 0;
  bool ok = false;
  ~Plan() {
    if (ok) cufftDestroy(h);
  }
};

}  // namespace

size_t check_workspace_bytes(const int* num_grid, int nstate, int rk, int npair) {
  (void)nstate;
  const long long ng = (long long)num_grid[0] * num_grid[1] * num_grid[2];
  const long long nh = (long long)(num_grid[0] / 2 + 1) * num_grid[1] * num_grid[2];
  Arena a;
  a.counting = true;
  carve(a, ng, nh, npair, rk, fit_tiles(ng, npair));
  return a.off;
}

int check_run(const CheckArgs& args, Arena& arena, cudaStream_t s, double* fit_err,
              double* coul_err) {
  const int nx = args.num_grid[0], ny = args.num_grid[1], nz = args.num_grid[2];
  const long long ng = (long long)nx * ny * nz;
  const long long nh = (long long)(nx / 2 + 1) * ny * nz;
  const int n1 = args.nv1 + args.nc1, n2 = args.nv2 + args.nc2;
  const int npair = n1 * n2, rk = args.rk;
  const int lo1 = args.nocc - args.nv1, lo2 = args.nocc - args.nv2;
  if (2 * nh * (long long)npair > (1LL << 31))
    return record_error(ISDF_ERR_UNSUPPORTED, "check: pair spectra above 2^31 entries");
  const int ftiles = fit_tiles(ng, npair);
  CheckBuffers b = carve(arena, ng, nh, npair, rk, ftiles);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "check: workspace too small");
  ISDF_CUDA(cudaMemcpyAsync(b.piv, args.piv, sizeof(int) * rk, cudaMemcpyHostToDevice, s));
  const double vol = args.length[0] * args.length[1] * args.length[2];
  k_weights<<<grid_for(nh, 256), 256, 0, s>>>(nx, ny, nz, args.length[0], args.length[1],
                                             args.length[2], vol / (double)ng, b.sw);
  k_cmat<<<grid_for((long long)rk * npair, 256), 256, 0, s>>>(args.d_psi, ng, b.piv, rk, lo1, lo2,
                                                             n2, npair, b.C);

  // fit error
  {
    static bool attr_set[64] = {};
    int dev = 0;
    ISDF_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> attr_lock(attr_mutex());
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
      ISDF_CUDA(cudaFuncSetAttribute(k_fit_err, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)CoreC::SMEM_BYTES));
      attr_set[dev] = true;
    }
    dim3 g((unsigned)((npair + CoreC::BN - 1) / CoreC::BN), (unsigned)((ng + CoreC::BM - 1) / CoreC::BM));
    k_fit_err<<<g, 256, CoreC::SMEM_BYTES, s>>>(args.d_theta, ng, rk, b.C, npair, args.d_psi, lo1,
                                                lo2, n2, b.part);
    ISDF_CHECK_LAUNCH();
    std::vector<double2> h(ftiles);
    ISDF_TRY(read_back(h.data(), b.part, sizeof(double2) * ftiles, s));
    double e2 = 0, r2 = 0;
    for (auto& v : h) {
      e2 += v.x;
      r2 += v.y;
    }
    *fit_err = std::sqrt(e2) / std::sqrt(r2);
  }

  // spectra of the pair densities and of theta
  Plan plan;
  int dims[3] = {nz, ny, nx};
  if (cufftPlanMany(&plan.h, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, kBatch) !=
      CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "check: cufftPlanMany failed");
  plan.ok = true;
  if (cufftSetStream(plan.h, s) != CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "check: cufftSetStream failed");
  auto transform = [&](const double* cols, int ncols, bool from_rho, double* Y, long long ldy) {
    for (int c0 = 0; c0 < ncols; c0 += kBatch) {
      const int bcount = std::min(kBatch, ncols - c0);
      const double* in = cols + (long long)c0 * ng;
      if (from_rho) {
        k_rho<<<grid_for(ng * kBatch, 256), 256, 0, s>>>(args.d_psi, ng, lo1, lo2, n2, c0, bcount,
                                                        b.rho);
        if (bcount < kBatch)
          cudaMemsetAsync(b.rho + (long long)bcount * ng, 0,
                          sizeof(double) * (size_t)(kBatch - bcount) * ng, s);
        in = b.rho;
      } else {
        // theta is the caller's output: transform a copy
        cudaMemcpyAsync(b.rho, in, sizeof(double) * (size_t)bcount * ng, cudaMemcpyDeviceToDevice, s);
        if (bcount < kBatch)
          cudaMemsetAsync(b.rho + (long long)bcount * ng, 0,
                          sizeof(double) * (size_t)(kBatch - bcount) * ng, s);
        in = b.rho;
      }
      if (cufftExecD2Z(plan.h, const_cast<double*>(in), b.spec) != CUFFT_SUCCESS) return -1;
      k_spectra_to_rows<<<grid_for(nh * bcount, 256), 256, 0, s>>>(b.spec, nh, bcount, b.sw, c0,
                                                                   ldy, Y);
    }
    return 0;
  };
  if (transform(nullptr, npair, true, b.Y, npair) != 0)
    return record_error(ISDF_ERR_CUDA, "check: cufftExecD2Z failed");
  if (transform(args.d_theta, rk, false, b.Yz, rk) != 0)
    return record_error(ISDF_ERR_CUDA, "check: cufftExecD2Z failed");
  ISDF_CHECK_LAUNCH();

  // (ij|V|kl) = Y Y^T; A = Yz Yz^T; T^T = C^T A; ISDF form = C^T T
  ISDF_TRY(dgemm_store(npair, npair, (int)(2 * nh), b.Y, npair, b.Y, npair, b.ijkl, npair, s));
  ISDF_TRY(dgemm_store(rk, rk, (int)(2 * nh), b.Yz, rk, b.Yz, rk, b.aux, rk, s));
  ISDF_TRY(dgemm_store(npair, rk, rk, b.C, npair, b.aux, rk, b.Tt, npair, s));
  ISDF_TRY(dgemm_store(npair, npair, rk, b.C, npair, b.Tt, npair, b.cac, npair, s));
  k_diff_norms<<<kDiffBlocks, 256, 0, s>>>(b.ijkl, b.cac, (long long)npair * npair, b.part);
  ISDF_CHECK_LAUNCH();
  std::vector<double2> h(kDiffBlocks);
  ISDF_TRY(read_back(h.data(), b.part, sizeof(double2) * kDiffBlocks, s));
  double e2 = 0, x2 = 0;
  for (auto& v : h) {
    e2 += v.x;
    x2 += v.y;
  }
  *coul_err = std::sqrt(e2) / std::sqrt(x2);
  return ISDF_OK;
}

// ---------------------------------------------------------------- sampled check
// The check's two errors restricted to a list of state pairs, for sizes whose
// all-pair spectra do not fit (an extension: the reference checks all pairs,
// checkcode.cpp:54-313, which is O(Ng Npair^2)). For the listed pairs:
//   fit error   = ||rho_s - theta C_s||_F / ||rho_s||_F over all grid points;
//   (ij|V|kl)   = Y Y^T from the spectra of rho_ij, and the ISDF form from the
//                 spectra of the fitted densities theta c_ij: by linearity of
//                 the FFT, Re(FFT(theta c_ij)^H V FFT(theta c_kl)) is the
//                 reference's c_ij^T Re(zeta^H V zeta) c_kl, at 2 npair_s
//                 transforms instead of mu + Npair.
namespace {
struct SampledBuffers {
  double *rho, *fit, *sw, *Y, *Yf, *Cb, *E, *Ef;
  cufftDoubleComplex* spec;
  int *piv, *pairs;
  double2* part;
};

SampledBuffers carve_sampled(Arena& a, long long ng, long long nh, int ns, int rk) {
  SampledBuffers b;
  b.rho = a.take<double>((size_t)ng * kBatch);
  b.fit = a.take<double>((size_t)ng * kBatch);
  b.spec = a.take<cufftDoubleComplex>((size_t)nh * kBatch);
  b.sw = a.take<double>((size_t)nh);
  b.Y = a.take<double>((size_t)ns * 2 * nh);
  b.Yf = a.take<double>((size_t)ns * 2 * nh);
  b.Cb = a.take<double>((size_t)rk * kBatch);
  b.E = a.take<double>((size_t)ns * ns);
  b.Ef = a.take<double>((size_t)ns * ns);
  b.piv = a.take<int>((size_t)rk);
  b.pairs = a.take<int>((size_t)ns);
  b.part = a.take<double2>((size_t)kDiffBlocks);
  return b;
}

int diff_norms(const double* X, const double* Y, long long n, double2* part, cudaStream_t s,
               double* e2, double* x2) {
  k_diff_norms<<<kDiffBlocks, 256, 0, s>>>(X, Y, n, part);
  ISDF_CHECK_LAUNCH();
  std::vector<double2> h(kDiffBlocks);
  ISDF_TRY(read_back(h.data(), part, sizeof(double2) * kDiffBlocks, s));
  for (auto& v : h) {
    *e2 += v.x;
    *x2 += v.y;
  }
  return ISDF_OK;
}
}  // namespace

size_t check_sampled_workspace_bytes(const int* num_grid, int rk, int npair_sample) {
  const long long ng = (long long)num_grid[0] * num_grid[1] * num_grid[2];
  const long long nh = (long long)(num_grid[0] / 2 + 1) * num_grid[1] * num_grid[2];
  Arena a;
  a.counting = true;
  carve_sampled(a, ng, nh, npair_sample, rk);
  return a.off;
}

int check_sampled_run(const CheckArgs& args, const int* pairs, int ns, Arena& arena,
                      cudaStream_t s, double* fit_err, double* coul_err) {
  const int nx = args.num_grid[0], ny = args.num_grid[1], nz = args.num_grid[2];
  const long long ng = (long long)nx * ny * nz;
  const long long nh = (long long)(nx / 2 + 1) * ny * nz;
  const int n2 = args.nv2 + args.nc2, rk = args.rk;
  const int lo1 = args.nocc - args.nv1, lo2 = args.nocc - args.nv2;
  if (2 * nh * (long long)ns > (1LL << 31))
    return record_error(ISDF_ERR_UNSUPPORTED, "sampled check: pair spectra above 2^31 entries");
  SampledBuffers b = carve_sampled(arena, ng, nh, ns, rk);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "sampled check: workspace too small");
  ISDF_CUDA(cudaMemcpyAsync(b.piv, args.piv, sizeof(int) * rk, cudaMemcpyHostToDevice, s));
  ISDF_CUDA(cudaMemcpyAsync(b.pairs, pairs, sizeof(int) * ns, cudaMemcpyHostToDevice, s));
  const double vol = args.length[0] * args.length[1] * args.length[2];
  k_weights<<<grid_for(nh, 256), 256, 0, s>>>(nx, ny, nz, args.length[0], args.length[1],
                                             args.length[2], vol / (double)ng, b.sw);
  Plan plan;
  int dims[3] = {nz, ny, nx};
  if (cufftPlanMany(&plan.h, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, kBatch) !=
      CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "sampled check: cufftPlanMany failed");
  plan.ok = true;
  if (cufftSetStream(plan.h, s) != CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "sampled check: cufftSetStream failed");
  double fe2 = 0, fr2 = 0;
  for (int c0 = 0; c0 < ns; c0 += kBatch) {
    const int bc = std::min(kBatch, ns - c0);
    k_rho_list<<<grid_for(ng * bc, 256), 256, 0, s>>>(args.d_psi, ng, lo1, lo2, n2, b.pairs, c0,
                                                      bc, b.rho);
    k_cmat_list<<<grid_for((long long)rk * bc, 256), 256, 0, s>>>(args.d_psi, ng, b.piv, rk, lo1,
                                                                  lo2, n2, b.pairs, c0, bc, b.Cb);
    ISDF_CHECK_LAUNCH();
    // fitted densities theta C_s of the batch (Ng x bc)
    ISDF_TRY(dgemm_store((int)ng, bc, rk, args.d_theta, ng, b.Cb, bc, b.fit, ng, s));
    ISDF_TRY(diff_norms(b.rho, b.fit, ng * bc, b.part, s, &fe2, &fr2));
    if (bc < kBatch) {
      ISDF_CUDA(cudaMemsetAsync(b.rho + (long long)bc * ng, 0,
                                sizeof(double) * (size_t)(kBatch - bc) * ng, s));
      ISDF_CUDA(cudaMemsetAsync(b.fit + (long long)bc * ng, 0,
                                sizeof(double) * (size_t)(kBatch - bc) * ng, s));
    }
    for (int which = 0; which < 2; ++which) {
      if (cufftExecD2Z(plan.h, which ? b.fit : b.rho, b.spec) != CUFFT_SUCCESS)
        return record_error(ISDF_ERR_CUDA, "sampled check: cufftExecD2Z failed");
      k_spectra_to_rows<<<grid_for(nh * bc, 256), 256, 0, s>>>(b.spec, nh, bc, b.sw, c0, ns,
                                                               which ? b.Yf : b.Y);
    }
    ISDF_CHECK_LAUNCH();
  }
  *fit_err = std::sqrt(fe2) / std::sqrt(fr2);
  ISDF_TRY(dgemm_store(ns, ns, (int)(2 * nh), b.Y, ns, b.Y, ns, b.E, ns, s));
  ISDF_TRY(dgemm_store(ns, ns, (int)(2 * nh), b.Yf, ns, b.Yf, ns, b.Ef, ns, s));
  double ce2 = 0, cx2 = 0;
  ISDF_TRY(diff_norms(b.E, b.Ef, (long long)ns * ns, b.part, s, &ce2, &cx2));
  *coul_err = std::sqrt(ce2) / std::sqrt(cx2);
  return ISDF_OK;
}

// ---------------------------------------------------------------- ISDF Coulomb matrix
// A(mu, nu) = Re sum_G conj(zeta_mu(G)) V(G) zeta_nu(G), zeta = the spectra of
// the theta columns scaled by vol/Ng (checkcode.cpp:249-288, which forms it
// from FFTW full spectra with a complex GEMM): the operator a GW / RPA / TDDFT
// code applies to interpolation-point quantities, the first consumer of theta.
// Here: batched cuFFT D2Z half spectra weighted by sqrt(w V) into one real
// matrix Yz (rk x 2 nh), then A = Yz Yz^T on the FP64 tensor cores.
size_t coulomb_matrix_workspace_bytes(const int* num_grid, int rk) {
  const long long ng = (long long)num_grid[0] * num_grid[1] * num_grid[2];
  const long long nh = (long long)(num_grid[0] / 2 + 1) * num_grid[1] * num_grid[2];
  Arena a;
  a.counting = true;
  a.take<double>((size_t)ng * kBatch);
  a.take<cufftDoubleComplex>((size_t)nh * kBatch);
  a.take<double>((size_t)nh);
  a.take<double>((size_t)rk * 2 * nh);
  return a.off;
}

int coulomb_matrix_run(const int* num_grid, const double* length, const double* d_theta, int rk,
                       double* d_A, Arena& arena, cudaStream_t s) {
  const int nx = num_grid[0], ny = num_grid[1], nz = num_grid[2];
  const long long ng = (long long)nx * ny * nz;
  const long long nh = (long long)(nx / 2 + 1) * ny * nz;
  double* buf = arena.take<double>((size_t)ng * kBatch);
  cufftDoubleComplex* spec = arena.take<cufftDoubleComplex>((size_t)nh * kBatch);
  double* sw = arena.take<double>((size_t)nh);
  double* Yz = arena.take<double>((size_t)rk * 2 * nh);
  if (arena.overflowed()) return record_error(ISDF_ERR_NOMEM, "Coulomb matrix: workspace too small");
  const double vol = length[0] * length[1] * length[2];
  k_weights<<<grid_for(nh, 256), 256, 0, s>>>(nx, ny, nz, length[0], length[1], length[2],
                                             vol / (double)ng, sw);
  Plan plan;
  int dims[3] = {nz, ny, nx};
  if (cufftPlanMany(&plan.h, 3, dims, nullptr, 1, 0, nullptr, 1, 0, CUFFT_D2Z, kBatch) !=
      CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "Coulomb matrix: cufftPlanMany failed");
  plan.ok = true;
  if (cufftSetStream(plan.h, s) != CUFFT_SUCCESS)
    return record_error(ISDF_ERR_CUDA, "Coulomb matrix: cufftSetStream failed");
  for (int c0 = 0; c0 < rk; c0 += kBatch) {
    const int bc = std::min(kBatch, rk - c0);
    // theta is the caller's: transform a copy
    ISDF_CUDA(cudaMemcpyAsync(buf, d_theta + (long long)c0 * ng, sizeof(double) * (size_t)bc * ng,
                              cudaMemcpyDeviceToDevice, s));
    if (bc < kBatch)
      ISDF_CUDA(cudaMemsetAsync(buf + (long long)bc * ng, 0,
                                sizeof(double) * (size_t)(kBatch - bc) * ng, s));
    if (cufftExecD2Z(plan.h, buf, spec) != CUFFT_SUCCESS)
      return record_error(ISDF_ERR_CUDA, "Coulomb matrix: cufftExecD2Z failed");
    k_spectra_to_rows<<<grid_for(nh * bc, 256), 256, 0, s>>>(spec, nh, bc, sw, c0, rk, Yz);
  }
  ISDF_CHECK_LAUNCH();
  const long long K = 2 * nh;  // the GEMM's depth is an int
  if (K > (1LL << 30)) return record_error(ISDF_ERR_UNSUPPORTED, "Coulomb matrix: grid too large");
  return dgemm_store(rk, rk, (int)K, Yz, rk, Yz, rk, d_A, rk, s);
}

}  // namespace isdf_b200
