// A caller of the reference's GPU ISDF() entry point, written the way the
// reference's example driver calls it (examples/si8/readpsi.cpp:219-237:
// cudaMalloc + cudaMemcpy of psi and theta, then
// isdffunc::ISDF(d_psirow, domain_, nocc, nstate, Nv1, Nc1, Nv2, Nc2, Nu,
// d_thetaCol, piv, KmeansMaxIter_ISDF, check)), compiled against
// include/isdf.hpp and linked to libisdf_b200.so instead of the reference.
//
// usage: drop_in psi.bin nx ny nz L nstate nocc nv1 nc1 nv2 nc2 mu iters qrcp_mu out_prefix
// psi.bin: Ng x nstate doubles, column-major. Writes out_prefix.kmeans.piv and
// out_prefix.qrcp.piv (int32[Ng]) and prints one line per call.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <stdexcept>
#include <string>
#include <vector>

#include "isdf.hpp"

using namespace isdf;

static bool write_ints(const std::string& path, const std::vector<int>& v) {
  FILE* f = std::fopen(path.c_str(), "wb");
  if (!f) return false;
  const bool ok = std::fwrite(v.data(), sizeof(int), v.size(), f) == v.size();
  std::fclose(f);
  return ok;
}

int main(int argc, char** argv) {
  if (argc != 16) {
    std::fprintf(stderr,
                 "usage: %s psi.bin nx ny nz L nstate nocc nv1 nc1 nv2 nc2 mu iters qrcp_mu out\n",
                 argv[0]);
    return 2;
  }
  Domain domain_;
  const int nx = std::atoi(argv[2]), ny = std::atoi(argv[3]), nz = std::atoi(argv[4]);
  const double L = std::atof(argv[5]);
  domain_.length = Point3(L, L, L);
  domain_.numGrid = Index3(nx, ny, nz);
  domain_.numGridFine = domain_.numGrid;
  const int nstate = std::atoi(argv[6]), nocc = std::atoi(argv[7]);
  const int Nv1 = std::atoi(argv[8]), Nc1 = std::atoi(argv[9]);
  const int Nv2 = std::atoi(argv[10]), Nc2 = std::atoi(argv[11]);
  const int Nu = std::atoi(argv[12]), KmeansMaxIter_ISDF = std::atoi(argv[13]);
  // the QRCP sketch width IRound(sqrt(1.5 mu)) must not exceed a state window
  const int NuQ = std::atoi(argv[14]);
  const std::string out = argv[15];
  const int Nr = domain_.NumGridTotal();

  std::vector<double> psirow((size_t)Nr * nstate);
  FILE* f = std::fopen(argv[1], "rb");
  if (!f || std::fread(psirow.data(), sizeof(double), psirow.size(), f) != psirow.size()) {
    std::fprintf(stderr, "cannot read %s\n", argv[1]);
    return 2;
  }
  std::fclose(f);

  double *d_psirow = nullptr, *d_theta = nullptr;
  if (cudaMalloc((void**)&d_psirow, psirow.size() * sizeof(double)) != cudaSuccess ||
      cudaMalloc((void**)&d_theta, (size_t)Nu * Nr * sizeof(double)) != cudaSuccess) {
    std::fprintf(stderr, "cudaMalloc failed\n");
    return 3;
  }
  cudaMemcpy(d_psirow, psirow.data(), psirow.size() * sizeof(double), cudaMemcpyHostToDevice);
  std::vector<int> piv(Nr);

  // 1. the reference's 13-argument GPU overload (K-means), with the check
  bool check = true;
  isdffunc::ISDF(d_psirow, domain_, nocc, nstate, Nv1, Nc1, Nv2, Nc2, Nu, d_theta, piv.data(),
                 KmeansMaxIter_ISDF, check);
  std::printf("kmeans ok piv0=%d\n", piv[0]);
  if (!write_ints(out + ".kmeans.piv", piv)) return 4;

  // 2. the overload with the selector of the reference's CPU entry point
  std::string s1 = "QRCP";
  isdffunc::ISDF(d_psirow, domain_, nocc, nstate, Nv1, Nc1, Nv2, Nc2, NuQ, d_theta, piv.data(),
                 KmeansMaxIter_ISDF, s1, false);
  std::printf("qrcp ok piv0=%d\n", piv[0]);
  if (!write_ints(out + ".qrcp.piv", piv)) return 4;

  // 3. failures arrive as std::runtime_error, as the reference's ErrorHandling throws
  try {
    isdffunc::ISDF(d_psirow, domain_, nocc, nstate, Nv1, Nc1, Nv2, Nc2, Nu, d_theta, piv.data(),
                   KmeansMaxIter_ISDF, std::string("Random"), false);
    std::printf("no exception for a bad selector\n");
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
  }
  try {
    isdffunc::ISDF(d_psirow, domain_, nocc, nstate, Nv1, Nc1, Nv2, Nc2, Nr + 1, d_theta,
                   piv.data(), KmeansMaxIter_ISDF, false);
    std::printf("no exception for mu > Ng\n");
  } catch (const std::runtime_error& e) {
    std::printf("caught: %s\n", e.what());
  }
  cudaFree(d_psirow);
  cudaFree(d_theta);
  return 0;
}
