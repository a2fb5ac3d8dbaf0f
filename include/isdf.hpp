// isdf.hpp - drop-in C++ entry point of the B200 ISDF engine.
//
// Replaces the GPU overload of the reference's public API,
//   void isdf::isdffunc::ISDF(double* d_psirow, Domain domain, int nocc,
//        int nstate, int nv1, int nc1, int nv2, int nc2, int mu_points,
//        double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF, bool check=false)
// (reference include/isdf.hpp:37, src/common/isdf.cpp:132-209), with the same
// argument meaning, the same Domain fields and the same failure behaviour
// (std::runtime_error, as the reference's ErrorHandling throws,
// src/common/global.cpp:7-11). A second overload takes the point selector
// ("Kmeans" | "QRCP") before `check`, as the reference's CPU overload does
// (include/isdf.hpp:39). Both are header-only wrappers over the C ABI in
// isdf_c.h; link with -lisdf_b200.
//
// One rank, one GPU: the communicators in Domain are carried for source
// compatibility and ignored.
#pragma once

#include <stdexcept>
#include <string>

#include "isdf_c.h"

namespace isdf {

typedef int Int;
typedef double Real;

// Same layout as the reference's Vec3T<F> (include/common/tinyvec_decl.hpp).
template <class F>
struct Vec3T {
  F v_[3];
  Vec3T() : v_{F(0), F(0), F(0)} {}
  Vec3T(F x, F y, F z) : v_{x, y, z} {}
  F& operator[](int i) { return v_[i]; }
  const F& operator[](int i) const { return v_[i]; }
};
typedef Vec3T<Real> Point3;
typedef Vec3T<Int> Index3;

#if defined(MPI_VERSION)
typedef MPI_Comm CommHandle;
#else
typedef void* CommHandle;  // MPI is not needed at world size 1
#endif

// Field order and types of the reference's Domain (include/common/domain.hpp:8-36).
struct Domain {
  Point3 length;
  Point3 posStart;
  Index3 numGrid;
  Index3 numGridFine;
  CommHandle comm;
  CommHandle rowComm;
  CommHandle colComm;

  Domain() : comm(), rowComm(), colComm() {}
  Real Volume() const { return length[0] * length[1] * length[2]; }
  Int NumGridTotal() const { return numGrid[0] * numGrid[1] * numGrid[2]; }
  Int NumGridTotalFine() const { return numGridFine[0] * numGridFine[1] * numGridFine[2]; }
};

namespace isdffunc {

inline isdf_domain_t to_c(const Domain& d) {
  isdf_domain_t c;
  for (int i = 0; i < 3; ++i) {
    c.length[i] = d.length[i];
    c.pos_start[i] = d.posStart[i];
    c.num_grid[i] = d.numGrid[i];
    c.num_grid_fine[i] = d.numGridFine[i];
  }
  return c;
}

inline void throw_on_error(int rc) {
  if (rc != ISDF_OK) {
    std::string msg = isdf_last_error();
    if (msg.empty()) msg = isdf_status_string(rc);
    throw std::runtime_error(msg);
  }
}

// The reference's GPU entry point, K-means selection.
inline void ISDF(double* d_psirow, Domain domain, int nocc, int nstate, int nv1, int nc1, int nv2,
                 int nc2, int mu_points, double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF,
                 bool check = false) {
  isdf_domain_t d = to_c(domain);
  throw_on_error(isdf_solve(&d, d_psirow, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_thetaCol,
                            piv, KmeansMaxIter_ISDF, ISDF_SELECT_KMEANS, check ? 1 : 0, nullptr,
                            nullptr));
}

// With the selector of the reference's CPU overload: s1 = "Kmeans" | "QRCP".
inline void ISDF(double* d_psirow, Domain domain, int nocc, int nstate, int nv1, int nc1, int nv2,
                 int nc2, int mu_points, double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF,
                 std::string s1, bool check = false) {
  int sel;
  if (s1 == "Kmeans") sel = ISDF_SELECT_KMEANS;
  else if (s1 == "QRCP") sel = ISDF_SELECT_QRCP;
  else throw std::runtime_error("Wrong select points method");  // isdf.cpp:71-74
  isdf_domain_t d = to_c(domain);
  throw_on_error(isdf_solve(&d, d_psirow, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_thetaCol,
                            piv, KmeansMaxIter_ISDF, sel, check ? 1 : 0, nullptr, nullptr));
}

}  // namespace isdffunc
}  // namespace isdf
