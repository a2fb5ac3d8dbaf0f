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
// Ranks: without MPI (mpi.h not included before this header) the
// communicators in Domain are carried for source compatibility and the solve
// runs on one GPU. With MPI, a communicator of more than one rank selects the
// reference's p-rank layout: d_psirow holds the rank's grid rows
// (isdf_row_block), d_thetaCol receives theta's columns r, r + p, ... over
// all Ng rows, as the reference's GPU_AlltoallBackward leaves them
// (src/common/utility.cpp:444-526), and piv is the same on every rank. The
// ranks then talk over NCCL (one communicator per MPI communicator, made on
// first use: rank 0's NCCL id goes out by MPI_Bcast; each rank's current CUDA
// device is its GPU). The check is not built for more than one rank.
#pragma once

#include <map>
#include <mutex>
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

#if defined(MPI_VERSION)
// The NCCL communicator of an MPI communicator (nullptr at one rank).
inline isdf_comm_t* sharded_comm(MPI_Comm c) {
  int rank = 0, size = 1;
  MPI_Comm_rank(c, &rank);
  MPI_Comm_size(c, &size);
  if (size == 1) return nullptr;
  static std::mutex mu;
  static std::map<MPI_Comm, isdf_comm_t*> made;
  std::lock_guard<std::mutex> lock(mu);
  auto it = made.find(c);
  if (it != made.end()) return it->second;
  unsigned char id[128] = {0};
  int rc = rank == 0 ? isdf_comm_nccl_unique_id(id) : ISDF_OK;
  MPI_Bcast(&rc, 1, MPI_INT, 0, c);
  if (rc != ISDF_OK) throw std::runtime_error("NCCL unique id: " + std::string(isdf_status_string(rc)));
  MPI_Bcast(id, 128, MPI_BYTE, 0, c);
  isdf_comm_t* comm = nullptr;
  throw_on_error(isdf_comm_create_nccl(id, rank, size, &comm));
  made[c] = comm;
  return comm;
}
#endif

// One GPU, or the p-rank layout for an MPI communicator of p > 1 ranks.
inline void solve_dispatch(double* d_psirow, const Domain& domain, int nocc, int nstate, int nv1,
                           int nc1, int nv2, int nc2, int mu_points, double* d_thetaCol, int* piv,
                           int iters, int sel, bool check) {
  isdf_domain_t d = to_c(domain);
#if defined(MPI_VERSION)
  if (isdf_comm_t* comm = sharded_comm(domain.comm)) {
    if (sel != ISDF_SELECT_KMEANS) throw std::runtime_error("QRCP is not built for more than one rank");
    if (check) throw std::runtime_error("the check is not built for more than one rank");
    throw_on_error(isdf_solve_sharded(comm, &d, d_psirow, nocc, nstate, nv1, nc1, nv2, nc2,
                                      mu_points, d_thetaCol, ISDF_THETA_CYCLIC, piv, iters,
                                      nullptr, nullptr));
    return;
  }
#endif
  throw_on_error(isdf_solve(&d, d_psirow, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_thetaCol,
                            piv, iters, sel, check ? 1 : 0, nullptr, nullptr));
}

// The reference's GPU entry point, K-means selection.
inline void ISDF(double* d_psirow, Domain domain, int nocc, int nstate, int nv1, int nc1, int nv2,
                 int nc2, int mu_points, double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF,
                 bool check = false) {
  solve_dispatch(d_psirow, domain, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_thetaCol, piv,
                 KmeansMaxIter_ISDF, ISDF_SELECT_KMEANS, check);
}

// With the selector of the reference's CPU overload: s1 = "Kmeans" | "QRCP".
inline void ISDF(double* d_psirow, Domain domain, int nocc, int nstate, int nv1, int nc1, int nv2,
                 int nc2, int mu_points, double* d_thetaCol, int* piv, int KmeansMaxIter_ISDF,
                 std::string s1, bool check = false) {
  int sel;
  if (s1 == "Kmeans") sel = ISDF_SELECT_KMEANS;
  else if (s1 == "QRCP") sel = ISDF_SELECT_QRCP;
  else throw std::runtime_error("Wrong select points method");  // isdf.cpp:71-74
  solve_dispatch(d_psirow, domain, nocc, nstate, nv1, nc1, nv2, nc2, mu_points, d_thetaCol, piv,
                 KmeansMaxIter_ISDF, sel, check);
}

}  // namespace isdffunc
}  // namespace isdf
