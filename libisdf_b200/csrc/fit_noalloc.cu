// isdf_fit_noalloc: the FP64 fit with its scratch in a fixed device array.
//
// Some callers cannot let the library allocate device memory while they run:
// a host code that reserves (nearly) all of HBM for its own memory pool at
// start-up (plane-wave DFT codes commonly do, for wavefunctions and FFT
// buffers), where a cudaMalloc mid-run fails or fragments that pool; and
// callers that must not pay the device-wide synchronisation that cudaFree
// brings. For them this entry point runs the same fit kernels as isdf_fit()
// but takes every scratch array from one file-scope __device__ array of
// ISDF_NOALLOC_SCRATCH_BYTES (8 MiB), so it calls no cudaMalloc / cudaFree and no allocating
// library routine. The caller still passes psi, the pivots and theta.
//
// Costs and rules:
//  * every process that loads libisdf_b200.so holds this array on every GPU
//    it uses, until the process exits;
//  * all calls on a device share the array: calls that overlap on the GPU
//    (other host threads, or streams that are not ordered) race on it;
//  * the array keeps the previous call's contents; the one scratch word that
//    must start at zero (the Cholesky failure index) is cleared by every call;
//  * every call looks up the array's device address on the current device
//    (cudaGetSymbolAddress: a cheap runtime query, so a cudaDeviceReset
//    between calls leaves no stale address behind); the first call on a
//    device also loads the module that holds the array, so make that first
//    call before any stream capture begins.
#include <cstdio>
#include <exception>

#include "arena.h"
#include "common.cuh"
#include "fit.h"
#include "readback.h"

namespace isdf_b200 {

namespace {

static __device__ __align__(256) char g_fit_scratch[ISDF_NOALLOC_SCRATCH_BYTES];

// Device address of g_fit_scratch on the current device, looked up with that
// device current. In host code the name g_fit_scratch is only a host-side
// stand-in: it must never be passed to a kernel, the address below must.
int scratch_address(void** out) {
  void* p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_fit_scratch);
  if (e != cudaSuccess)
    return record_cuda_error(e, "cudaGetSymbolAddress(g_fit_scratch)", __FILE__, __LINE__);
  *out = p;
  return ISDF_OK;
}

int fit_noalloc(const double* d_psi, long long ng, int nstate, int nocc, int nv1, int nc1,
                int nv2, int nc2, int rk, const int* piv, double* d_theta, int* chol_info,
                void* stream) {
  if (!d_psi || !d_theta || !piv || ng <= 0 || rk <= 0 || rk > ng || nstate <= 0)
    return record_error(ISDF_ERR_ARG, "isdf_fit_noalloc: bad arguments");
  if (nv1 < 0 || nc1 < 0 || nv2 < 0 || nc2 < 0 || nv1 + nc1 <= 0 || nv2 + nc2 <= 0 ||
      nocc - nv1 < 0 || nocc + nc1 > nstate || nocc - nv2 < 0 || nocc + nc2 > nstate)
    return record_error(ISDF_ERR_ARG, "isdf_fit_noalloc: state window outside [0, nstate)");
  for (int j = 0; j < rk; ++j)
    if (piv[j] < 0 || piv[j] >= ng)
      return record_error(ISDF_ERR_ARG, "isdf_fit_noalloc: pivot outside the grid");
  const size_t need = fit_workspace_bytes(ng, nstate, rk);
  if (need > (size_t)ISDF_NOALLOC_SCRATCH_BYTES) {
    static thread_local char msg[200];
    snprintf(msg, sizeof(msg),
             "isdf_fit_noalloc: rk=%d, nstate=%d needs %zu bytes of scratch; the fixed array "
             "holds %zu (use isdf_fit)",
             rk, nstate, need, (size_t)ISDF_NOALLOC_SCRATCH_BYTES);
    return record_error(ISDF_ERR_UNSUPPORTED, msg);
  }
  void* base = nullptr;
  ISDF_TRY(scratch_address(&base));
  Arena arena;
  arena.base = static_cast<char*>(base);
  arena.cap = ISDF_NOALLOC_SCRATCH_BYTES;
  arena.off = 0;
  FitArgs fa;
  fa.d_psi = d_psi;
  fa.ng = ng;
  fa.nstate = nstate;
  fa.nocc = nocc;
  fa.nv1 = nv1;
  fa.nc1 = nc1;
  fa.nv2 = nv2;
  fa.nc2 = nc2;
  fa.rk = rk;
  fa.piv = piv;
  fa.d_theta = d_theta;
  FitResult fr;
  cudaStream_t s = (cudaStream_t)stream;  // NULL: the legacy default stream
  // no pinned mailbox either: the small status reads go by cudaMemcpyAsync
  const bool mailbox = readback_mailbox();
  set_readback_mailbox(false);
  struct MailboxRestore {
    bool on;
    ~MailboxRestore() { set_readback_mailbox(on); }
  } restore{mailbox};
  int rc = fit_fp64(fa, arena, s, &fr, /*timed=*/false);
  if (chol_info) *chol_info = fr.chol_info;
  if (rc == ISDF_OK) ISDF_CUDA(cudaStreamSynchronize(s));
  return rc;
}

}  // namespace

}  // namespace isdf_b200

using namespace isdf_b200;

extern "C" int isdf_fit_noalloc(const double* d_psi, long long ng, int nstate, int nocc, int nv1,
                                int nc1, int nv2, int nc2, int rk, const int* piv,
                                double* d_theta, int* chol_info, void* stream) {
  try {
    return fit_noalloc(d_psi, ng, nstate, nocc, nv1, nc1, nv2, nc2, rk, piv, d_theta, chol_info,
                       stream);
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_CUDA, e.what());
  } catch (...) {
    return record_error(ISDF_ERR_CUDA, "isdf_fit_noalloc: unknown exception");
  }
}
