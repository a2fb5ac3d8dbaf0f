// Test infrastructure only (oracle). Runs the reference's own KMEAN
// (src/common/utility.cpp:631-988), compiled unmodified, as p MPI ranks: the
// ranks are forked processes joined by the shared-memory MPI stand-in of
// oracle/shims_mp. This is the p-rank reference that the grid-row sharded
// GPU selection is checked against. Built by oracle/build_ref.sh into
// oracle/_ref/libisdf_ref_mp.so; only tests load it.
#include "isdf.hpp"

#include <signal.h>
#include <sys/mman.h>
#include <sys/wait.h>
#include <time.h>
#include <unistd.h>

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>
#include <string>
#include <vector>

using namespace isdf;

namespace {

struct Result {
  int status;  // 0 = ok
  int rk;
  int iters;
};

// Routes the reference's log stream (isdfOFS) into a string for one call.
struct LogCapture {
  std::stringbuf buf;
  std::streambuf* old;
  LogCapture() {
    std::ostream& os = isdfOFS;
    old = os.rdbuf(&buf);
    os.clear();
  }
  ~LogCapture() {
    std::ostream& os = isdfOFS;
    os.rdbuf(old);
  }
};

double now_s() {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

}  // namespace

extern "C" {

// KMEAN(n, w, mu, 1e-5, iters, 1e-8) as `ranks` MPI ranks (the tolerances of
// src/cuda/isdf-gpu.cpp:31-32), piv zeroed first as src/common/isdf.cpp:174-175
// does unless warm != 0 (then piv holds the previous pivots on entry, as for
// ref_kmeans_warm); each rank seeds std::rand with rand_seed. Every rank
// computes the same piv; rank 0's is returned, and the call fails (-4) if
// another rank's differs. Returns 0, or -1 (setup), -2 (a rank failed or
// exited abnormally), -3 (timeout after timeout_s).
int ref_kmeans_ranks(int ranks, const double* w, const int* ng, const double* len, int mu,
                     int iters, int warm, unsigned rand_seed, int* piv, int* rk_eff, int* n_iter,
                     double timeout_s) {
  if (ranks < 1 || ranks > 64) return -1;
  const long long n = (long long)ng[0] * ng[1] * ng[2];
  // the largest message: 3 mu doubles (centroid sums), mu (double, int) pairs
  const size_t slot = (size_t)mu * 3 * sizeof(double) + 4096;
  const size_t ctl = isdf_shim_mp_region_bytes(ranks, slot);
  const size_t res_off = (ctl + 63) & ~(size_t)63;
  const size_t piv_off = res_off + (((size_t)ranks * sizeof(Result) + 63) & ~(size_t)63);
  const size_t total = piv_off + (size_t)ranks * (size_t)n * sizeof(int);
  void* region = mmap(nullptr, total, PROT_READ | PROT_WRITE, MAP_SHARED | MAP_ANONYMOUS, -1, 0);
  if (region == MAP_FAILED) return -1;
  if (isdf_shim_mp_init(region, ranks, slot) != 0) {
    munmap(region, total);
    return -1;
  }
  Result* res = reinterpret_cast<Result*>((char*)region + res_off);
  int* pivs = reinterpret_cast<int*>((char*)region + piv_off);
  for (int r = 0; r < ranks; ++r) res[r].status = -1;
  std::vector<pid_t> pids;
  fflush(stdout);
  fflush(stderr);
  for (int r = 0; r < ranks; ++r) {
    pid_t pid = fork();
    if (pid < 0) break;
    if (pid == 0) {
      isdf_shim_mp_attach(region, r);
      std::srand(rand_seed);  // only the npt < mu branch draws from it
      int* mine = pivs + (size_t)r * n;
      if (warm) std::memcpy(mine, piv, sizeof(int) * (size_t)n);
      else std::memset(mine, 0, sizeof(int) * (size_t)n);
      LogCapture cap;
      Domain d;
      d.length = Point3(len[0], len[1], len[2]);
      d.posStart = Point3(0.0, 0.0, 0.0);
      d.numGrid = Index3(ng[0], ng[1], ng[2]);
      d.numGridFine = Index3(ng[0], ng[1], ng[2]);
      d.comm = MPI_COMM_WORLD;
      DblNumVec weight((Int)n);
      std::memcpy(weight.Data(), w, sizeof(double) * (size_t)n);
      Int rk = mu;
      KMEAN((Int)n, weight, rk, 1e-5, iters, 1e-8, d, mine);
      std::string log = cap.buf.str();
      size_t p = log.rfind("Converged in ");
      res[r].iters = p == std::string::npos ? -1 : std::atoi(log.c_str() + p + 13);
      res[r].rk = rk;
      res[r].status = 0;
      _exit(0);
    }
    pids.push_back(pid);
  }
  int rc = (int)pids.size() == ranks ? 0 : -1;
  // wait for every rank; on a failed rank or the deadline, end the others
  const double t_end = now_s() + timeout_s;
  std::vector<int> live(pids.size(), 1);
  size_t left = pids.size();
  while (left > 0) {
    bool progressed = false;
    for (size_t i = 0; i < pids.size(); ++i) {
      if (!live[i]) continue;
      int st = 0;
      pid_t got = waitpid(pids[i], &st, WNOHANG);
      if (got == pids[i]) {
        live[i] = 0;
        --left;
        progressed = true;
        if (!WIFEXITED(st) || WEXITSTATUS(st) != 0) rc = rc ? rc : -2;
      }
    }
    if (left == 0) break;
    if (rc != 0 || now_s() > t_end) {
      if (rc == 0) rc = -3;
      for (size_t i = 0; i < pids.size(); ++i)
        if (live[i]) kill(pids[i], SIGKILL);
      for (size_t i = 0; i < pids.size(); ++i)
        if (live[i]) waitpid(pids[i], nullptr, 0);
      break;
    }
    if (!progressed) usleep(2000);
  }
  if (rc == 0) {
    for (int r = 0; r < ranks; ++r)
      if (res[r].status != 0) rc = -2;
  }
  if (rc == 0) {
    for (int r = 1; r < ranks; ++r)
      if (res[r].rk != res[0].rk || res[r].iters != res[0].iters ||
          std::memcmp(pivs, pivs + (size_t)r * n, sizeof(int) * (size_t)n) != 0)
        rc = -4;
    std::memcpy(piv, pivs, sizeof(int) * (size_t)n);
    *rk_eff = res[0].rk;
    *n_iter = res[0].iters;
  }
  isdf_shim_mp_destroy(region);
  munmap(region, total);
  return rc;
}

}  // extern "C"
