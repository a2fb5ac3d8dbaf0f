// Continuous-batching ISDF server (isdf_server_* in include/isdf_c.h).
//
// No counterpart in the reference, which solves one system per call. The
// server keeps a queue of requests and `slots` workers; each worker owns a
// CUDA stream and takes its workspace from a private stream-ordered memory
// pool, so solves on different slots run concurrently and their kernels
// overlap on the GPU. psi and theta stay in the caller's device buffers.
//
// Admission is by device footprint: a request starts only when its
// workspace fits in what the budget has left. A free slot takes the oldest
// queued request that fits; smaller requests may start ahead of a large head
// that does not fit yet, but only until the head has been passed over
// `max_skips` times, after which nothing new starts until it fits. Latency
// is measured from submit to completion; p50 / p99 and solves/s are
// reported by isdf_server_stats(). The fits of large systems (Ng rk^2 >=
// 1e13) run one at a time: two of them on the tensor cores at once only
// share the units and the power cap, while another request's K-means
// selection (FP64 CUDA cores) overlaps a running fit.
//
// Small K-means requests (Ng <= 2^20, mu <= 512, cold start) queue apart: a
// batcher thread takes up to batch_small of them at once, computes their
// weights and runs all their selections in one cooperative launch
// (kmeans_select_batch), then puts them back at the head of the main queue,
// where the slots run their fits. A small solve is latency bound (about a
// hundred Lloyd iterations of ten small kernels each), so one launch for many
// of them raises the rate at which they are served.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/isdf_c.h"
#include "arena.h"
#include "kmeans.h"
#include "solve.h"

namespace isdf_b200 {
namespace {

using Clock = std::chrono::steady_clock;

struct Job {
  long long ticket;
  isdf_request_t req;
  size_t footprint;
  int state = 0;  // 0 queued, 1 running, 2 done
  int status = ISDF_OK;
  int skips = 0;
  isdf_report_t rep;
  Clock::time_point submit, start, finish;
  bool small = false;     // selection by the batcher
  bool selected = false;  // the batcher has run its selection
  size_t batch_bytes = 0;
  KmeansResult sel;
  double select_ms = 0;
};

struct Server {
  isdf_server_config_t cfg;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<long long> queue;
  std::deque<long long> small_queue;  // small K-means requests waiting for the batcher
  std::map<long long, Job> jobs;
  long long next_ticket = 1;
  size_t in_use = 0, peak_bytes = 0;
  int running = 0, peak_running = 0;
  bool stopping = false;
  std::vector<std::thread> workers;
  std::thread batcher;
  bool batcher_active = false;  // the batcher may still hand requests to the slots
  cudaMemPool_t pool = nullptr;
  std::vector<double> latencies_ms;
  Clock::time_point first_submit, last_finish;
  bool any_submit = false;
  long long completed = 0, failed = 0, cancelled = 0;
  std::mutex fit_mutex;  // large fits one at a time (SolveResources::fit_lock)
};

int set_err(int code, const char* msg);

// Next job a free slot may start (under the lock), or -1.
long long pick(Server* s) {
  const size_t left = s->cfg.hbm_budget_bytes > s->in_use ? s->cfg.hbm_budget_bytes - s->in_use : 0;
  for (size_t i = 0; i < s->queue.size(); ++i) {
    Job& j = s->jobs[s->queue[i]];
    if (j.footprint <= left) {
      if (i > 0) {
        Job& head = s->jobs[s->queue[0]];
        if (head.skips >= s->cfg.max_skips) return -1;  // the head waits for room; nothing passes it
        head.skips++;
      }
      long long t = s->queue[i];
      s->queue.erase(s->queue.begin() + (long)i);
      return t;
    }
  }
  return -1;
}

void worker(Server* s, int slot) {
  cudaSetDevice(s->cfg.device);
  cudaStream_t stream = nullptr;
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  (void)slot;
  for (;;) {
    long long t = -1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      // on stop, the slots still finish the requests whose selection the
      // batcher has done (and may still hand over) before they exit
      s->cv_work.wait(lk, [&] {
        if ((t = pick(s)) >= 0) return true;
        return s->stopping && !s->batcher_active;
      });
      if (t < 0) break;  // stopping and nothing startable
      Job& j = s->jobs[t];
      if (!j.selected) j.start = Clock::now();
      j.state = 1;
      s->in_use += j.footprint;
      s->peak_bytes = std::max(s->peak_bytes, s->in_use);
      s->running++;
      s->peak_running = std::max(s->peak_running, s->running);
    }
    Job* jp;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      jp = &s->jobs[t];
    }
    isdf_request_t req = jp->req;
    const bool pre = jp->selected;
    const KmeansResult sel = jp->sel;
    isdf_report_t rep;
    std::memset(&rep, 0, sizeof(rep));
    int rc = ISDF_OK;
    void* ws = nullptr;
    if (cudaMallocFromPoolAsync(&ws, jp->footprint, s->pool, stream) != cudaSuccess) {
      (void)cudaGetLastError();
      rc = set_err(ISDF_ERR_NOMEM, "server: workspace allocation failed");
    } else {
      SolveResources res{static_cast<char*>(ws), jp->footprint, stream, &s->fit_mutex,
                         pre ? &sel : nullptr};
      rc = solve(&req.dom, req.d_psi, req.nocc, req.nstate, req.nv1, req.nc1, req.nv2, req.nc2,
                 req.mu_points, req.d_theta, req.piv, req.kmeans_max_iter, req.selector, req.check,
                 &req.opt, &rep, &res);
      cudaFreeAsync(ws, stream);
      cudaStreamSynchronize(stream);
    }
    {
      std::lock_guard<std::mutex> lk(s->mu);
      Job& j = s->jobs[t];
      j.state = 2;
      j.status = rc;
      j.rep = rep;
      if (j.selected) j.rep.t_select_ms = j.select_ms;
      j.finish = Clock::now();
      s->in_use -= j.footprint;
      s->running--;
      s->last_finish = j.finish;
      if (rc == ISDF_OK) {
        s->completed++;
        s->latencies_ms.push_back(
            std::chrono::duration<double, std::milli>(j.finish - j.submit).count());
      } else {
        s->failed++;
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  cudaStreamDestroy(stream);
}

// The batcher: small K-means requests' weights and selections, many per launch.
void batcher(Server* s) {
  cudaSetDevice(s->cfg.device);
  cudaStream_t stream = nullptr;
  cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking);
  for (;;) {
    std::vector<long long> batch;
    size_t bytes = 0;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      s->cv_work.wait(lk, [&] {
        if (s->stopping) return true;
        if (s->small_queue.empty()) return false;
        const Job& h = s->jobs[s->small_queue.front()];
        return s->in_use + h.batch_bytes <= s->cfg.hbm_budget_bytes;
      });
      if (s->stopping && s->small_queue.empty()) {
        s->batcher_active = false;
        break;
      }
      while (!s->small_queue.empty() && (int)batch.size() < s->cfg.batch_small) {
        Job& j = s->jobs[s->small_queue.front()];
        if (s->in_use + bytes + j.batch_bytes > s->cfg.hbm_budget_bytes) break;
        bytes += j.batch_bytes;
        batch.push_back(j.ticket);
        s->small_queue.pop_front();
        j.state = 1;
        j.start = Clock::now();
      }
      if (batch.empty()) continue;
      s->in_use += bytes;
      s->peak_bytes = std::max(s->peak_bytes, s->in_use);
      s->running += (int)batch.size();
      s->peak_running = std::max(s->peak_running, s->running);
    }
    const auto t0 = Clock::now();
    std::vector<KmeansArgs> args(batch.size());
    std::vector<KmeansResult> res(batch.size());
    int rc = ISDF_OK;
    void* ws = nullptr;
    if (cudaMallocFromPoolAsync(&ws, bytes + 4096, s->pool, stream) != cudaSuccess) {
      (void)cudaGetLastError();
      rc = set_err(ISDF_ERR_NOMEM, "server: batch workspace allocation failed");
    } else {
      Arena arena;
      arena.base = static_cast<char*>(ws);
      arena.cap = bytes + 4096;
      arena.off = 0;
      for (size_t i = 0; i < batch.size() && rc == ISDF_OK; ++i) {
        isdf_request_t r;
        {
          std::lock_guard<std::mutex> lk(s->mu);
          r = s->jobs[batch[i]].req;
        }
        const long long ng = (long long)r.dom.num_grid[0] * r.dom.num_grid[1] * r.dom.num_grid[2];
        double* d_w = arena.take<double>((size_t)ng);
        rc = kmeans_weight(r.d_psi, ng, r.nocc, r.nv1, r.nc1, r.nv2, r.nc2, d_w, stream);
        KmeansArgs& a = args[i];
        a.d_w = d_w;
        a.ng = ng;
        for (int k = 0; k < 3; ++k) {
          a.num_grid[k] = r.dom.num_grid[k];
          a.length[k] = r.dom.length[k];
        }
        a.mu = r.mu_points == 0 ? default_mu(r.nv1, r.nc1, r.nv2, r.nc2) : r.mu_points;
        a.max_iter = r.kmeans_max_iter;
        a.rand_seed = r.opt.rand_seed;
        a.piv = r.piv;
      }
      if (rc == ISDF_OK) rc = kmeans_select_batch(args.data(), (int)args.size(), arena, stream, res.data());
      cudaFreeAsync(ws, stream);
      cudaStreamSynchronize(stream);
    }
    const double ms = std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->in_use -= bytes;
      s->running -= (int)batch.size();
      // back to the head of the main queue, in arrival order, for their fits
      for (size_t k = batch.size(); k-- > 0;) {
        Job& j = s->jobs[batch[k]];
        if (rc == ISDF_OK) {
          j.selected = true;
          j.sel = res[k];
          j.select_ms = ms;
          s->queue.push_front(j.ticket);
        } else {
          j.state = 2;
          j.status = rc;
          j.finish = Clock::now();
          s->last_finish = j.finish;
          s->failed++;
        }
      }
    }
    s->cv_done.notify_all();
    s->cv_work.notify_all();
  }
  s->cv_work.notify_all();
  cudaStreamDestroy(stream);
}

double percentile(std::vector<double> v, double q) {
  if (v.empty()) return 0.0;
  std::sort(v.begin(), v.end());
  const double pos = q * (double)(v.size() - 1);
  const size_t lo = (size_t)pos;
  const size_t hi = std::min(lo + 1, v.size() - 1);
  return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
}

}  // namespace
}  // namespace isdf_b200

using namespace isdf_b200;

namespace isdf_b200 {
namespace {
int set_err(int code, const char* msg) { return record_error(code, msg); }

// Runs a C entry point's body and turns what the standard library may throw
// (host allocation, thread or mutex errors) into a status, so that no
// exception crosses the C ABI.
template <class F>
int guarded(F&& body) {
  try {
    return body();
  } catch (const std::exception& e) {
    return record_error(ISDF_ERR_NOMEM, e.what());
  } catch (...) {
    return record_error(ISDF_ERR_CUDA, "server: unknown exception");
  }
}
}  // namespace
}  // namespace isdf_b200

extern "C" {

void isdf_server_default_config(isdf_server_config_t* cfg) {
  if (!cfg) return;
  std::memset(cfg, 0, sizeof(*cfg));
  cfg->device = 0;
  cfg->slots = 4;
  cfg->hbm_budget_bytes = 0;
  cfg->max_queue = 4096;
  cfg->max_skips = 64;
  cfg->batch_small = 32;
}

int isdf_server_create(const isdf_server_config_t* cfg_in, void** out) {
  return guarded([&]() -> int {
    if (!out) return record_error(ISDF_ERR_ARG, "server: null output");
    isdf_server_config_t cfg;
    isdf_server_default_config(&cfg);
    if (cfg_in) cfg = *cfg_in;
    if (cfg.slots < 1 || cfg.slots > 64)
      return record_error(ISDF_ERR_ARG, "server: slots in [1, 64]");
    if (cfg.batch_small < 0 || cfg.batch_small > 1024)
      return record_error(ISDF_ERR_ARG, "server: batch_small in [0, 1024]");
    if (cudaSetDevice(cfg.device) != cudaSuccess)
      return record_error(ISDF_ERR_ARG, "server: device");
    if (cfg.hbm_budget_bytes == 0) {
      size_t free_b = 0, total_b = 0;
      if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess)
        return record_error(ISDF_ERR_CUDA, "server: cudaMemGetInfo failed");
      cfg.hbm_budget_bytes = free_b / 2;
    }
    Server* s = new Server();
    s->cfg = cfg;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg.device;
    if (cudaMemPoolCreate(&s->pool, &props) != cudaSuccess) {
      delete s;
      return record_error(ISDF_ERR_CUDA, "server: cudaMemPoolCreate failed");
    }
    unsigned long long keep = cfg.hbm_budget_bytes;
    cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    try {
      for (int i = 0; i < cfg.slots; ++i) s->workers.emplace_back(worker, s, i);
      if (cfg.batch_small > 0) {
        s->batcher_active = true;
        s->batcher = std::thread(batcher, s);
      }
    } catch (...) {  // a thread did not start: stop the ones that did
      {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stopping = true;
        s->batcher_active = false;
      }
      s->cv_work.notify_all();
      for (auto& w : s->workers) w.join();
      cudaMemPoolDestroy(s->pool);
      delete s;
      return record_error(ISDF_ERR_NOMEM, "server: a worker thread could not be started");
    }
    *out = s;
    return ISDF_OK;
  });
}

int isdf_server_submit(void* server, const isdf_request_t* req, long long* ticket) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s || !req || !ticket) return record_error(ISDF_ERR_ARG, "server: null argument");
    if (!req->d_psi || !req->d_theta || !req->piv)
      return record_error(ISDF_ERR_ARG, "server: request buffers");
    const size_t fp = request_footprint(&req->dom, req->nstate, req->nv1, req->nc1, req->nv2,
                                        req->nc2, req->mu_points, req->selector, req->check,
                                        &req->opt);
    if (fp > s->cfg.hbm_budget_bytes)
      return record_error(ISDF_ERR_UNSUPPORTED, "server: request larger than the whole budget");
    {
      std::lock_guard<std::mutex> lk(s->mu);
      if (s->stopping) return record_error(ISDF_ERR_CANCELLED, "server: stopping");
      if ((int)s->queue.size() >= s->cfg.max_queue)
        return record_error(ISDF_ERR_BUSY, "server: queue full");
      Job j;
      j.ticket = s->next_ticket++;
      j.req = *req;
      j.req.opt.stream = nullptr;
      j.footprint = fp;
      j.submit = Clock::now();
      {
        const isdf_domain_t& d = req->dom;
        const long long ng = (long long)d.num_grid[0] * d.num_grid[1] * d.num_grid[2];
        const int rk = req->mu_points == 0 ? default_mu(req->nv1, req->nc1, req->nv2, req->nc2)
                                           : req->mu_points;
        j.small = s->cfg.batch_small > 0 && req->selector == ISDF_SELECT_KMEANS &&
                  !req->opt.kmeans_warm_start && ng > 1 && ng <= kKmeansBatchMaxNg && rk > 0 &&
                  rk <= kKmeansBatchMaxMu && rk <= ng && req->kmeans_max_iter >= 0 &&
                  d.num_grid[0] > 0 && d.num_grid[1] > 0 && d.num_grid[2] > 0 &&
                  req->opt.refine_steps == 0 && req->nv1 >= 0 && req->nc1 >= 0 && req->nv2 >= 0 &&
                  req->nc2 >= 0 && req->nv1 + req->nc1 > 0 && req->nv2 + req->nc2 > 0 &&
                  req->nocc - req->nv1 >= 0 && req->nocc + req->nc1 <= req->nstate &&
                  req->nocc - req->nv2 >= 0 && req->nocc + req->nc2 <= req->nstate;
        if (j.small)
          j.batch_bytes = kmeans_batch_workspace_bytes(ng, rk) + sizeof(double) * ng + 512;
      }
      std::memset(&j.rep, 0, sizeof(j.rep));
      if (!s->any_submit) {
        s->first_submit = j.submit;
        s->any_submit = true;
      }
      *ticket = j.ticket;
      s->jobs[j.ticket] = j;
      if (j.small) s->small_queue.push_back(j.ticket);
      else s->queue.push_back(j.ticket);
    }
    s->cv_work.notify_all();
    return ISDF_OK;
  });
}

int isdf_server_poll(void* server, long long ticket, int* state, int* status, isdf_report_t* rep) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s) return record_error(ISDF_ERR_ARG, "server: null");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return record_error(ISDF_ERR_ARG, "server: unknown ticket");
    if (state) *state = it->second.state;
    if (status) *status = it->second.status;
    if (rep && it->second.state == 2) *rep = it->second.rep;
    return ISDF_OK;
  });
}

int isdf_server_wait(void* server, long long ticket, double timeout_ms, int* status,
                     isdf_report_t* rep) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s) return record_error(ISDF_ERR_ARG, "server: null");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(ticket);
    if (it == s->jobs.end()) return record_error(ISDF_ERR_ARG, "server: unknown ticket");
    auto done = [&] { return s->jobs[ticket].state == 2; };
    if (timeout_ms < 0) s->cv_done.wait(lk, done);
    else if (!s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms), done))
      return record_error(ISDF_ERR_TIMEOUT, "server: wait timed out");
    Job& j = s->jobs[ticket];
    if (status) *status = j.status;
    if (rep) *rep = j.rep;
    return ISDF_OK;
  });
}

int isdf_server_cancel(void* server, long long ticket) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s) return record_error(ISDF_ERR_ARG, "server: null");
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = std::find(s->small_queue.begin(), s->small_queue.end(), ticket);
    if (it != s->small_queue.end()) {
      s->small_queue.erase(it);
    } else {
      auto qt = std::find(s->queue.begin(), s->queue.end(), ticket);
      if (qt == s->queue.end() || s->jobs[ticket].selected)
        return record_error(ISDF_ERR_ARG, "server: not queued (running or done)");
      s->queue.erase(qt);
    }
    Job& j = s->jobs[ticket];
    j.state = 2;
    j.status = ISDF_ERR_CANCELLED;
    j.finish = Clock::now();
    s->cancelled++;
    s->cv_done.notify_all();
    return ISDF_OK;
  });
}

int isdf_server_stats(void* server, isdf_server_stats_t* st) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s || !st) return record_error(ISDF_ERR_ARG, "server: null");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(st, 0, sizeof(*st));
    st->submitted = s->next_ticket - 1;
    st->completed = s->completed;
    st->failed = s->failed;
    st->cancelled = s->cancelled;
    st->p50_ms = percentile(s->latencies_ms, 0.50);
    st->p99_ms = percentile(s->latencies_ms, 0.99);
    double sum = 0;
    for (double v : s->latencies_ms) sum += v;
    st->mean_ms = s->latencies_ms.empty() ? 0.0 : sum / (double)s->latencies_ms.size();
    const auto busy = s->last_finish - s->first_submit;
    const double span =
        s->any_submit && s->completed ? std::chrono::duration<double>(busy).count() : 0.0;
    st->solves_per_s = span > 0 ? (double)s->completed / span : 0.0;
    st->peak_concurrency = s->peak_running;
    st->peak_bytes = s->peak_bytes;
    st->queued = (int)(s->queue.size() + s->small_queue.size());
    st->running = s->running;
    return ISDF_OK;
  });
}

int isdf_server_destroy(void* server) {
  return guarded([&]() -> int {
    Server* s = static_cast<Server*>(server);
    if (!s) return ISDF_OK;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      std::deque<long long> keep;  // selected small requests finish their fits
      for (long long t : s->queue) {
        Job& j = s->jobs[t];
        if (j.selected) {
          keep.push_back(t);
          continue;
        }
        j.state = 2;
        j.status = ISDF_ERR_CANCELLED;
        s->cancelled++;
      }
      for (long long t : s->small_queue) {
        Job& j = s->jobs[t];
        j.state = 2;
        j.status = ISDF_ERR_CANCELLED;
        s->cancelled++;
      }
      s->small_queue.clear();
      s->queue = keep;
      s->stopping = true;
    }
    s->cv_work.notify_all();
    s->cv_done.notify_all();
    if (s->batcher.joinable()) s->batcher.join();
    for (auto& w : s->workers) w.join();
    if (s->pool) cudaMemPoolDestroy(s->pool);
    delete s;
    return ISDF_OK;
  });
}

}  // extern "C"
