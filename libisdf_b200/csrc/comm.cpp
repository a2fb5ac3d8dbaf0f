// Collective transports of the sharded solve and their C ABI (isdf_comm_*).
//
// NCCL: one process (or thread) per GPU; NCCL is opened at run time
// (dlopen of libnccl.so.2, the copy torch loads when it is already in the
// process), so the library itself has no link-time dependency on it and a
// process that never shards never loads it. The all-gather of equal blocks is
// ncclAllGather; of unequal blocks, one ncclBroadcast per rank inside a group;
// the all-to-all is grouped ncclSend / ncclRecv, the rank's own block a device
// copy.
//
// Local group: several ranks in one process, one host thread per rank, on one
// or several devices. A collective records an event on every rank's stream,
// meets the other ranks at a host barrier (bounded: a rank that does not
// arrive within the group's timeout fails the collective and the group), and
// each rank's stream then waits for the others' events and copies what it
// needs from their buffers (cudaMemcpyAsync with cudaMemcpyDefault, direct or
// through the host between devices without peer access). A second barrier and
// event round keeps a rank from reusing its send buffer before the others have
// read it. No kernel ever waits on another rank: the ordering is carried by
// stream events.
//
// Callbacks: the caller's own collectives (an MPI code's CUDA-aware
// MPI_Allgatherv / MPI_Alltoallv, for instance), called with device pointers
// and the stream.
#include "comm.h"

#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "errors.h"

namespace isdf_b200 {

Transport::~Transport() {
  if (!ws && !stream && !status) return;
  int cur = -1;
  cudaGetDevice(&cur);
  cudaSetDevice(device);
  if (ws) cudaFree(ws);
  if (status) cudaFree(status);
  if (stream) cudaStreamDestroy(stream);
  if (cur >= 0) cudaSetDevice(cur);
}

int Transport::ensure_stream() {
  ISDF_CUDA(cudaSetDevice(device));
  if (!stream) ISDF_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
  return ISDF_OK;
}

int Transport::ensure_status() {
  if (status) return ISDF_OK;
  int cur = -1;
  ISDF_CUDA(cudaGetDevice(&cur));
  ISDF_CUDA(cudaSetDevice(device));
  const cudaError_t e = cudaMalloc((void**)&status, kStatusBytes * (size_t)(size + 1));
  cudaSetDevice(cur);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();
    status = nullptr;
    return record_error(ISDF_ERR_NOMEM, "communicator: status buffer allocation failed");
  }
  return ISDF_OK;
}

int Transport::acquire(size_t bytes, Arena* arena) {
  ISDF_TRY(ensure_stream());
  if (ws_cap < bytes) {
    if (ws) {
      ISDF_CUDA(cudaStreamSynchronize(stream));
      ISDF_CUDA(cudaFree(ws));
      ws = nullptr;
      ws_cap = 0;
    }
    if (cudaMalloc((void**)&ws, bytes) != cudaSuccess) {
      (void)cudaGetLastError();
      return record_error(ISDF_ERR_NOMEM, "sharded solve: workspace allocation failed");
    }
    ws_cap = bytes;
  }
  arena->base = ws;
  arena->cap = ws_cap;
  arena->off = 0;
  arena->counting = false;
  return ISDF_OK;
}

namespace {

// ----------------------------------------------------------------- NCCL
struct NcclApi {
  void* h = nullptr;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*CommAbort)(ncclComm_t) = nullptr;
  const char* (*GetErrorString)(ncclResult_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Broadcast)(const void*, void*, size_t, ncclDataType_t, int, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*AllGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t,
                            cudaStream_t) = nullptr;
};

int nccl_api(NcclApi** out) {
  static NcclApi api;
  static std::mutex mu;
  static std::string failure;
  std::lock_guard<std::mutex> g(mu);
  if (!api.h && failure.empty()) {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnccl.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      const char* why = dlerror();  // read once: the call clears the message
      failure = std::string("NCCL not found: ") + (why ? why : "dlopen failed");
    } else {
      bool ok = true;
      auto sym = [&](auto& fn, const char* name) {
        fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(h, name));
        ok = ok && fn;
      };
      sym(api.GetUniqueId, "ncclGetUniqueId");
      sym(api.CommInitRank, "ncclCommInitRank");
      sym(api.CommDestroy, "ncclCommDestroy");
      sym(api.CommAbort, "ncclCommAbort");
      sym(api.GetErrorString, "ncclGetErrorString");
      sym(api.GroupStart, "ncclGroupStart");
      sym(api.GroupEnd, "ncclGroupEnd");
      sym(api.Send, "ncclSend");
      sym(api.Recv, "ncclRecv");
      sym(api.Broadcast, "ncclBroadcast");
      sym(api.AllGather, "ncclAllGather");
      if (ok) {
        api.h = h;
      } else {
        failure = "NCCL library lacks an entry point this library uses";
        dlclose(h);
      }
    }
  }
  if (!api.h) return record_error(ISDF_ERR_UNSUPPORTED, failure.c_str());
  *out = &api;
  return ISDF_OK;
}

int nccl_fail(NcclApi* api, ncclResult_t r, const char* what) {
  std::string m = std::string(what) + ": " + (api->GetErrorString ? api->GetErrorString(r) : "?");
  return record_error(ISDF_ERR_COMM, m.c_str());
}

#define ISDF_NCCL(api, x, what)                          \
  do {                                                   \
    ncclResult_t r_ = (x);                               \
    if (r_ != ncclSuccess) return nccl_fail(api, r_, what); \
  } while (0)

struct NcclTransport : Transport {
  NcclApi* api = nullptr;
  ncclComm_t comm = nullptr;
  ~NcclTransport() override {
    if (comm && api) api->CommDestroy(comm);
  }
  int allgatherv(const void* d_send, size_t send_bytes, void* d_recv, const size_t* counts,
                 const size_t* displs, cudaStream_t s) override {
    if (send_bytes != counts[rank]) return record_error(ISDF_ERR_ARG, "allgatherv: send size");
    bool equal = true;
    for (int q = 0; q < size; ++q)
      equal = equal && counts[q] == counts[0] && displs[q] == (size_t)q * counts[0];
    if (equal) {
      if (counts[0])
        ISDF_NCCL(api, api->AllGather(d_send, d_recv, counts[0], ncclChar, comm, s), "ncclAllGather");
      return ISDF_OK;
    }
    ISDF_NCCL(api, api->GroupStart(), "ncclGroupStart");
    for (int q = 0; q < size; ++q) {
      if (!counts[q]) continue;
      ncclResult_t r = api->Broadcast(q == rank ? d_send : nullptr, (char*)d_recv + displs[q],
                                      counts[q], ncclChar, q, comm, s);
      if (r != ncclSuccess) {
        api->GroupEnd();
        return nccl_fail(api, r, "ncclBroadcast");
      }
    }
    ISDF_NCCL(api, api->GroupEnd(), "ncclGroupEnd");
    return ISDF_OK;
  }
  int alltoallv(const void* d_send, const size_t* send_counts, const size_t* send_displs,
                void* d_recv, const size_t* recv_counts, const size_t* recv_displs,
                cudaStream_t s) override {
    if (send_counts[rank] != recv_counts[rank])
      return record_error(ISDF_ERR_ARG, "alltoallv: own block sizes differ");
    if (send_counts[rank])
      ISDF_CUDA(cudaMemcpyAsync((char*)d_recv + recv_displs[rank],
                                (const char*)d_send + send_displs[rank], send_counts[rank],
                                cudaMemcpyDeviceToDevice, s));
    ISDF_NCCL(api, api->GroupStart(), "ncclGroupStart");
    for (int q = 0; q < size; ++q) {
      if (q == rank) continue;
      ncclResult_t r = ncclSuccess;
      if (send_counts[q])
        r = api->Send((const char*)d_send + send_displs[q], send_counts[q], ncclChar, q, comm, s);
      if (r == ncclSuccess && recv_counts[q])
        r = api->Recv((char*)d_recv + recv_displs[q], recv_counts[q], ncclChar, q, comm, s);
      if (r != ncclSuccess) {
        api->GroupEnd();
        return nccl_fail(api, r, "ncclSend/ncclRecv");
      }
    }
    ISDF_NCCL(api, api->GroupEnd(), "ncclGroupEnd");
    return ISDF_OK;
  }
  int abort() override {
    if (comm && api) {
      api->CommAbort(comm);
      comm = nullptr;
    }
    return ISDF_OK;
  }
};

// ----------------------------------------------------------------- local group
struct LocalGroup {
  int size;
  double timeout_s;
  std::mutex mu;
  std::condition_variable cv;
  int arrived = 0;
  long long generation = 0;
  bool broken = false;
  struct Slot {
    const void* send = nullptr;
    const size_t* counts = nullptr;  // alltoallv: the rank's send counts
    const size_t* displs = nullptr;  // alltoallv: the rank's send displacements
    cudaEvent_t ready = nullptr;     // the rank's send buffer is complete
    cudaEvent_t done = nullptr;      // the rank has read everything it needs
  };
  std::vector<Slot> slots;
  int members = 0;  // live Transport objects

  // All ranks meet here; false when the group broke or the wait ran out.
  bool barrier() {
    std::unique_lock<std::mutex> lk(mu);
    if (broken) return false;
    const long long gen = generation;
    if (++arrived == size) {
      arrived = 0;
      ++generation;
      cv.notify_all();
      return true;
    }
    const bool ok = cv.wait_for(lk, std::chrono::duration<double>(timeout_s),
                                [&] { return generation != gen || broken; });
    if (!ok || broken) {
      broken = true;
      cv.notify_all();
      return false;
    }
    return true;
  }
  void break_group() {
    std::lock_guard<std::mutex> lk(mu);
    broken = true;
    cv.notify_all();
  }
};

struct LocalTransport : Transport {
  std::shared_ptr<LocalGroup> g;
  ~LocalTransport() override {
    LocalGroup::Slot& sl = g->slots[rank];
    int cur = -1;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    if (sl.ready) cudaEventDestroy(sl.ready);
    if (sl.done) cudaEventDestroy(sl.done);
    sl.ready = sl.done = nullptr;
    if (cur >= 0) cudaSetDevice(cur);
  }
  int fail() {
    g->break_group();
    return record_error(ISDF_ERR_COMM, "local group: a rank did not reach the collective in time");
  }
  // Publishes this rank's buffer and waits for all ranks (first round).
  int publish(const void* send, const size_t* counts, const size_t* displs, cudaStream_t s) {
    LocalGroup::Slot& sl = g->slots[rank];
    sl.send = send;
    sl.counts = counts;
    sl.displs = displs;
    ISDF_CUDA(cudaEventRecord(sl.ready, s));
    if (!g->barrier()) return fail();
    return ISDF_OK;
  }
  // Second round: every rank has queued its reads of the others' buffers.
  int finish(cudaStream_t s) {
    ISDF_CUDA(cudaEventRecord(g->slots[rank].done, s));
    if (!g->barrier()) return fail();
    for (int q = 0; q < size; ++q)
      if (q != rank) ISDF_CUDA(cudaStreamWaitEvent(s, g->slots[q].done, 0));
    return ISDF_OK;
  }
  int allgatherv(const void* d_send, size_t send_bytes, void* d_recv, const size_t* counts,
                 const size_t* displs, cudaStream_t s) override {
    if (send_bytes != counts[rank]) return record_error(ISDF_ERR_ARG, "allgatherv: send size");
    ISDF_TRY(publish(d_send, nullptr, nullptr, s));
    for (int q = 0; q < size; ++q) {
      if (!counts[q]) continue;
      ISDF_CUDA(cudaStreamWaitEvent(s, g->slots[q].ready, 0));
      ISDF_CUDA(cudaMemcpyAsync((char*)d_recv + displs[q], g->slots[q].send, counts[q],
                                cudaMemcpyDefault, s));
    }
    return finish(s);
  }
  int alltoallv(const void* d_send, const size_t* send_counts, const size_t* send_displs,
                void* d_recv, const size_t* recv_counts, const size_t* recv_displs,
                cudaStream_t s) override {
    ISDF_TRY(publish(d_send, send_counts, send_displs, s));
    for (int q = 0; q < size; ++q) {
      const LocalGroup::Slot& src = g->slots[q];
      if (src.counts[rank] != recv_counts[q]) {
        g->break_group();
        return record_error(ISDF_ERR_ARG, "alltoallv: send and receive sizes disagree");
      }
      if (!recv_counts[q]) continue;
      ISDF_CUDA(cudaStreamWaitEvent(s, src.ready, 0));
      ISDF_CUDA(cudaMemcpyAsync((char*)d_recv + recv_displs[q],
                                (const char*)src.send + src.displs[rank], recv_counts[q],
                                cudaMemcpyDefault, s));
    }
    return finish(s);
  }
  int abort() override {
    g->break_group();
    return ISDF_OK;
  }
};

// ----------------------------------------------------------------- callbacks
struct CallbackTransport : Transport {
  isdf_comm_ops_t ops;
  void* ctx = nullptr;
  int allgatherv(const void* d_send, size_t send_bytes, void* d_recv, const size_t* counts,
                 const size_t* displs, cudaStream_t s) override {
    int rc = ops.allgatherv(ctx, d_send, send_bytes, d_recv, counts, displs, (void*)s);
    return rc == 0 ? ISDF_OK : record_error(ISDF_ERR_COMM, "caller's allgatherv failed");
  }
  int alltoallv(const void* d_send, const size_t* send_counts, const size_t* send_displs,
                void* d_recv, const size_t* recv_counts, const size_t* recv_displs,
                cudaStream_t s) override {
    int rc = ops.alltoallv(ctx, d_send, send_counts, send_displs, d_recv, recv_counts, recv_displs,
                           (void*)s);
    return rc == 0 ? ISDF_OK : record_error(ISDF_ERR_COMM, "caller's alltoallv failed");
  }
};

}  // namespace
}  // namespace isdf_b200

using namespace isdf_b200;

struct isdf_comm {
  std::unique_ptr<Transport> t;
};

Transport* isdf_comm_transport(isdf_comm_t* c) { return c ? c->t.get() : nullptr; }

extern "C" {

int isdf_comm_nccl_unique_id(unsigned char id[128]) {
  try {
    if (!id) return record_error(ISDF_ERR_ARG, "null id");
    NcclApi* api = nullptr;
    ISDF_TRY(nccl_api(&api));
    ncclUniqueId u;
    ISDF_NCCL(api, api->GetUniqueId(&u), "ncclGetUniqueId");
    static_assert(sizeof(u) == 128, "NCCL unique id size");
    std::memcpy(id, &u, sizeof(u));
    return ISDF_OK;
  } catch (...) {
    return record_error(ISDF_ERR_COMM, "isdf_comm_nccl_unique_id: exception");
  }
}

int isdf_comm_create_nccl(const unsigned char id[128], int rank, int size, isdf_comm_t** out) {
  try {
    if (!id || !out || size < 1 || rank < 0 || rank >= size)
      return record_error(ISDF_ERR_ARG, "isdf_comm_create_nccl: bad arguments");
    *out = nullptr;
    NcclApi* api = nullptr;
    ISDF_TRY(nccl_api(&api));
    auto t = std::make_unique<NcclTransport>();
    t->api = api;
    t->rank = rank;
    t->size = size;
    ISDF_CUDA(cudaGetDevice(&t->device));
    ISDF_TRY(t->ensure_status());
    ncclUniqueId u;
    std::memcpy(&u, id, sizeof(u));
    ISDF_NCCL(api, api->CommInitRank(&t->comm, size, u, rank), "ncclCommInitRank");
    auto* c = new isdf_comm;
    c->t = std::move(t);
    *out = c;
    return ISDF_OK;
  } catch (...) {
    return record_error(ISDF_ERR_COMM, "isdf_comm_create_nccl: exception");
  }
}

int isdf_comm_create_local(int size, const int* devices, double timeout_s, isdf_comm_t** comms) {
  try {
    if (size < 1 || size > 64 || !comms || !(timeout_s > 0))
      return record_error(ISDF_ERR_ARG, "isdf_comm_create_local: bad arguments");
    auto g = std::make_shared<LocalGroup>();
    g->size = size;
    g->timeout_s = timeout_s;
    g->slots.resize(size);
    int cur = 0;
    ISDF_CUDA(cudaGetDevice(&cur));
    std::vector<isdf_comm*> made;
    for (int r = 0; r < size; ++r) {
      auto t = std::make_unique<LocalTransport>();
      t->g = g;
      t->rank = r;
      t->size = size;
      t->device = devices ? devices[r] : cur;
      int rc = ISDF_OK;
      if (cudaSetDevice(t->device) != cudaSuccess ||
          cudaEventCreateWithFlags(&g->slots[r].ready, cudaEventDisableTiming) != cudaSuccess ||
          cudaEventCreateWithFlags(&g->slots[r].done, cudaEventDisableTiming) != cudaSuccess)
        rc = record_error(ISDF_ERR_CUDA, "isdf_comm_create_local: device or event setup failed");
      if (rc == ISDF_OK) rc = t->ensure_status();
      if (rc != ISDF_OK) {
        for (auto* m : made) delete m;
        cudaSetDevice(cur);
        return rc;
      }
      auto* c = new isdf_comm;
      c->t = std::move(t);
      made.push_back(c);
    }
    ISDF_CUDA(cudaSetDevice(cur));
    for (int r = 0; r < size; ++r) comms[r] = made[r];
    return ISDF_OK;
  } catch (...) {
    return record_error(ISDF_ERR_COMM, "isdf_comm_create_local: exception");
  }
}

int isdf_comm_create_callbacks(const isdf_comm_ops_t* ops, void* ctx, int rank, int size,
                               isdf_comm_t** out) {
  try {
    if (!ops || !ops->allgatherv || !ops->alltoallv || !out || size < 1 || rank < 0 ||
        rank >= size)
      return record_error(ISDF_ERR_ARG, "isdf_comm_create_callbacks: bad arguments");
    auto t = std::make_unique<CallbackTransport>();
    t->ops = *ops;
    t->ctx = ctx;
    t->rank = rank;
    t->size = size;
    ISDF_CUDA(cudaGetDevice(&t->device));
    ISDF_TRY(t->ensure_status());
    auto* c = new isdf_comm;
    c->t = std::move(t);
    *out = c;
    return ISDF_OK;
  } catch (...) {
    return record_error(ISDF_ERR_COMM, "isdf_comm_create_callbacks: exception");
  }
}

int isdf_comm_rank(const isdf_comm_t* comm, int* rank, int* size) {
  if (!comm || !comm->t) return record_error(ISDF_ERR_ARG, "null comm");
  if (rank) *rank = comm->t->rank;
  if (size) *size = comm->t->size;
  return ISDF_OK;
}

int isdf_comm_abort(isdf_comm_t* comm) {
  if (!comm || !comm->t) return record_error(ISDF_ERR_ARG, "null comm");
  return comm->t->abort();
}

int isdf_comm_destroy(isdf_comm_t* comm) {
  try {
    delete comm;
    return ISDF_OK;
  } catch (...) {
    return record_error(ISDF_ERR_COMM, "isdf_comm_destroy: exception");
  }
}

int isdf_row_block(long long n, int size, int rank, long long* start, long long* count) {
  if (n < 0 || size < 1 || rank < 0 || rank >= size || !start || !count)
    return record_error(ISDF_ERR_ARG, "isdf_row_block: bad arguments");
  *start = block_start(n, size, rank);
  *count = block_count(n, size, rank);
  return ISDF_OK;
}

}  // extern "C"
