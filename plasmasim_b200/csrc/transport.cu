// Transports for the exchanges between ranks of a decomposed run (the
// pic_transport interface of plasma_b200.h):
//  - pic_group: the ranks are contexts of one process, one host thread each;
//    a sendrecv posts the send buffer with a CUDA event that marks it ready,
//    takes the partner's posted buffer, copies it on its own stream after that
//    event, and hands back an event that marks the copy done, which the
//    sender's stream waits on before it may overwrite its buffer. No kernel
//    ever waits for another rank: every rendezvous is on the host, with a
//    time limit.
//  - NCCL: ncclSend/ncclRecv in one group per sendrecv, ncclAllReduce for the
//    sums; libnccl.so.2 is loaded with dlopen on first use.
#include <cuda_runtime.h>
#include <dlfcn.h>
#include <nccl.h>

#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <new>
#include <vector>

#include "../../include/plasma_b200.h"

namespace {

constexpr int kMaxRanks = 64;
constexpr int kDefaultTimeoutMs = 60000;

struct Msg {
  const void* ptr = nullptr;
  size_t bytes = 0;
  cudaEvent_t ready = nullptr;  // recorded on the sender's stream after its writes
  cudaEvent_t done = nullptr;   // recorded on the receiver's stream after its copy
  bool taken = false;
};

struct Member;

}  // namespace

struct pic_group {
  int n = 0;
  int timeout_ms = kDefaultTimeoutMs;  // host rendezvous limit of every exchange
  std::mutex mu;
  std::condition_variable cv;
  std::deque<Msg*> box[kMaxRanks][kMaxRanks];  // box[dest][src], FIFO per pair
  // allreduce rendezvous
  std::vector<std::vector<double>> part;
  int arrived = 0, departed = 0;
  unsigned long long gen = 0;
  std::vector<Member*> members;
};

namespace {

struct Member {
  pic_group* g;
  int rank;
};

int group_sendrecv(void* user, const void* send, size_t send_bytes, int dest, void* recv, size_t recv_bytes,
                   int src, void* stream_p) {
  Member* me = static_cast<Member*>(user);
  pic_group* g = me->g;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  if (dest < 0 || dest >= g->n || src < 0 || src >= g->n) return 1;
  Msg* out = new (std::nothrow) Msg();
  if (!out) return 1;
  out->ptr = send;
  out->bytes = send_bytes;
  if (cudaEventCreateWithFlags(&out->ready, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(out->ready, stream) != cudaSuccess) {
    delete out;
    return 1;
  }
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(g->timeout_ms);
  {
    std::lock_guard<std::mutex> lk(g->mu);
    g->box[dest][me->rank].push_back(out);
  }
  g->cv.notify_all();
  // take the partner's message
  Msg* in = nullptr;
  {
    std::unique_lock<std::mutex> lk(g->mu);
    auto& q = g->box[me->rank][src];
    if (!g->cv.wait_until(lk, deadline, [&] { return !q.empty(); })) {
      fprintf(stderr, "plasma_b200: rank %d: no message from rank %d within %d ms\n", me->rank, src, g->timeout_ms);
      return 1;
    }
    in = q.front();
    q.pop_front();
  }
  int rc = 0;
  cudaEvent_t done = nullptr;
  if (cudaStreamWaitEvent(stream, in->ready, 0) != cudaSuccess) rc = 1;
  const size_t n = in->bytes < recv_bytes ? in->bytes : recv_bytes;
  if (!rc && n > 0 && cudaMemcpyAsync(recv, in->ptr, n, cudaMemcpyDeviceToDevice, stream) != cudaSuccess) rc = 1;
  if (cudaEventCreateWithFlags(&done, cudaEventDisableTiming) != cudaSuccess ||
      cudaEventRecord(done, stream) != cudaSuccess)
    rc = 1;
  {
    std::lock_guard<std::mutex> lk(g->mu);
    in->done = done;
    in->taken = true;
  }
  g->cv.notify_all();
  // wait until the partner has queued its copy of our buffer
  {
    std::unique_lock<std::mutex> lk(g->mu);
    if (!g->cv.wait_until(lk, deadline, [&] { return out->taken; })) {
      fprintf(stderr, "plasma_b200: rank %d: rank %d did not take its message within %d ms\n", me->rank, dest,
              g->timeout_ms);
      return 1;  // `out` stays queued; the group is unusable after a timeout
    }
  }
  if (out->done && cudaStreamWaitEvent(stream, out->done, 0) != cudaSuccess) rc = 1;
  cudaEventDestroy(out->ready);
  if (out->done) cudaEventDestroy(out->done);
  delete out;
  return rc;
}

int group_allreduce(void* user, double* buf, int n, void* stream_p) {
  Member* me = static_cast<Member*>(user);
  pic_group* g = me->g;
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  std::vector<double> h((size_t)n);
  if (cudaMemcpyAsync(h.data(), buf, sizeof(double) * n, cudaMemcpyDeviceToHost, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return 1;
  const auto deadline = std::chrono::steady_clock::now() + std::chrono::milliseconds(g->timeout_ms);
  std::vector<double> sum((size_t)n, 0.0);
  {
    std::unique_lock<std::mutex> lk(g->mu);
    // a rank that comes back before everyone has left the previous reduction waits
    if (!g->cv.wait_until(lk, deadline, [&] { return g->departed == 0; })) return 1;
    const unsigned long long gen = g->gen;
    g->part[me->rank] = h;
    ++g->arrived;
    g->cv.notify_all();
    if (!g->cv.wait_until(lk, deadline, [&] { return g->arrived == g->n || g->gen != gen; })) {
      fprintf(stderr, "plasma_b200: rank %d: allreduce partners missing after %d ms\n", me->rank, g->timeout_ms);
      return 1;
    }
    for (int r = 0; r < g->n; ++r)  // rank order: the same bits on every rank
      for (int q = 0; q < n; ++q) sum[q] += g->part[r][q];
    if (++g->departed == g->n) {
      g->arrived = 0;
      g->departed = 0;
      ++g->gen;
    }
    g->cv.notify_all();
  }
  if (cudaMemcpyAsync(buf, sum.data(), sizeof(double) * n, cudaMemcpyHostToDevice, stream) != cudaSuccess ||
      cudaStreamSynchronize(stream) != cudaSuccess)
    return 1;
  return 0;
}

// --------------------------------------------------------------- NCCL
struct NcclApi {
  bool loaded = false;
  ncclResult_t (*GetUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*CommInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*CommDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*Send)(const void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*Recv)(void*, size_t, ncclDataType_t, int, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*AllReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  ncclResult_t (*GroupStart)() = nullptr;
  ncclResult_t (*GroupEnd)() = nullptr;
};

NcclApi& nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void* h = dlopen("libnccl.so.2", RTLD_NOW | RTLD_GLOBAL);
    if (!h) {
      fprintf(stderr, "plasma_b200: cannot load libnccl.so.2: %s\n", dlerror());
      return;
    }
    api.GetUniqueId = reinterpret_cast<decltype(api.GetUniqueId)>(dlsym(h, "ncclGetUniqueId"));
    api.CommInitRank = reinterpret_cast<decltype(api.CommInitRank)>(dlsym(h, "ncclCommInitRank"));
    api.CommDestroy = reinterpret_cast<decltype(api.CommDestroy)>(dlsym(h, "ncclCommDestroy"));
    api.Send = reinterpret_cast<decltype(api.Send)>(dlsym(h, "ncclSend"));
    api.Recv = reinterpret_cast<decltype(api.Recv)>(dlsym(h, "ncclRecv"));
    api.AllReduce = reinterpret_cast<decltype(api.AllReduce)>(dlsym(h, "ncclAllReduce"));
    api.GroupStart = reinterpret_cast<decltype(api.GroupStart)>(dlsym(h, "ncclGroupStart"));
    api.GroupEnd = reinterpret_cast<decltype(api.GroupEnd)>(dlsym(h, "ncclGroupEnd"));
    api.loaded = api.GetUniqueId && api.CommInitRank && api.CommDestroy && api.Send && api.Recv && api.AllReduce &&
                 api.GroupStart && api.GroupEnd;
  });
  return api;
}

struct NcclMember {
  ncclComm_t comm = nullptr;
  int device = 0;
};

int nccl_sendrecv(void* user, const void* send, size_t send_bytes, int dest, void* recv, size_t recv_bytes, int src,
                  void* stream_p) {
  NcclMember* m = static_cast<NcclMember*>(user);
  NcclApi& a = nccl();
  cudaStream_t stream = static_cast<cudaStream_t>(stream_p);
  if (a.GroupStart() != ncclSuccess) return 1;
  ncclResult_t r1 = ncclSuccess, r2 = ncclSuccess;
  if (send_bytes > 0) r1 = a.Send(send, send_bytes, ncclInt8, dest, m->comm, stream);
  if (recv_bytes > 0) r2 = a.Recv(recv, recv_bytes, ncclInt8, src, m->comm, stream);
  const ncclResult_t r3 = a.GroupEnd();
  return (r1 != ncclSuccess || r2 != ncclSuccess || r3 != ncclSuccess) ? 1 : 0;
}

int nccl_allreduce(void* user, double* buf, int n, void* stream_p) {
  NcclMember* m = static_cast<NcclMember*>(user);
  return nccl().AllReduce(buf, buf, (size_t)n, ncclFloat64, ncclSum, m->comm, static_cast<cudaStream_t>(stream_p)) ==
                 ncclSuccess
             ? 0
             : 1;
}

}  // namespace

extern "C" {

int pic_group_create(int nranks, pic_group** out) {
  if (!out || nranks < 1 || nranks > kMaxRanks) return PIC_ERR_ARG;
  pic_group* g = new (std::nothrow) pic_group();
  if (!g) return PIC_ERR_ARG;
  g->n = nranks;
  g->part.assign((size_t)nranks, std::vector<double>());
  for (int r = 0; r < nranks; ++r) g->members.push_back(new Member{g, r});
  *out = g;
  return PIC_OK;
}

int pic_group_destroy(pic_group* g) {
  if (!g) return PIC_OK;
  for (int d = 0; d < g->n; ++d)
    for (int s = 0; s < g->n; ++s)
      for (Msg* m : g->box[d][s]) {
        if (m->ready) cudaEventDestroy(m->ready);
        delete m;
      }
  for (Member* m : g->members) delete m;
  delete g;
  return PIC_OK;
}

int pic_group_set_timeout(pic_group* g, int ms) {
  if (!g || ms < 1) return PIC_ERR_ARG;
  std::lock_guard<std::mutex> lk(g->mu);
  g->timeout_ms = ms;
  return PIC_OK;
}

int pic_group_transport(pic_group* g, int rank, pic_transport* out) {
  if (!g || !out || rank < 0 || rank >= g->n) return PIC_ERR_ARG;
  out->user = g->members[rank];
  out->sendrecv = group_sendrecv;
  out->allreduce_sum_f64 = group_allreduce;
  return PIC_OK;
}

int pic_nccl_unique_id(unsigned char id[128]) {
  if (!id) return PIC_ERR_ARG;
  NcclApi& a = nccl();
  if (!a.loaded) return PIC_ERR_COMM;
  ncclUniqueId u;
  if (a.GetUniqueId(&u) != ncclSuccess) return PIC_ERR_COMM;
  static_assert(sizeof(u) == 128, "NCCL unique id is 128 bytes");
  std::memcpy(id, &u, 128);
  return PIC_OK;
}

int pic_nccl_transport_create(const unsigned char id[128], int nranks, int rank, int device, pic_transport* out) {
  if (!id || !out || nranks < 1 || rank < 0 || rank >= nranks) return PIC_ERR_ARG;
  NcclApi& a = nccl();
  if (!a.loaded) return PIC_ERR_COMM;
  if (cudaSetDevice(device) != cudaSuccess) return PIC_ERR_CUDA;
  NcclMember* m = new (std::nothrow) NcclMember();
  if (!m) return PIC_ERR_ARG;
  m->device = device;
  ncclUniqueId u;
  std::memcpy(&u, id, 128);
  if (a.CommInitRank(&m->comm, nranks, u, rank) != ncclSuccess) {
    delete m;
    return PIC_ERR_COMM;
  }
  out->user = m;
  out->sendrecv = nccl_sendrecv;
  out->allreduce_sum_f64 = nccl_allreduce;
  return PIC_OK;
}

int pic_nccl_transport_destroy(pic_transport* t) {
  if (!t || !t->user) return PIC_ERR_ARG;
  NcclMember* m = static_cast<NcclMember*>(t->user);
  if (m->comm) nccl().CommDestroy(m->comm);
  delete m;
  t->user = nullptr;
  t->sendrecv = nullptr;
  t->allreduce_sum_f64 = nullptr;
  return PIC_OK;
}

}  // extern "C"
