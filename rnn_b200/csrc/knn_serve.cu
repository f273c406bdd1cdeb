// knn_serve.cu -- the serving form: a request loop against a device-resident reference set.
//
// The reference has no serving path; a caller would run sgsknn once per request. Here:
//   * the reference set is prepared once (packed in the tensor-core format with its norms and
//     bound statistics, tc_cand_prepare) and stays resident;
//   * gsknn_serve_submit() queues a request (m query rows copied from the caller, a k);
//   * a dispatcher thread admits queued requests in arrival order while their result heaps fit
//     the heap arena (the HBM budget), packs admitted requests into batches of at most
//     `max_batch_queries` rows, and launches each batch on a free stream slot, so batches formed
//     from later arrivals run while earlier ones are still on the GPU (continuous batching);
//   * per batch: one host-to-device copy of the queries, their norms, the tensor-core pass with
//     the exact FP64 re-rank (tc_run_prepared) at the batch's largest k, and a scatter kernel
//     that writes each request's k smallest into its own heap, which stays on the device until
//     the caller releases the request;
//   * a host function queued behind the batch marks its requests done (no polling).
// Results are the exact FP64 top-k of each query (ties to the lower id), so they are identical
// whatever a request was batched with.
#include "gsknn.h"
#include "knn_common.cuh"
#include "knn_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

namespace gsknn {
struct Engine;
namespace serve {

// |q|^2 of each query row, accumulated in FP64 and rounded to float (one warp per row)
__global__ void query_norms(const float *__restrict__ Q, int d, int n, float *__restrict__ Q2) {
  const int lane = threadIdx.x & 31;
  const int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (r >= n) return;
  double s = 0.0;
  for (int p = lane; p < d; p += 32) {
    const double v = (double)Q[(size_t)r * d + p];
    s += v * v;
  }
  for (int o = 16; o; o >>= 1) s += __shfl_xor_sync(FULL_MASK, s, o);
  if (lane == 0) Q2[r] = (float)s;
}

__global__ void iota(int *__restrict__ a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) a[i] = i;
}

__global__ void fill_heap(float *__restrict__ D, int *__restrict__ I, long long n) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) {
    D[i] = Num<float>::inf();
    I[i] = -1;
  }
}

struct ReqDesc {     // one request of a batch, for the scatter kernel
  int row0, m, k, pad;
  float *D;          // its heap, m x k
  int *I;
};

// Batch rows are written in descending order (k_b entries, the k_b-th distance first): the
// request's k smallest are the last k of its rows, written again in descending order.
__global__ void scatter(const float *__restrict__ Db, const int *__restrict__ Ib, int kb,
                        const ReqDesc *__restrict__ reqs, int nreq, int total_rows) {
  const int r = blockIdx.x * blockDim.y + threadIdx.y;  // batch row
  if (r >= total_rows) return;
  int lo = 0, hi = nreq - 1;  // request holding row r
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (reqs[mid].row0 <= r) lo = mid;
    else hi = mid - 1;
  }
  const ReqDesc q = reqs[lo];
  const int j = r - q.row0;
  for (int t = threadIdx.x; t < q.k; t += blockDim.x) {
    q.D[(size_t)j * q.k + t] = Db[(size_t)r * kb + (kb - q.k) + t];
    q.I[(size_t)j * q.k + t] = Ib[(size_t)r * kb + (kb - q.k) + t];
  }
}

// First-fit allocator over a fixed byte range (the heap arena).
class Arena {
 public:
  explicit Arena(size_t bytes) { free_[0] = bytes; }
  // offset, or -1 when no free range fits
  long long alloc(size_t n) {
    n = (n + 255) & ~(size_t)255;
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= n) {
        const size_t off = it->first, len = it->second;
        free_.erase(it);
        if (len > n) free_[off + n] = len - n;
        used_ += n;
        return (long long)off;
      }
    }
    return -1;
  }
  void release(size_t off, size_t n) {
    n = (n + 255) & ~(size_t)255;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t used_ = 0;
};

using Clock = std::chrono::steady_clock;

struct Request {
  long long id;
  int m, k;
  std::vector<float> q;     // the caller's query rows
  long long heap_off = -1;  // in the arena
  size_t heap_bytes = 0;
  float *D = nullptr;
  int *I = nullptr;
  int state = 0;            // 0 queued, 1 admitted, 2 running, 3 done, 4 failed
  int batch = -1, batch_rows = 0;
  Clock::time_point t_submit, t_launch, t_done;
};

struct Slot {
  cudaStream_t st = nullptr;
  bool busy = false;
  float *Xq = nullptr, *Xq2 = nullptr, *Db = nullptr;
  int *Ib = nullptr, *qidx = nullptr, *status = nullptr;
  ReqDesc *reqs_d = nullptr;
  void *ws = nullptr;
  float *h_q = nullptr;       // pinned staging of the batch's queries
  ReqDesc *h_reqs = nullptr;  // pinned staging of the request table
  std::vector<std::shared_ptr<Request>> batch;
  gsknn::Engine *eng = nullptr;
  int index = 0;
};

}  // namespace serve

struct Engine {
  int device;
  int nref, d, mode, max_q, max_k, kp_max, sms, nslots;
  size_t heap_budget;
  TcCand C{};
  void *cand_mem = nullptr;
  int *cidx = nullptr, *status = nullptr;
  char *arena_mem = nullptr;
  std::unique_ptr<serve::Arena> arena;
  size_t ws_bytes = 0;
  std::vector<serve::Slot> slots;
  std::mutex mu;
  std::condition_variable cv;     // dispatcher: work or a free slot
  std::condition_variable done_cv;  // waiters: a request finished
  std::deque<std::shared_ptr<serve::Request>> queue;  // queued or admitted, not launched
  std::map<long long, std::shared_ptr<serve::Request>> reqs;
  long long next_id = 0;
  int next_batch = 0;
  bool stop = false;
  bool paused = false;  // no new batches while set (requests still queue and are admitted)
  int error = 0;
  char errmsg[256] = {0};
  std::thread dispatcher;
};

}  // namespace gsknn

using gsknn::Engine;
namespace gs = gsknn::serve;

static int serr(int code, const char *msg) { return gsknn::set_status(code, "%s", msg); }

// Host function queued behind a batch: marks its requests done and frees the slot.
static void CUDART_CB batch_done(void *p) {
  gs::Slot *s = static_cast<gs::Slot *>(p);
  Engine *E = s->eng;
  const auto now = gs::Clock::now();
  {
    std::lock_guard<std::mutex> lk(E->mu);
    int st = 0;
    std::memcpy(&st, s->h_reqs + E->max_q, sizeof(int));  // status copied back by the batch
    for (auto &r : s->batch) {
      r->t_done = now;
      r->state = st == 0 ? 3 : 4;
    }
    s->batch.clear();
    s->busy = false;
  }
  E->cv.notify_all();
  E->done_cv.notify_all();
}

// Launch one batch on slot s (called by the dispatcher without the lock held).
static cudaError_t launch_batch(Engine *E, gs::Slot &s) {
  using namespace gsknn;
  int rows = 0, kb = 0;
  const int nreq = (int)s.batch.size();
  for (int i = 0; i < nreq; i++) {
    auto &r = s.batch[i];
    std::memcpy(s.h_q + (size_t)rows * E->d, r->q.data(), (size_t)r->m * E->d * 4);
    s.h_reqs[i] = {rows, r->m, r->k, 0, r->D, r->I};
    rows += r->m;
    kb = std::max(kb, r->k);
  }
  const TcPlan P = tc_plan(rows, E->nref, E->d, kb, E->mode, E->sms, false, E->sms);
  if (!P.ok || P.bytes > E->ws_bytes) return cudaErrorInvalidValue;
  cudaStream_t st = s.st;
  cudaError_t e = cudaMemcpyAsync(s.Xq, s.h_q, (size_t)rows * E->d * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.reqs_d, s.h_reqs, (size_t)nreq * sizeof(gs::ReqDesc),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.status, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  gs::query_norms<<<(rows + 7) / 8, 256, 0, st>>>(s.Xq, E->d, rows, s.Xq2);
  const long long n = (long long)rows * kb;
  gs::fill_heap<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s.Db, s.Ib, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = tc_run_prepared(P, E->C, rows, E->d, kb, s.Xq, s.Xq2, E->max_q, s.qidx, s.Db, s.Ib, kb,
                      s.ws, s.status, nullptr, 0, nullptr, st, nullptr, nullptr);
  if (e != cudaSuccess) return e;
  dim3 blk(32, 8);
  gs::scatter<<<(rows + 7) / 8, blk, 0, st>>>(s.Db, s.Ib, kb, s.reqs_d, nreq, rows);
  e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_reqs + E->max_q, s.status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaLaunchHostFunc(st, batch_done, &s);
  return e;
}

static void dispatcher_loop(Engine *E) {
  const int dev = E->device;
  cudaSetDevice(dev);
  while (true) {
    std::unique_lock<std::mutex> lk(E->mu);
    gs::Slot *slot = nullptr;
    E->cv.wait(lk, [&] {
      if (E->stop) return true;
      if (E->paused) return false;
      slot = nullptr;
      for (auto &s : E->slots)
        if (!s.busy) { slot = &s; break; }
      if (!slot || E->queue.empty()) return false;
      // admit in arrival order while the heaps fit the arena
      for (auto &r : E->queue) {
        if (r->state != 0) continue;
        const long long off = E->arena->alloc(r->heap_bytes);
        if (off < 0) break;
        r->heap_off = off;
        r->D = reinterpret_cast<float *>(E->arena_mem + off);
        r->I = reinterpret_cast<int *>(E->arena_mem + off + (size_t)r->m * r->k * 4);
        r->state = 1;
      }
      return !E->queue.empty() && E->queue.front()->state == 1;
    });
    if (E->stop) return;
    // batch: admitted requests from the front, up to max_q rows
    int rows = 0, bid = E->next_batch++;
    while (!E->queue.empty() && E->queue.front()->state == 1 &&
           rows + E->queue.front()->m <= E->max_q) {
      auto r = E->queue.front();
      E->queue.pop_front();
      r->state = 2;
      r->batch = bid;
      r->t_launch = gs::Clock::now();
      rows += r->m;
      slot->batch.push_back(r);
    }
    for (auto &r : slot->batch) r->batch_rows = rows;
    slot->busy = true;
    lk.unlock();
    cudaSetDevice(dev);
    const cudaError_t e = launch_batch(E, *slot);
    if (e != cudaSuccess) {
      std::lock_guard<std::mutex> g(E->mu);
      E->error = GSKNN_ERR_CUDA;
      std::snprintf(E->errmsg, sizeof(E->errmsg), "serving batch launch failed: %s",
                    cudaGetErrorString(e));
      for (auto &r : slot->batch) {
        r->state = 4;
        r->t_done = gs::Clock::now();
      }
      slot->batch.clear();
      slot->busy = false;
      E->done_cv.notify_all();
    }
  }
}

extern "C" {

gsknn_serve_t *gsknn_serve_create(const float *R, const float *R2, int nref, int d, int mode,
                                  int max_batch_queries, int max_k, size_t heap_budget,
                                  int slots) {
  using namespace gsknn;
  if (!R || !R2 || nref <= 0 || d <= 0 || max_batch_queries <= 0 || max_k <= 0 ||
      max_k > 256 || slots <= 0 || heap_budget == 0) {
    serr(GSKNN_ERR_ARG, "gsknn_serve_create: invalid argument");
    return nullptr;
  }
  if (mode == GSKNN_MODE_AUTO)
    mode = tc_plan(max_batch_queries, nref, d, max_k, GSKNN_TC_BF16X3, 148, false, 148).ok
               ? GSKNN_MODE_BF16X3
               : GSKNN_MODE_TF32;
  if (mode < GSKNN_MODE_TF32 || mode > GSKNN_MODE_BF16X3) {
    serr(GSKNN_ERR_ARG, "gsknn_serve_create: mode must be AUTO, TF32, BF16 or BF16X3");
    return nullptr;
  }
  auto E = std::make_unique<Engine>();
  E->nref = nref; E->d = d; E->mode = mode; E->max_q = max_batch_queries; E->max_k = max_k;
  E->heap_budget = heap_budget; E->nslots = slots;
  E->kp_max = 32;
  while (E->kp_max < max_k) E->kp_max <<= 1;
  int dev = 0;
  cudaGetDevice(&dev);
  E->device = dev;
  cudaDeviceGetAttribute(&E->sms, cudaDevAttrMultiProcessorCount, dev);
  // query-side workspace: the largest plan over batch sizes (whole query tiles) and k
  for (int kk = 1; kk <= max_k; kk++)
    for (int q = 128; q < E->max_q + 128; q += 128) {
      const TcPlan P = tc_plan(std::min(q, E->max_q), nref, d, kk, mode, E->sms, false, E->sms);
      if (!P.ok) {
        serr(GSKNN_ERR_UNSUPPORTED, "gsknn_serve_create: d or k outside the tensor-core form");
        return nullptr;
      }
      E->ws_bytes = std::max(E->ws_bytes, P.bytes);
    }
  const size_t cb = tc_cand_bytes(nref, d, mode);
  bool ok = cudaMalloc(&E->cand_mem, cb) == cudaSuccess &&
            cudaMalloc((void **)&E->cidx, (size_t)nref * 4) == cudaSuccess &&
            cudaMalloc((void **)&E->status, 4) == cudaSuccess &&
            cudaMalloc((void **)&E->arena_mem, heap_budget) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    serr(GSKNN_ERR_NOMEM, "gsknn_serve_create: device memory exhausted");
    gsknn_serve_destroy(reinterpret_cast<gsknn_serve_t *>(E.release()));
    return nullptr;
  }
  E->arena = std::make_unique<gs::Arena>(heap_budget);
  cudaStream_t st0 = nullptr;
  cudaStreamCreateWithFlags(&st0, cudaStreamNonBlocking);
  gs::iota<<<(nref + 255) / 256, 256, 0, st0>>>(E->cidx, nref);
  cudaMemsetAsync(E->status, 0, 4, st0);
  cudaError_t e = tc_cand_prepare(&E->C, E->cand_mem, nref, d, mode, R, R2, nref, E->cidx,
                                  E->status, st0);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st0);
  int st = 0;
  if (e == cudaSuccess) e = cudaMemcpy(&st, E->status, 4, cudaMemcpyDeviceToHost);
  cudaStreamDestroy(st0);
  if (e != cudaSuccess || st != 0) {
    serr(GSKNN_ERR_CUDA, "gsknn_serve_create: preparing the reference set failed");
    gsknn_serve_destroy(reinterpret_cast<gsknn_serve_t *>(E.release()));
    return nullptr;
  }
  E->slots.resize(slots);
  for (int i = 0; i < slots; i++) {
    gs::Slot &s = E->slots[i];
    s.eng = E.get();
    s.index = i;
    const size_t q = (size_t)E->max_q;
    ok = cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking) == cudaSuccess &&
         cudaMalloc((void **)&s.Xq, q * d * 4) == cudaSuccess &&
         cudaMalloc((void **)&s.Xq2, q * 4) == cudaSuccess &&
         cudaMalloc((void **)&s.Db, q * E->kp_max * 4) == cudaSuccess &&
         cudaMalloc((void **)&s.Ib, q * E->kp_max * 4) == cudaSuccess &&
         cudaMalloc((void **)&s.qidx, q * 4) == cudaSuccess &&
         cudaMalloc((void **)&s.status, 4) == cudaSuccess &&
         cudaMalloc((void **)&s.reqs_d, (q + 1) * sizeof(gs::ReqDesc)) == cudaSuccess &&
         cudaMalloc(&s.ws, E->ws_bytes) == cudaSuccess &&
         cudaHostAlloc((void **)&s.h_q, q * d * 4, cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc((void **)&s.h_reqs, (q + 1) * sizeof(gs::ReqDesc),
                       cudaHostAllocDefault) == cudaSuccess;
    if (!ok) break;
    gs::iota<<<(E->max_q + 255) / 256, 256, 0, s.st>>>(s.qidx, E->max_q);
    ok = cudaStreamSynchronize(s.st) == cudaSuccess;
    if (!ok) break;
  }
  if (!ok) {
    cudaGetLastError();
    serr(GSKNN_ERR_NOMEM, "gsknn_serve_create: slot buffers could not be allocated");
    gsknn_serve_destroy(reinterpret_cast<gsknn_serve_t *>(E.release()));
    return nullptr;
  }
  Engine *raw = E.release();
  raw->dispatcher = std::thread(dispatcher_loop, raw);
  set_status(GSKNN_OK, nullptr);
  return reinterpret_cast<gsknn_serve_t *>(raw);
}

long long gsknn_serve_submit(gsknn_serve_t *eng, const float *Q, int m, int k) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E || !Q || m <= 0 || k <= 0) return serr(GSKNN_ERR_ARG, "gsknn_serve_submit: bad args") * -1LL;
  if (m > E->max_q || k > E->max_k)
    return -1LL * serr(GSKNN_ERR_UNSUPPORTED,
                       "gsknn_serve_submit: m above max_batch_queries or k above max_k");
  const size_t hb = (size_t)m * k * 8;
  if (hb > E->heap_budget)
    return -1LL * serr(GSKNN_ERR_UNSUPPORTED, "gsknn_serve_submit: heap larger than the budget");
  auto r = std::make_shared<gs::Request>();
  r->m = m;
  r->k = k;
  r->q.assign(Q, Q + (size_t)m * E->d);
  r->heap_bytes = hb;
  r->t_submit = gs::Clock::now();
  long long id;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    id = E->next_id++;
    r->id = id;
    E->reqs[id] = r;
    E->queue.push_back(r);
  }
  E->cv.notify_all();
  gsknn::set_status(GSKNN_OK, nullptr);
  return id;
}

// 1 done, 0 pending, negative: unknown request or failed
int gsknn_serve_test(gsknn_serve_t *eng, long long id) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return -GSKNN_ERR_ARG;
  std::lock_guard<std::mutex> lk(E->mu);
  auto it = E->reqs.find(id);
  if (it == E->reqs.end()) return -GSKNN_ERR_ARG;
  const int st = it->second->state;
  return st == 3 ? 1 : st == 4 ? -GSKNN_ERR_CUDA : 0;
}

int gsknn_serve_wait(gsknn_serve_t *eng, long long id, double timeout_s) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return serr(GSKNN_ERR_ARG, "gsknn_serve_wait: null engine");
  std::unique_lock<std::mutex> lk(E->mu);
  auto it = E->reqs.find(id);
  if (it == E->reqs.end()) return serr(GSKNN_ERR_ARG, "gsknn_serve_wait: unknown request");
  auto r = it->second;
  const auto until = gs::Clock::now() + std::chrono::duration_cast<gs::Clock::duration>(
                                            std::chrono::duration<double>(timeout_s));
  if (!E->done_cv.wait_until(lk, until, [&] { return r->state >= 3; }))
    return serr(GSKNN_ERR_TIMEOUT, "gsknn_serve_wait: timed out");
  if (r->state == 4)
    return serr(GSKNN_ERR_CUDA, E->errmsg[0] ? E->errmsg : "serving batch failed");
  gsknn::set_status(GSKNN_OK, nullptr);
  return GSKNN_OK;
}

int gsknn_serve_heap(gsknn_serve_t *eng, long long id, float **D, int **I) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return serr(GSKNN_ERR_ARG, "gsknn_serve_heap: null engine");
  std::lock_guard<std::mutex> lk(E->mu);
  auto it = E->reqs.find(id);
  if (it == E->reqs.end() || it->second->state != 3)
    return serr(GSKNN_ERR_ARG, "gsknn_serve_heap: unknown or unfinished request");
  if (D) *D = it->second->D;
  if (I) *I = it->second->I;
  return GSKNN_OK;
}

int gsknn_serve_fetch(gsknn_serve_t *eng, long long id, float *D, int *I) {
  float *dD = nullptr;
  int *dI = nullptr;
  const int rc = gsknn_serve_heap(eng, id, &dD, &dI);
  if (rc != GSKNN_OK) return rc;
  Engine *E = reinterpret_cast<Engine *>(eng);
  size_t n;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    auto &r = E->reqs[id];
    n = (size_t)r->m * r->k;
  }
  if (cudaMemcpy(D, dD, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess ||
      cudaMemcpy(I, dI, n * 4, cudaMemcpyDeviceToHost) != cudaSuccess)
    return serr(GSKNN_ERR_CUDA, "gsknn_serve_fetch: copy failed");
  gsknn::set_status(GSKNN_OK, nullptr);
  return GSKNN_OK;
}

int gsknn_serve_stats(gsknn_serve_t *eng, long long id, double *queue_ms, double *total_ms,
                      int *batch, int *batch_rows) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return serr(GSKNN_ERR_ARG, "gsknn_serve_stats: null engine");
  std::lock_guard<std::mutex> lk(E->mu);
  auto it = E->reqs.find(id);
  if (it == E->reqs.end() || it->second->state != 3)
    return serr(GSKNN_ERR_ARG, "gsknn_serve_stats: unknown or unfinished request");
  auto &r = it->second;
  using ms = std::chrono::duration<double, std::milli>;
  if (queue_ms) *queue_ms = ms(r->t_launch - r->t_submit).count();
  if (total_ms) *total_ms = ms(r->t_done - r->t_submit).count();
  if (batch) *batch = r->batch;
  if (batch_rows) *batch_rows = r->batch_rows;
  return GSKNN_OK;
}

int gsknn_serve_release(gsknn_serve_t *eng, long long id) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return serr(GSKNN_ERR_ARG, "gsknn_serve_release: null engine");
  {
    std::lock_guard<std::mutex> lk(E->mu);
    auto it = E->reqs.find(id);
    if (it == E->reqs.end() || it->second->state < 3)
      return serr(GSKNN_ERR_ARG, "gsknn_serve_release: unknown or unfinished request");
    if (it->second->heap_off >= 0) E->arena->release((size_t)it->second->heap_off,
                                                     it->second->heap_bytes);
    E->reqs.erase(it);
  }
  E->cv.notify_all();  // freed heap memory may admit queued requests
  return GSKNN_OK;
}

int gsknn_serve_pause(gsknn_serve_t *eng, int paused) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return serr(GSKNN_ERR_ARG, "gsknn_serve_pause: null engine");
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->paused = paused != 0;
  }
  E->cv.notify_all();
  return GSKNN_OK;
}

void gsknn_serve_destroy(gsknn_serve_t *eng) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->stop = true;
  }
  E->cv.notify_all();
  if (E->dispatcher.joinable()) E->dispatcher.join();
  for (auto &s : E->slots) {
    if (s.st) cudaStreamSynchronize(s.st);
    cudaFree(s.Xq); cudaFree(s.Xq2); cudaFree(s.Db); cudaFree(s.Ib); cudaFree(s.qidx);
    cudaFree(s.status); cudaFree(s.reqs_d); cudaFree(s.ws);
    if (s.h_q) cudaFreeHost(s.h_q);
    if (s.h_reqs) cudaFreeHost(s.h_reqs);
    if (s.st) cudaStreamDestroy(s.st);
  }
  cudaFree(E->cand_mem);
  cudaFree(E->cidx);
  cudaFree(E->status);
  cudaFree(E->arena_mem);
  delete E;
}

}  // extern "C"
