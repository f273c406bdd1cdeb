// knn_serve.cu -- the serving form: a request loop against a device-resident reference set.
//
// The reference has no serving path; a caller would run sgsknn once per request. Here:
//   * the reference set is prepared once (packed in the tensor-core format with its norms and
//     bound statistics, tc_cand_prepare) and stays resident;
//   * gsknn_serve_submit() queues a request (m query rows copied from the caller, a k);
//   * a dispatcher thread admits queued requests in arrival order while their result heaps fit
//     the heap arena (the HBM budget) and launches batches on free stream slots, so batches
//     formed from later arrivals run while earlier ones are still on the GPU (continuous
//     batching);
//   * a batch holds at most `slice` rows, sized so that one batch is a few milliseconds of
//     tensor work. The tensor-core kernel keeps one CTA on every SM for the whole batch, so a
//     small request launched behind a long batch would wait for all of it. Larger requests run
//     as row pieces over several batches, and whole requests that fit go first, so a small
//     arrival waits for at most about one slice. The oldest request too large to fit whole
//     still gets half of every batch, so it cannot starve;
//   * per batch: one host-to-device copy of the queries, their norms, the tensor-core pass with
//     the exact FP64 re-rank (tc_run_prepared) at the batch's largest k, and a scatter kernel
//     that writes each request's k smallest into its own heap, which stays on the device until
//     the caller releases the request;
//   * a completion thread watches one event per batch (recorded after the batch's last copy)
//     and marks its requests done. It polls every ~20 us while batches are in flight and
//     sleeps otherwise. Host functions queued on the stream (cudaLaunchHostFunc) were measured
//     to run up to 75 ms after the batch's last kernel had ended, a few times per 300 batches,
//     which set the whole latency tail.
// Results are the exact FP64 top-k of each query (ties to the lower id), so they are identical
// whatever a request was batched with.
#include "gsknn.h"
#include "knn_common.cuh"
#include "knn_internal.h"

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdio>
#include <cstdlib>
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

// GPU wall clock (ns) into *t, for the per-batch trace
__global__ void stamp(unsigned long long *t) {
  unsigned long long v;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(v));
  *t = v;
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
  int taken = 0;            // rows handed to batches so far
  int pending = 0;          // pieces launched and not finished
  bool failed = false;
  std::vector<float> q;     // the caller's query rows
  long long heap_off = -1;  // in the arena
  size_t heap_bytes = 0;
  float *D = nullptr;
  int *I = nullptr;
  int state = 0;            // 0 queued, 1 admitted, 2 all rows launched, 3 done, 4 failed
  int batch = -1, batch_rows = 0;
  Clock::time_point t_submit, t_launch, t_done;
};

struct Piece {             // rows [row0, row0 + rows) of a request, inside one batch
  std::shared_ptr<Request> r;
  int row0, rows;
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
  std::vector<Piece> batch;
  int batch_id = -1, batch_rows = 0, batch_k = 0;
  Clock::time_point t_formed, t_launched;  // for GSKNN_SERVE_TRACE
  cudaEvent_t done_ev = nullptr;           // recorded behind the batch's status copy
  bool inflight = false;                   // launched; the completion thread owns it
  gsknn::Engine *eng = nullptr;
  int index = 0;
};

}  // namespace serve

struct Engine {
  int device;
  int nref, d, mode, max_q, max_k, kp_max, sms, nslots;
  int slice = 0;  // rows per batch
  size_t heap_budget;
  TcCand C{};
  void *cand_mem = nullptr;
  void *ecand_mem = nullptr;  // the resident set's panels in the escalation format
  // The resident set as batches use it: C itself, or (when the engine measured the escalation
  // format faster) C's escalation panels run as the main format.
  TcCand Crun{};
  double probe_ms[2] = {0.0, 0.0};  // AUTO: probe batch in BF16 (+escalation) and split BF16
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
  std::thread completer;
  std::condition_variable ccv;  // completion thread: a batch was launched
  bool trace = false;  // GSKNN_SERVE_TRACE=1: one stderr line per batch
  serve::Clock::time_point t0 = serve::Clock::now();
};

}  // namespace gsknn

using gsknn::Engine;
namespace gs = gsknn::serve;

static int serr(int code, const char *msg) { return gsknn::set_status(code, "%s", msg); }

// A piece of r finished (ok or not), called with the lock held: the request is done once all
// its rows were launched and every piece has finished.
static void piece_finished(gs::Request &r, bool ok, gs::Clock::time_point now) {
  r.pending--;
  if (!ok) r.failed = true;
  if (r.taken == r.m && r.pending == 0) {
    r.t_done = now;
    r.state = r.failed ? 4 : 3;
  }
}

// The batch of slot s has finished on the GPU: finish its pieces and free the slot.
static void batch_done(gs::Slot *s) {
  Engine *E = s->eng;
  const auto now = gs::Clock::now();
  {
    std::lock_guard<std::mutex> lk(E->mu);
    s->inflight = false;
    int st = 0;
    std::memcpy(&st, s->h_reqs + E->max_q, sizeof(int));  // status copied back by the batch
    for (auto &pc : s->batch) piece_finished(*pc.r, st == 0, now);
    if (E->trace) {
      using ms = std::chrono::duration<double, std::milli>;
      unsigned long long g[4];
      std::memcpy(g, reinterpret_cast<const char *>(s->h_reqs + E->max_q) + 8, sizeof(g));
      std::fprintf(stderr,
                   "gsknn serve: slot %d batch %d pieces %zu rows %d k %d formed %.3f "
                   "launched %.3f done %.3f ms | gpu start %.3f prep %.3f tc %.3f scatter %.3f "
                   "ms\n",
                   s->index, s->batch_id, s->batch.size(), s->batch_rows, s->batch_k,
                   ms(s->t_formed - E->t0).count(), ms(s->t_launched - E->t0).count(),
                   ms(now - E->t0).count(), (double)(g[0] % 1000000000000ull) * 1e-6,
                   (double)(g[1] - g[0]) * 1e-6, (double)(g[2] - g[1]) * 1e-6,
                   (double)(g[3] - g[2]) * 1e-6);
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
  const int npc = (int)s.batch.size();
  for (int i = 0; i < npc; i++) {
    const gs::Piece &pc = s.batch[i];
    const gs::Request &r = *pc.r;
    std::memcpy(s.h_q + (size_t)rows * E->d, r.q.data() + (size_t)pc.row0 * E->d,
                (size_t)pc.rows * E->d * 4);
    s.h_reqs[i] = {rows, pc.rows, r.k, 0, r.D + (size_t)pc.row0 * r.k,
                   r.I + (size_t)pc.row0 * r.k};
    rows += pc.rows;
    kb = std::max(kb, r.k);
  }
  const TcPlan P = tc_plan(rows, E->nref, E->d, kb, E->mode, E->sms, false, E->sms);
  if (!P.ok || P.bytes > E->ws_bytes) return cudaErrorInvalidValue;
  cudaStream_t st = s.st;
  cudaError_t e = cudaMemcpyAsync(s.Xq, s.h_q, (size_t)rows * E->d * 4, cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.reqs_d, s.h_reqs, (size_t)npc * sizeof(gs::ReqDesc),
                        cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(s.status, 0, sizeof(int), st);
  if (e != cudaSuccess) return e;
  unsigned long long *stamps = reinterpret_cast<unsigned long long *>(s.status) + 1;
  if (E->trace) gs::stamp<<<1, 1, 0, st>>>(stamps + 0);
  gs::query_norms<<<(rows + 7) / 8, 256, 0, st>>>(s.Xq, E->d, rows, s.Xq2);
  const long long n = (long long)rows * kb;
  gs::fill_heap<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(s.Db, s.Ib, n);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  if (E->trace) gs::stamp<<<1, 1, 0, st>>>(stamps + 1);
  e = tc_run_prepared(P, E->Crun, rows, E->d, kb, s.Xq, s.Xq2, E->max_q, s.qidx, s.Db, s.Ib, kb,
                      s.ws, s.status, nullptr, 0, nullptr, st, nullptr, nullptr);
  if (e != cudaSuccess) return e;
  dim3 blk(32, 8);
  if (E->trace) gs::stamp<<<1, 1, 0, st>>>(stamps + 2);
  gs::scatter<<<(rows + 7) / 8, blk, 0, st>>>(s.Db, s.Ib, kb, s.reqs_d, npc, rows);
  if (E->trace) gs::stamp<<<1, 1, 0, st>>>(stamps + 3);
  e = cudaGetLastError();
  // the status word (and, when tracing, the four stamps after it) to the slot's host area
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(s.h_reqs + E->max_q, s.status, E->trace ? 40 : sizeof(int),
                        cudaMemcpyDeviceToHost, st);
  s.t_launched = gs::Clock::now();
  if (e == cudaSuccess) e = cudaEventRecord(s.done_ev, st);
  return e;
}

// Fill slot s with the next batch (lock held; the front of the queue is admitted). Whole
// requests go first-fit in arrival order; if the oldest request is too large to fit whole, half
// the slice is held for it and it gets a piece of at least that size.
static void form_batch(Engine *E, gs::Slot &s) {
  const int cap = E->slice, bid = E->next_batch++;
  const auto now = gs::Clock::now();
  auto front = E->queue.front();
  const int reserve = front->m - front->taken > cap ? cap / 2 : 0;
  int rows = 0;
  auto take = [&](const std::shared_ptr<gs::Request> &r, int n) {
    if (r->taken == 0) {
      r->batch = bid;
      r->t_launch = now;
    }
    s.batch.push_back({r, r->taken, n});
    r->taken += n;
    r->pending++;
    rows += n;
  };
  for (auto &r : E->queue) {
    if (r->state != 1) break;  // admission is a prefix of the queue
    const int rem = r->m - r->taken;
    if (rem <= cap - reserve - rows) take(r, rem);
  }
  if (front->taken < front->m && rows < cap) take(front, std::min(front->m - front->taken, cap - rows));
  for (auto &pc : s.batch)
    if (pc.r->taken == pc.r->m) pc.r->state = 2;
  for (auto &pc : s.batch)
    if (pc.r->batch == bid && pc.row0 == 0) pc.r->batch_rows = rows;
  s.batch_id = bid;
  s.batch_rows = rows;
  s.batch_k = 0;
  for (auto &pc : s.batch) s.batch_k = std::max(s.batch_k, pc.r->k);
  s.t_formed = now;
  E->queue.erase(std::remove_if(E->queue.begin(), E->queue.end(),
                                [](const std::shared_ptr<gs::Request> &r) { return r->state == 2; }),
                 E->queue.end());
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
    form_batch(E, *slot);
    slot->busy = true;
    lk.unlock();
    cudaSetDevice(dev);
    const cudaError_t e = launch_batch(E, *slot);
    if (e == cudaSuccess) {
      {
        std::lock_guard<std::mutex> g(E->mu);
        slot->inflight = true;
      }
      E->ccv.notify_one();
    } else {
      std::lock_guard<std::mutex> g(E->mu);
      E->error = GSKNN_ERR_CUDA;
      std::snprintf(E->errmsg, sizeof(E->errmsg), "serving batch launch failed: %s",
                    cudaGetErrorString(e));
      const auto now = gs::Clock::now();
      for (auto &pc : slot->batch) {
        gs::Request &r = *pc.r;
        if (r.taken < r.m) {  // no further pieces of a failed request
          r.taken = r.m;
          E->queue.erase(std::remove(E->queue.begin(), E->queue.end(), pc.r), E->queue.end());
        }
        piece_finished(r, false, now);
      }
      slot->batch.clear();
      slot->busy = false;
      E->done_cv.notify_all();
    }
  }
}

// Completion thread: polls the events of in-flight batches (cudaEventQuery) every ~20 us while
// there are any, sleeps on ccv otherwise.
static void completion_loop(Engine *E) {
  cudaSetDevice(E->device);
  std::vector<gs::Slot *> live;
  while (true) {
    {
      std::unique_lock<std::mutex> lk(E->mu);
      E->ccv.wait(lk, [&] {
        if (E->stop) return true;
        for (auto &s : E->slots)
          if (s.inflight) return true;
        return false;
      });
      if (E->stop) return;
      live.clear();
      for (auto &s : E->slots)
        if (s.inflight) live.push_back(&s);
    }
    bool any = false;
    for (gs::Slot *s : live) {
      const cudaError_t q = cudaEventQuery(s->done_ev);
      if (q == cudaErrorNotReady) continue;
      if (q != cudaSuccess) {  // a failed batch: its status word is not trustworthy
        std::lock_guard<std::mutex> g(E->mu);
        E->error = GSKNN_ERR_CUDA;
        std::snprintf(E->errmsg, sizeof(E->errmsg), "serving batch failed: %s",
                      cudaGetErrorString(q));
        int bad = GSKNN_ERR_CUDA;
        std::memcpy(s->h_reqs + E->max_q, &bad, sizeof(int));
      }
      batch_done(s);
      any = true;
    }
    if (!any) std::this_thread::sleep_for(std::chrono::microseconds(20));
  }
}

// Rows per batch that keep one batch near 3 ms of tensor work on one B200: the exact forms
// measured about 1.5e12 evals/s at d = 64 and 8.6e11 at d = 128, i.e. about 3e11 eval-dims per
// 3 ms. Whole query tiles (128 rows), at least one, at most max_batch_queries.
// The resident set's escalation panels as a main-format candidate set of their own.
static gsknn::TcCand escalation_as_main(const gsknn::TcCand &C, int esc_mode) {
  gsknn::TcCand S = C;
  const gsknn::TcPlan P = gsknn::tc_plan(128, C.nc, C.d, 1, esc_mode, 148, false, 148);
  S.fmt = C.efmt;
  S.elem = C.efmt == 0 ? 4 : 2;
  S.d_pad = P.d_pad;
  S.pb = C.epb;
  S.pb_lo = C.epb_lo;
  S.pn = C.epn;
  S.efmt = -1;
  S.epb = S.epb_lo = S.epn = nullptr;
  return S;
}

// Times one probe batch (the first min(max_q, 1024) resident points as queries, k = max_k) in
// the prepared mode with escalation and in the escalation mode alone; keeps the faster (second
// of two runs each, on slot 0's buffers). Returns false when a probe call fails.
static bool probe_modes(Engine *E, int esc) {
  using namespace gsknn;
  gs::Slot &s = E->slots[0];
  const int rows = std::min(E->max_q, 1024), kb = E->max_k;
  const TcCand Cesc = escalation_as_main(E->C, esc);
  const int modes[2] = {E->mode, esc};
  const TcCand *cands[2] = {&E->C, &Cesc};
  cudaEvent_t a = nullptr, b = nullptr;
  if (cudaEventCreate(&a) != cudaSuccess || cudaEventCreate(&b) != cudaSuccess) return false;
  bool ok = cudaMemsetAsync(s.status, 0, sizeof(int), s.st) == cudaSuccess;
  for (int m = 0; m < 2 && ok; m++) {
    const TcPlan P = tc_plan(rows, E->nref, E->d, kb, modes[m], E->sms, false, E->sms);
    if (!P.ok || P.bytes > E->ws_bytes) {
      E->probe_ms[m] = 1e30;
      continue;
    }
    float ms = 0.f;
    for (int rep = 0; rep < 2 && ok; rep++) {
      const long long n = (long long)rows * kb;
      gs::fill_heap<<<(unsigned)((n + 255) / 256), 256, 0, s.st>>>(s.Db, s.Ib, n);
      ok = cudaEventRecord(a, s.st) == cudaSuccess &&
           tc_run_prepared(P, *cands[m], rows, E->d, kb, E->C.Xc, E->C.Xc2, E->nref, s.qidx,
                           s.Db, s.Ib, kb, s.ws, s.status, nullptr, 0, nullptr, s.st, nullptr,
                           nullptr) == cudaSuccess &&
           cudaEventRecord(b, s.st) == cudaSuccess &&
           cudaEventSynchronize(b) == cudaSuccess && cudaEventElapsedTime(&ms, a, b) ==
                                                        cudaSuccess;
    }
    E->probe_ms[m] = ms;
  }
  int st = 0;
  if (ok) ok = cudaMemcpy(&st, s.status, 4, cudaMemcpyDeviceToHost) == cudaSuccess && st == 0;
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ok && E->probe_ms[1] < E->probe_ms[0]) {
    E->mode = esc;
    E->Crun = Cesc;
  }
  return ok;
}

static int auto_slice(const Engine *E) {
  const double rows = 3.0e11 / ((double)E->nref * (double)E->d);
  int s = (int)(rows / 128.0) * 128;
  return std::min(E->max_q, std::max(128, s));
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
  // AUTO prepares the resident set in BF16 with split-BF16 escalation panels (queries whose
  // BF16 band overflows finish in split BF16), then measures a probe batch both ways -- BF16
  // with escalation, and split BF16 alone on the escalation panels -- and serves with the
  // faster. Where split tiles do not fit, TF32.
  const bool auto_mode = mode == GSKNN_MODE_AUTO;
  if (auto_mode)
    mode = tc_plan(max_batch_queries, nref, d, max_k, GSKNN_TC_BF16X3, 148, false, 148).ok
               ? GSKNN_MODE_BF16
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
  // query-side workspace: the largest plan over batch sizes (whole query tiles) and k, in the
  // prepared mode and (AUTO) in the escalation mode run alone
  const int esc = tc_escalation_mode(E->max_q, nref, d, max_k, mode, E->sms);
  for (int kk = 1; kk <= max_k; kk++)
    for (int q = 128; q < E->max_q + 128; q += 128) {
      const TcPlan P = tc_plan(std::min(q, E->max_q), nref, d, kk, mode, E->sms, false, E->sms);
      if (!P.ok) {
        serr(GSKNN_ERR_UNSUPPORTED, "gsknn_serve_create: d or k outside the tensor-core form");
        return nullptr;
      }
      E->ws_bytes = std::max(E->ws_bytes, P.bytes);
      if (auto_mode && esc) {
        const TcPlan P2 = tc_plan(std::min(q, E->max_q), nref, d, kk, esc, E->sms, false, E->sms);
        if (P2.ok) E->ws_bytes = std::max(E->ws_bytes, P2.bytes);
      }
    }
  const size_t cb = tc_cand_bytes(nref, d, mode);
  // queries whose band log overflows in this format run again in a narrower one: its panels of
  // the resident set are prepared once, beside the first
  bool ok = (!esc || cudaMalloc(&E->ecand_mem, tc_cand_panel_bytes(nref, d, esc)) ==
                         cudaSuccess) &&
            cudaMalloc(&E->cand_mem, cb) == cudaSuccess &&
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
  if (e == cudaSuccess && esc)
    e = tc_cand_prepare_escalation(&E->C, E->ecand_mem, esc, E->status, st0);
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
         cudaMalloc((void **)&s.status, 64) == cudaSuccess &&
         cudaMalloc((void **)&s.reqs_d, (q + 1) * sizeof(gs::ReqDesc)) == cudaSuccess &&
         cudaMalloc(&s.ws, E->ws_bytes) == cudaSuccess &&
         cudaHostAlloc((void **)&s.h_q, q * d * 4, cudaHostAllocDefault) == cudaSuccess &&
         cudaHostAlloc((void **)&s.h_reqs, (q + 2) * sizeof(gs::ReqDesc),
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
  E->Crun = E->C;
  if (auto_mode && esc && !probe_modes(E.get(), esc)) {
    serr(GSKNN_ERR_CUDA, "gsknn_serve_create: the probe batch failed");
    gsknn_serve_destroy(reinterpret_cast<gsknn_serve_t *>(E.release()));
    return nullptr;
  }
  E->slice = auto_slice(E.get());
  E->trace = std::getenv("GSKNN_SERVE_TRACE") != nullptr;
  for (auto &sl : E->slots)
    if (cudaEventCreateWithFlags(&sl.done_ev, cudaEventDisableTiming) != cudaSuccess) {
      serr(GSKNN_ERR_CUDA, "gsknn_serve_create: event creation failed");
      gsknn_serve_destroy(reinterpret_cast<gsknn_serve_t *>(E.release()));
      return nullptr;
    }
  Engine *raw = E.release();
  raw->completer = std::thread(completion_loop, raw);
  raw->dispatcher = std::thread(dispatcher_loop, raw);
  set_status(GSKNN_OK, nullptr);
  return reinterpret_cast<gsknn_serve_t *>(raw);
}

int gsknn_serve_mode(gsknn_serve_t *eng, double *probe_bf16_ms, double *probe_bf16x3_ms) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return -GSKNN_ERR_ARG;
  if (probe_bf16_ms) *probe_bf16_ms = E->probe_ms[0];
  if (probe_bf16x3_ms) *probe_bf16x3_ms = E->probe_ms[1];
  return E->mode;
}

long long gsknn_serve_submit(gsknn_serve_t *eng, const float *Q, int m, int k) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E || !Q || m <= 0 || k <= 0) return serr(GSKNN_ERR_ARG, "gsknn_serve_submit: bad args") * -1LL;
  if (k > E->max_k) return -1LL * serr(GSKNN_ERR_UNSUPPORTED, "gsknn_serve_submit: k above max_k");
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

int gsknn_serve_set_slice(gsknn_serve_t *eng, int rows) {
  Engine *E = reinterpret_cast<Engine *>(eng);
  if (!E) return -serr(GSKNN_ERR_ARG, "gsknn_serve_set_slice: null engine");
  int s;
  {
    std::lock_guard<std::mutex> lk(E->mu);
    E->slice = rows <= 0 ? auto_slice(E) : std::min(E->max_q, (rows + 127) / 128 * 128);
    s = E->slice;
  }
  gsknn::set_status(GSKNN_OK, nullptr);
  return s;
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
  E->ccv.notify_all();
  if (E->dispatcher.joinable()) E->dispatcher.join();
  if (E->completer.joinable()) E->completer.join();
  for (auto &s : E->slots) {
    if (s.st) cudaStreamSynchronize(s.st);
    if (s.done_ev) cudaEventDestroy(s.done_ev);
    cudaFree(s.Xq); cudaFree(s.Xq2); cudaFree(s.Db); cudaFree(s.Ib); cudaFree(s.qidx);
    cudaFree(s.status); cudaFree(s.reqs_d); cudaFree(s.ws);
    if (s.h_q) cudaFreeHost(s.h_q);
    if (s.h_reqs) cudaFreeHost(s.h_reqs);
    if (s.st) cudaStreamDestroy(s.st);
  }
  cudaFree(E->cand_mem);
  cudaFree(E->ecand_mem);
  cudaFree(E->cidx);
  cudaFree(E->status);
  cudaFree(E->arena_mem);
  delete E;
}

}  // extern "C"
