// gsknn_api.cu -- the C ABI of libgsknn.so (declared in include/gsknn.h).
//
// Host-pointer entry points (the reference API) copy the referenced row range of each point
// table, the index lists and the heap rows to the GPU, run the device pipeline, copy D/I back
// and return when done. Device-pointer entry points (gsknn_*_device) enqueue the same pipeline
// on a caller stream. Scratch memory comes from a cache keyed by (device, stream, slot).
#include "gsknn.h"
#include "knn_internal.h"

#include <algorithm>
#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <type_traits>
#include <thread>
#include <vector>

#if defined(__x86_64__)
#include <emmintrin.h>
#endif

namespace gsknn {

// ------------------------------------------------------------------------------------------
// status
// ------------------------------------------------------------------------------------------
static thread_local int t_status = 0;
static thread_local char t_msg[512] = "ok";

int set_status(int code, const char *fmt, ...) {
  t_status = code;
  if (fmt) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_msg, sizeof(t_msg), fmt, ap);
    va_end(ap);
  } else {
    snprintf(t_msg, sizeof(t_msg), "%s", code == 0 ? "ok" : "error");
  }
  return code;
}

#define CU(call)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess)                                                                \
      return set_status(e_ == cudaErrorMemoryAllocation ? GSKNN_ERR_NOMEM : GSKNN_ERR_CUDA, \
                        "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__,  \
                        __LINE__);                                                        \
  } while (0)

// ------------------------------------------------------------------------------------------
// scratch cache
// ------------------------------------------------------------------------------------------
enum Slot { SLOT_KERNEL = 0, SLOT_STATUS, SLOT_HQTAB, SLOT_HCTAB, SLOT_HQNRM, SLOT_HCNRM,
            SLOT_HQIDX, SLOT_HCIDX, SLOT_HD, SLOT_HI, SLOT_AUX, SLOT_HGATHER };

struct Buf {
  void *p = nullptr;
  size_t n = 0;
};
static std::mutex g_mu;
static std::map<std::tuple<int, uintptr_t, int>, Buf> g_bufs;

static cudaError_t scratch(int slot, size_t bytes, cudaStream_t st, void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(g_mu);
  Buf &b = g_bufs[std::make_tuple(dev, (uintptr_t)st, slot)];
  if (b.n < bytes) {
    if (b.p) {
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) return e;
      cudaFree(b.p);
      b.p = nullptr;
      b.n = 0;
    }
    size_t nb = std::max(bytes, (size_t)4096);
    e = cudaMalloc(&b.p, nb);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return e;
    }
    b.n = nb;
  }
  *out = b.p;
  return cudaSuccess;
}

static void release_all_for_device(int dev) {
  std::lock_guard<std::mutex> lk(g_mu);
  for (auto it = g_bufs.begin(); it != g_bufs.end();) {
    if (std::get<0>(it->first) == dev) {
      cudaStreamSynchronize((cudaStream_t)std::get<1>(it->first));
      cudaFree(it->second.p);
      it = g_bufs.erase(it);
    } else {
      ++it;
    }
  }
}

// ------------------------------------------------------------------------------------------
// launch tracing: CUDA events around every kernel launch of the library, on its stream
// ------------------------------------------------------------------------------------------
struct TraceRec {
  const char *name;
  cudaEvent_t a, b;
  int nk;  // kernels of the library launched between a and b
};
static std::mutex g_tmu;
static bool g_trace = false;
static std::vector<TraceRec> g_recs;
static std::vector<cudaEvent_t> g_evpool;

static cudaEvent_t ev_get() {
  if (!g_evpool.empty()) {
    cudaEvent_t e = g_evpool.back();
    g_evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

struct TraceScope {
  const char *name;
  cudaStream_t st;
  int nk;
  cudaEvent_t a = nullptr;
  TraceScope(const char *n, cudaStream_t s, int kernels = 1) : name(n), st(s), nk(kernels) {
    if (!g_trace) return;
    std::lock_guard<std::mutex> lk(g_tmu);
    a = ev_get();
    cudaEventRecord(a, st);
  }
  ~TraceScope() {
    if (!a) return;
    std::lock_guard<std::mutex> lk(g_tmu);
    cudaEvent_t b = ev_get();
    cudaEventRecord(b, st);
    g_recs.push_back({name, a, b, nk});
  }
};

// Pinned host staging of the calling thread (the gathered rows of a host call), kept between
// calls and freed when the thread exits.
struct PinnedStage {
  void *p = nullptr;
  size_t n = 0;
  ~PinnedStage() {
    if (p) cudaFreeHost(p);
  }
};
static thread_local PinnedStage t_stage;

static cudaError_t pinned_stage(size_t bytes, void **out) {
  if (t_stage.n < bytes) {
    if (t_stage.p) cudaFreeHost(t_stage.p);
    t_stage.p = nullptr;
    t_stage.n = 0;
    cudaError_t e = cudaHostAlloc(&t_stage.p, bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
      (void)cudaGetLastError();
      return e;
    }
    t_stage.n = bytes;
  }
  *out = t_stage.p;
  return cudaSuccess;
}

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

// Host threads of the host-pointer path: one per hardware thread, at most 32.
static unsigned host_threads() {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  return nt > 32 ? 32 : nt;
}

// memcpy of `bytes` split over the host threads (one thread below 4 MiB).
static void par_copy(void *dst, const void *src, size_t bytes) {
  unsigned nt = host_threads();
  if (bytes < ((size_t)4 << 20)) nt = 1;
  auto work = [&](unsigned w) {
    const size_t a = bytes * w / nt, b = bytes * (w + 1) / nt;
    std::memcpy(static_cast<char *>(dst) + a, static_cast<const char *>(src) + a, b - a);
  };
  std::vector<std::thread> pool;
  for (unsigned w = 1; w < nt; w++) pool.emplace_back(work, w);
  work(0);
  for (auto &t : pool) t.join();
}

// Rows qidx[0..nq) of Xq, then cidx[0..nc) of Xc, and their norms, gathered by the host threads
// into pinned hrows / hn and copied to drows / dn on stream st. The rows go in chunks: every
// thread gathers its part of chunk j, and the calling thread enqueues chunk j's copy as soon as
// all parts are in, so the copies overlap the gathering of the next chunks. Returns the first
// copy error.
template <typename T>
static cudaError_t gather_rows_to_device(const T *Xq, const T *Xq2, const int *qidx, int nq,
                                         const T *Xc, const T *Xc2, const int *cidx, int nc,
                                         int d, T *hrows, T *hn, T *drows, T *dn,
                                         cudaStream_t st) {
  const size_t n = (size_t)nq + nc, row_bytes = (size_t)d * sizeof(T);
  const bool big = n * row_bytes >= ((size_t)8 << 20);
  const unsigned nt = big ? host_threads() : 1;
  const int nch = n * row_bytes >= ((size_t)32 << 20) ? 8 : 1;
  std::unique_ptr<std::atomic<unsigned>[]> done(new std::atomic<unsigned>[nch]);
  for (int j = 0; j < nch; j++) done[j].store(0);
#if defined(__x86_64__)
  // The staging rows are written once and then read only by the DMA engine: non-temporal
  // stores skip the read-for-ownership of every destination line (a third of the host memory
  // traffic of this copy). Used when rows and the staging base are 16-byte aligned.
  const bool stream = row_bytes % 16 == 0 && (reinterpret_cast<uintptr_t>(hrows) & 15) == 0;
#endif
  auto part = [&](unsigned w, int j) {
    const size_t c0 = n * j / nch, c1 = n * (j + 1) / nch;
    const size_t a = c0 + (c1 - c0) * w / nt, b = c0 + (c1 - c0) * (w + 1) / nt;
    for (size_t i = a; i < b; i++) {
      const bool q = i < (size_t)nq;
      const size_t r = q ? (size_t)qidx[i] : (size_t)cidx[i - nq];
      const T *src = (q ? Xq : Xc) + r * d;
#if defined(__x86_64__)
      if (stream) {
        const __m128i *s4 = reinterpret_cast<const __m128i *>(src);
        __m128i *d4 = reinterpret_cast<__m128i *>(hrows + i * d);
        for (size_t v = 0; v < row_bytes / 16; v++)
          _mm_stream_si128(d4 + v, _mm_loadu_si128(s4 + v));
      } else {
        std::memcpy(hrows + i * d, src, row_bytes);
      }
#else
      std::memcpy(hrows + i * d, src, row_bytes);
#endif
      hn[i] = (q ? Xq2 : Xc2)[r];
    }
#if defined(__x86_64__)
    _mm_sfence();  // the streamed rows are visible before the chunk is handed to the DMA
#endif
    done[j].fetch_add(1, std::memory_order_release);
  };
  std::vector<std::thread> pool;
  for (unsigned w = 1; w < nt; w++)
    pool.emplace_back([&, w] {
      for (int j = 0; j < nch; j++) part(w, j);
    });
  cudaError_t err = cudaSuccess;
  for (int j = 0; j < nch; j++) {
    part(0, j);
    while (done[j].load(std::memory_order_acquire) < nt) std::this_thread::yield();
    const size_t c0 = n * j / nch, c1 = n * (j + 1) / nch;
    if (err == cudaSuccess)
      err = cudaMemcpyAsync(drows + c0 * d, hrows + c0 * d, (c1 - c0) * row_bytes,
                            cudaMemcpyHostToDevice, st);
  }
  for (auto &t : pool) t.join();
  if (err == cudaSuccess) err = cudaMemcpyAsync(dn, hn, n * sizeof(T), cudaMemcpyHostToDevice, st);
  return err;
}

// table[(idx[i] - lo)] = rows[i] (and the norms), one warp per row
template <typename T>
__global__ void scatter_rows(const T *__restrict__ rows, const T *__restrict__ rows2,
                             const int *__restrict__ idx, int n, int d, int lo, T *__restrict__ tab,
                             T *__restrict__ tab2) {
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= n) return;
  const size_t r = (size_t)(idx[i] - lo);
  for (int p = lane; p < d; p += 32) tab[r * d + p] = rows[(size_t)i * d + p];
  if (lane == 0) tab2[r] = rows2[i];
}

static cudaStream_t host_stream() {
  static thread_local std::map<int, cudaStream_t> streams;
  int dev = 0;
  cudaGetDevice(&dev);
  auto it = streams.find(dev);
  if (it != streams.end()) return it->second;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) s = nullptr;
  streams[dev] = s;
  return s;
}

static int sm_count() {
  int dev = 0, n = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
  return n > 0 ? n : 148;
}

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

// Number of candidate splits per query tile: balances the waves of CTAs over the SMs.
static int choose_splits(int qtiles, int rtiles, int slots) {
  int best_s = 1;
  double best = 1e300;
  const int smax = std::min(rtiles, 64);
  for (int s = 1; s <= smax; s++) {
    const long long items = (long long)qtiles * s;
    const double waves = (double)((items + slots - 1) / slots);
    const double cost = waves / s * (1.0 + 0.004 * s);  // small per-split merge cost
    if (cost < best - 1e-12) {
      best = cost;
      best_s = s;
    }
  }
  return best_s;
}

// Tracer hook for pipelines that bracket groups of launches themselves (the tensor-core path).
static void trace_hook(void *, const char *name, bool begin, cudaStream_t st, int nkernels) {
  if (!g_trace) return;
  std::lock_guard<std::mutex> lk(g_tmu);
  static thread_local std::vector<std::pair<const char *, cudaEvent_t>> pending;
  if (begin) {
    cudaEvent_t a = ev_get();
    cudaEventRecord(a, st);
    pending.push_back({name, a});
    return;
  }
  for (size_t i = pending.size(); i-- > 0;) {
    if (std::strcmp(pending[i].first, name) == 0) {
      cudaEvent_t b = ev_get();
      cudaEventRecord(b, st);
      g_recs.push_back({name, pending[i].second, b, nkernels});
      pending.erase(pending.begin() + (long)i);
      return;
    }
  }
}

// ------------------------------------------------------------------------------------------
// device pipeline: pack -> fused select -> finalize (queries = heap rows)
// ------------------------------------------------------------------------------------------
template <typename T>
int knn_device_simt(int nq, int nc, int d, int k, const T *Xq, const T *Xq2, long long nrows_q,
                    const int *qidx, const T *Xc, const T *Xc2, long long nrows_c,
                    const int *cidx, T *D, int *I, int ldD, cudaStream_t st, int metric = 0) {
  if (nq == 0 || nc == 0 || d == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, d or k is 0");
  if (nq < 0 || nc < 0 || d < 0 || k < 0 || ldD < k)
    return set_status(GSKNN_ERR_ARG, "invalid sizes (n=%d m=%d d=%d k=%d ldD=%d)", nq, nc, d,
                      k, ldD);
  // the 1-norm reads no norms
  if (!Xq || !qidx || !Xc || !cidx || !D || !I || (metric == 0 && (!Xq2 || !Xc2)))
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  if (metric) Xq2 = Xc2 = nullptr;
  const SimtGeom g = simt_geometry<T>(k);
  if (g.kp == 0)
    return set_status(GSKNN_ERR_UNSUPPORTED, "k=%d exceeds the fused kernel's list size", k);

  const int nkc = (d + g.dk - 1) / g.dk;
  const int qtiles = (nq + g.bq - 1) / g.bq;
  const int rtiles = (nc + g.br - 1) / g.br;
  const int S = choose_splits(qtiles, rtiles, sm_count() * std::max(1, g.minb));
  const int tps = (rtiles + S - 1) / S;

  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
  const size_t oA = take((size_t)qtiles * nkc * g.dk * g.bq * sizeof(T));
  const size_t oB = take((size_t)rtiles * nkc * g.dk * g.br * sizeof(T));
  const size_t oQN = take((size_t)qtiles * g.bq * sizeof(T));
  const size_t oCN = take((size_t)rtiles * g.br * sizeof(T));
  const size_t oCI = take((size_t)rtiles * g.br * 4);
  const size_t oPD = take((size_t)S * nq * k * sizeof(T));
  const size_t oPI = take((size_t)S * nq * k * 4);
  void *ws = nullptr, *stv = nullptr;
  CU(scratch(SLOT_KERNEL, off, st, &ws));
  CU(scratch(SLOT_STATUS, 256, st, &stv));
  char *base = static_cast<char *>(ws);
  int *status = static_cast<int *>(stv);
  CU(cudaMemsetAsync(status, 0, sizeof(int), st));

  T *Apack = reinterpret_cast<T *>(base + oA);
  T *Bpack = reinterpret_cast<T *>(base + oB);
  T *qn = reinterpret_cast<T *>(base + oQN);
  T *cn = reinterpret_cast<T *>(base + oCN);
  uint32_t *cid = reinterpret_cast<uint32_t *>(base + oCI);
  T *partD = reinterpret_cast<T *>(base + oPD);
  uint32_t *partI = reinterpret_cast<uint32_t *>(base + oPI);

  {
    TraceScope ts("pack_panels", st);
    CU(launch_pack<T>(Xq, Xq2, d, nrows_q, qidx, nq, g.bq, g.dk, nkc, Apack, qn, nullptr,
                      status, st));
  }
  {
    TraceScope ts("pack_panels", st);
    CU(launch_pack<T>(Xc, Xc2, d, nrows_c, cidx, nc, g.br, g.dk, nkc, Bpack, cn, cid, status,
                      st));
  }
  SimtArgs<T> sa{};
  sa.Apack = Apack; sa.Bpack = Bpack; sa.qn = qn; sa.cn = cn; sa.cid = cid;
  sa.Din = D; sa.ldD = ldD; sa.Q = nq; sa.k = k; sa.nkc = nkc;
  sa.ntiles_r = rtiles; sa.tiles_per_split = tps; sa.partD = partD; sa.partI = partI;
  sa.metric = metric;
  {
    TraceScope ts("fused_knn_simt", st);
    CU(launch_simt<T>(sa, g.kp, qtiles, S, st));
  }
  FinalizeArgs<T> fa{};
  fa.Din = D; fa.Iin = I; fa.ldD = ldD; fa.Q = nq; fa.k = k; fa.S = S;
  fa.partD = partD; fa.partI = partI; fa.Dout = D; fa.Iout = I;
  {
    TraceScope ts("finalize_heap", st);
    CU(launch_finalize<T>(fa, g.kp, st));
  }
  return set_status(GSKNN_OK, nullptr);
}

static int g_mode = GSKNN_MODE_AUTO;

// Tensor-core approximate pass + FP64 re-rank (float inputs). `dbg`, when set, also receives
// the approximate distance of every (query, candidate) pair (row stride dbg_ld) and `margin`
// the per-query band width 2E.
static int knn_device_tc(int mode, int nq, int nc, int d, int k, const float *Xq,
                         const float *Xq2, long long nrows_q, const int *qidx, const float *Xc,
                         const float *Xc2, long long nrows_c, const int *cidx, float *D, int *I,
                         int ldD, cudaStream_t st, float *dbg = nullptr, long long dbg_ld = 0,
                         float *margin = nullptr) {
  if (nq == 0 || nc == 0 || d == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, d or k is 0");
  if (nq < 0 || nc < 0 || d < 0 || k < 0 || ldD < k)
    return set_status(GSKNN_ERR_ARG, "invalid sizes (n=%d m=%d d=%d k=%d ldD=%d)", nq, nc, d,
                      k, ldD);
  if (!Xq || !Xq2 || !qidx || !Xc || !Xc2 || !cidx || !D || !I)
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  const TcPlan P = tc_plan(nq, nc, d, k, mode, sm_count());
  if (!P.ok)
    return set_status(GSKNN_ERR_UNSUPPORTED,
                      "tensor-core mode %d does not support d=%d k=%d (shared memory)", mode, d,
                      k);
  void *ws = nullptr, *stv = nullptr;
  CU(scratch(SLOT_KERNEL, P.bytes, st, &ws));
  CU(scratch(SLOT_STATUS, 256, st, &stv));
  int *status = static_cast<int *>(stv);
  CU(cudaMemsetAsync(status, 0, sizeof(int), st));
  // GSKNN_TC_COUNTERS=1: per-call diagnostics of the tensor-core epilogue on stderr
  static const bool want_counters = std::getenv("GSKNN_TC_COUNTERS") != nullptr;
  unsigned long long *counters = nullptr;
  if (want_counters) {
    void *cv = nullptr;
    CU(scratch(SLOT_AUX, 128, st, &cv));
    counters = static_cast<unsigned long long *>(cv);
    CU(cudaMemsetAsync(counters, 0, 128, st));
  }
  CU(tc_run(P, nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx, D, I, ldD, ws,
            status, dbg, dbg_ld, counters, st, trace_hook, nullptr));
  if (counters) {
    unsigned long long h[16] = {};
    int nfb = 0;
    CU(cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, st));
    CU(cudaMemcpyAsync(&nfb, static_cast<char *>(ws) + P.o_fbc, sizeof(int),
                       cudaMemcpyDeviceToHost, st));
    CU(cudaStreamSynchronize(st));
    const double ctas = (double)P.qtiles * P.S, warps = ctas * TC_EPI_WARPS;
    std::fprintf(stderr,
                 "gsknn tc: mode=%d n=%d m=%d d=%d k=%d S=%d N=%d NST=%d: logged/query=%.1f "
                 "inserts/query=%.1f loop-iters/warp=%.1f slow-chunks/warp=%.1f "
                 "chunks/warp=%.1f rerank-scanned/query=%.1f exact/query=%.1f fallback=%d | "
                 "cycles/CTA: mma-loop=%.0f mma-wait-tma=%.0f mma-wait-epilogue=%.0f | "
                 "cycles/warp: epi-loop=%.0f epi-wait-mma=%.0f\n",
                 mode, nq, nc, d, k, P.S, P.N, P.NST, (double)h[0] / nq, (double)h[1] / nq,
                 (double)h[2] / warps, (double)h[3] / warps, (double)h[4] / warps,
                 (double)h[5] / nq, (double)h[6] / nq, nfb, (double)h[10] / ctas,
                 (double)h[7] / ctas, (double)h[8] / ctas, (double)h[11] / warps,
                 (double)h[9] / warps);
  }
  if (margin)
    CU(cudaMemcpyAsync(margin, static_cast<char *>(ws) + P.o_margin, (size_t)nq * 4,
                       cudaMemcpyDeviceToDevice, st));
  return set_status(GSKNN_OK, nullptr);
}

// The arithmetic used for a float call: explicit modes are honoured; AUTO takes the
// tensor-core form with the exact FP64 re-rank where it fits (split BF16 below d = 128, BF16
// from there, TF32 where neither fits), else the CUDA-core FP32 kernel.
static int pick_mode(int nq, int nc, int d, int k) {
  if (g_mode != GSKNN_MODE_AUTO) return g_mode;
  // Split BF16 keeps the re-rank band narrowest (input error ~u^2): at d = 64 plain BF16's band
  // overflows the logs and most queries run again. From d = 128 one BF16 MMA per product was
  // measured fastest (d = 256: 10.8 ms against 13.9 ms in split BF16 for 32,768 x 262,144,
  // k = 64); the few queries whose log overflows run again in split BF16.
  if (d >= 128 && tc_plan(nq, nc, d, k, GSKNN_TC_BF16, sm_count()).ok) return GSKNN_TC_BF16;
  if (tc_plan(nq, nc, d, k, GSKNN_TC_BF16X3, sm_count()).ok) return GSKNN_TC_BF16X3;
  if (tc_plan(nq, nc, d, k, GSKNN_TC_TF32, sm_count()).ok) return GSKNN_TC_TF32;
  return GSKNN_MODE_FP32;
}

template <typename T>
int knn_device_large(int nq, int nc, int d, int k, const T *Xq, const T *Xq2, long long nrows_q,
                     const int *qidx, const T *Xc, const T *Xc2, long long nrows_c,
                     const int *cidx, T *D, int *I, int ldD, int four_ary, cudaStream_t st,
                     int metric = 0) {
  if (nq == 0 || nc == 0 || d == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, d or k is 0");
  const int need = four_ary ? k + KNN_HEAP_OFFSET : k;
  if (nq < 0 || nc < 0 || d < 0 || k < 0 || ldD < need)
    return set_status(GSKNN_ERR_ARG, "invalid sizes (n=%d m=%d d=%d k=%d ldD=%d)", nq, nc, d,
                      k, ldD);
  if (!Xq || !qidx || !Xc || !cidx || !D || !I || (metric == 0 && (!Xq2 || !Xc2)))
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  if (large_select_smem(k, sizeof(T)) > 227 * 1024)
    return set_status(GSKNN_ERR_UNSUPPORTED, "k=%d exceeds the selection kernel (k <= %d)", k,
                      sizeof(T) == 8 ? 16384 : 16384);
  const LargePlan P = large_plan<T>(nq, nc, d, k, (size_t)1 << 30);
  void *ws = nullptr, *stv = nullptr;
  CU(scratch(SLOT_KERNEL, P.bytes, st, &ws));
  CU(scratch(SLOT_STATUS, 256, st, &stv));
  int *status = static_cast<int *>(stv);
  CU(cudaMemsetAsync(status, 0, sizeof(int), st));
  {
    // two packing launches, then a distance block and a selection per chunk of query rows
    TraceScope ts("select_rows", st, 2 + 2 * ((nq + P.chunk_rows - 1) / P.chunk_rows));
    CU(large_run<T>(P, nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx, D, I, ldD,
                    four_ary, ws, status, st, metric));
  }
  return set_status(GSKNN_OK, nullptr);
}

template <typename T>
int knn_device(int nq, int nc, int d, int k, const T *Xq, const T *Xq2, long long nrows_q,
               const int *qidx, const T *Xc, const T *Xc2, long long nrows_c, const int *cidx,
               T *D, int *I, int ldD, cudaStream_t st, int metric = 0) {
  if (metric != 0) {  // the 1-norm: CUDA cores only (it is no inner product)
    if (simt_geometry<T>(k).kp == 0)
      return knn_device_large<T>(nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx,
                                 D, I, ldD, 0, st, metric);
    return knn_device_simt<T>(nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx, D,
                              I, ldD, st, metric);
  }
  if constexpr (std::is_same<T, float>::value) {
    const int mode = pick_mode(nq, nc, d, k);
    if (mode != GSKNN_MODE_FP32)
      return knn_device_tc(mode, nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx,
                           D, I, ldD, st);
  }
  // lists beyond the fused kernels' capacity: explicit distance block + row selection
  if (simt_geometry<T>(k).kp == 0)
    return knn_device_large<T>(nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx, D,
                               I, ldD, 0, st);
  return knn_device_simt<T>(nq, nc, d, k, Xq, Xq2, nrows_q, qidx, Xc, Xc2, nrows_c, cidx, D, I,
                            ldD, st);
}

// Reads back the device status word of `st` (after synchronising it).
static int device_status(cudaStream_t st) {
  void *stv = nullptr;
  CU(scratch(SLOT_STATUS, 256, st, &stv));
  CU(cudaStreamSynchronize(st));
  int h = 0;
  CU(cudaMemcpy(&h, stv, sizeof(int), cudaMemcpyDeviceToHost));
  if (h == GSKNN_ERR_INDEX)
    return set_status(GSKNN_ERR_INDEX, "an alpha/beta index lies outside its point table");
  if (h == GSKNN_ERR_TIMEOUT)
    return set_status(GSKNN_ERR_TIMEOUT, "a bounded device-side wait gave up");
  if (h != 0) return set_status(h, "device-side error %d", h);
  return GSKNN_OK;
}

// ------------------------------------------------------------------------------------------
// host-pointer path
// ------------------------------------------------------------------------------------------
static bool index_range(const int *idx, int n, int *lo, int *hi) {
  int a = idx[0], b = idx[0];
  for (int i = 1; i < n; i++) {
    const int v = idx[i];
    a = v < a ? v : a;
    b = v > b ? v : b;
  }
  *lo = a;
  *hi = b;
  return a >= 0;
}

template <typename T>
// path: 0 = the default dispatch, 1 = explicit distance block + selection into binary heaps,
// 2 = the same into 4-ary heaps with the 3-slot header (rows of ldD >= k + 3).
// metric: 0 = squared 2-norm, 1 = 1-norm (heap_t.type KNN_1NORM).
int knn_host(int nq, int nc, int d, int k, const T *Xq, const T *Xq2, const int *qidx,
             const T *Xc, const T *Xc2, const int *cidx, T *D, int *I, int ldD, int path = 0,
             int metric = 0) {
  if (nq == 0 || nc == 0 || d == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, d or k is 0");
  if (nq < 0 || nc < 0 || d < 0 || k < 0 || ldD < (path == 2 ? k + KNN_HEAP_OFFSET : k))
    return set_status(GSKNN_ERR_ARG, "invalid sizes");
  if (!Xq || !Xq2 || !qidx || !Xc || !Xc2 || !cidx || !D || !I)
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  // GSKNN_HOST_TRACE=1: one stderr line per call with the host-side phases in milliseconds
  static const bool host_trace = std::getenv("GSKNN_HOST_TRACE") != nullptr;
  using hclock = std::chrono::steady_clock;
  const auto h0 = hclock::now();
  auto hms = [&](hclock::time_point t) {
    return std::chrono::duration<double, std::milli>(t - h0).count();
  };
  hclock::time_point h_gather = h0, h_copy = h0, h_enq = h0, h_done = h0;
  int qlo, qhi, clo, chi;
  if (!index_range(qidx, nq, &qlo, &qhi) || !index_range(cidx, nc, &clo, &chi))
    return set_status(GSKNN_ERR_INDEX, "negative point index");
  cudaStream_t st = host_stream();
  const bool same = (Xq == Xc) && (Xq2 == Xc2);
  if (same) {
    qlo = clo = std::min(qlo, clo);
    qhi = chi = std::max(qhi, chi);
  }
  void *pqi, *pci, *pD, *pI;
  CU(scratch(SLOT_HQIDX, (size_t)nq * 4, st, &pqi));
  CU(scratch(SLOT_HCIDX, (size_t)nc * 4, st, &pci));
  CU(scratch(SLOT_HD, (size_t)nq * ldD * sizeof(T), st, &pD));
  CU(scratch(SLOT_HI, (size_t)nq * ldD * 4, st, &pI));
  CU(cudaMemcpyAsync(pqi, qidx, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pci, cidx, (size_t)nc * 4, cudaMemcpyHostToDevice, st));
  // Device copy of each table over the row range the index lists reach, so that global row ids
  // index it directly. When the lists reference well under that range (random subsets of a
  // large table), only the referenced rows travel: gathered on the host into pinned staging,
  // one copy, then scattered into place on the device. Otherwise the range is copied as is.
  const size_t qrows = (size_t)(qhi - qlo + 1), crows = (size_t)(chi - clo + 1);
  const size_t range_rows = same ? qrows : qrows + crows;
  const bool sparse = (size_t)(nq + nc) * 10 < range_rows * 6;
  void *pqt = nullptr, *pqn = nullptr, *pct = nullptr, *pcn = nullptr;
  CU(scratch(SLOT_HQTAB, qrows * d * sizeof(T), st, &pqt));
  CU(scratch(SLOT_HQNRM, qrows * sizeof(T), st, &pqn));
  if (!same) {
    CU(scratch(SLOT_HCTAB, crows * d * sizeof(T), st, &pct));
    CU(scratch(SLOT_HCNRM, crows * sizeof(T), st, &pcn));
  } else {
    pct = pqt;
    pcn = pqn;
  }
  // Pinned staging of this call: the heaps first (both directions go through it, so their
  // copies run at DMA speed), then, on the sparse path, the gathered rows and their norms. The
  // heaps' copy to the device overlaps the gathering of the rows.
  const size_t n = (size_t)nq + nc;
  const size_t hd_bytes = (size_t)nq * ldD * sizeof(T), hi_bytes = (size_t)nq * ldD * 4;
  const size_t rows_off = al256(al256(hd_bytes) + hi_bytes);
  const size_t bytes = rows_off + (sparse ? n * d * sizeof(T) + n * sizeof(T) : 0);
  void *stage = nullptr;
  CU(cudaStreamSynchronize(st));  // the staging buffer of the previous call is free
  CU(pinned_stage(bytes, &stage));
  T *hD = static_cast<T *>(stage);
  int *hI = reinterpret_cast<int *>(static_cast<char *>(stage) + al256(hd_bytes));
  par_copy(hD, D, hd_bytes);
  par_copy(hI, I, hi_bytes);
  CU(cudaMemcpyAsync(pD, hD, hd_bytes, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pI, hI, hi_bytes, cudaMemcpyHostToDevice, st));
  if (sparse) {
    void *dg = nullptr;
    CU(scratch(SLOT_HGATHER, n * d * sizeof(T) + n * sizeof(T), st, &dg));
    T *hrows = reinterpret_cast<T *>(static_cast<char *>(stage) + rows_off);
    T *hn = hrows + n * d;
    T *grows = static_cast<T *>(dg);
    T *gn = grows + n * d;
    CU(gather_rows_to_device<T>(Xq, Xq2, qidx, nq, Xc, Xc2, cidx, nc, d, hrows, hn, grows, gn,
                                st));
    h_gather = hclock::now();
    scatter_rows<T><<<(nq + 7) / 8, 256, 0, st>>>(grows, gn, static_cast<const int *>(pqi), nq,
                                                  d, qlo, static_cast<T *>(pqt),
                                                  static_cast<T *>(pqn));
    scatter_rows<T><<<(nc + 7) / 8, 256, 0, st>>>(grows + (size_t)nq * d, gn + nq,
                                                  static_cast<const int *>(pci), nc, d, clo,
                                                  static_cast<T *>(pct), static_cast<T *>(pcn));
    CU(cudaGetLastError());
  } else {
    CU(cudaMemcpyAsync(pqt, Xq + (size_t)qlo * d, qrows * d * sizeof(T), cudaMemcpyHostToDevice,
                       st));
    CU(cudaMemcpyAsync(pqn, Xq2 + qlo, qrows * sizeof(T), cudaMemcpyHostToDevice, st));
    if (!same) {
      CU(cudaMemcpyAsync(pct, Xc + (size_t)clo * d, crows * d * sizeof(T),
                         cudaMemcpyHostToDevice, st));
      CU(cudaMemcpyAsync(pcn, Xc2 + clo, crows * sizeof(T), cudaMemcpyHostToDevice, st));
    }
  }
  const T *dXq = static_cast<const T *>(pqt) - (size_t)qlo * d;
  const T *dXq2 = static_cast<const T *>(pqn) - qlo;
  const T *dXc = static_cast<const T *>(pct) - (size_t)clo * d;
  const T *dXc2 = static_cast<const T *>(pcn) - clo;
  int rc = GSKNN_OK;
  h_copy = hclock::now();
  if (path == 0)
    rc = knn_device<T>(nq, nc, d, k, dXq, dXq2, (long long)qhi + 1, static_cast<int *>(pqi),
                       dXc, dXc2, (long long)chi + 1, static_cast<int *>(pci),
                       static_cast<T *>(pD), static_cast<int *>(pI), ldD, st, metric);
  else
    rc = knn_device_large<T>(nq, nc, d, k, dXq, dXq2, (long long)qhi + 1,
                             static_cast<int *>(pqi), dXc, dXc2, (long long)chi + 1,
                             static_cast<int *>(pci), static_cast<T *>(pD),
                             static_cast<int *>(pI), ldD, path == 2 ? 1 : 0, st, metric);
  if (rc != GSKNN_OK) {
    cudaStreamSynchronize(st);
    return rc;
  }
  h_enq = hclock::now();
  rc = device_status(st);
  if (rc != GSKNN_OK) return rc;
  h_done = hclock::now();
  CU(cudaMemcpyAsync(hD, pD, hd_bytes, cudaMemcpyDeviceToHost, st));
  CU(cudaMemcpyAsync(hI, pI, hi_bytes, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  par_copy(D, hD, hd_bytes);
  par_copy(I, hI, hi_bytes);
  if (host_trace)
    std::fprintf(stderr,
                 "gsknn host: n=%d m=%d sparse=%d gather %.3f copies-enqueued %.3f "
                 "kernels-enqueued %.3f device-done %.3f heaps-back %.3f ms\n",
                 nq, nc, sparse ? 1 : 0, hms(h_gather), hms(h_copy), hms(h_enq), hms(h_done),
                 hms(hclock::now()));
  return set_status(GSKNN_OK, nullptr);
}

// Distance block of host tables: C[j*ldc + i] for rows j < nq (qidx) and columns i < nc (cidx).
template <typename T>
int sq2nrm_host(int nq, int nc, int d, const T *Xq, const T *Xq2, const int *qidx, const T *Xc,
                const T *Xc2, const int *cidx, T *C, int ldc) {
  if (nq == 0 || nc == 0 || d == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n or k is 0");
  if (nq < 0 || nc < 0 || d < 0 || ldc < nc)
    return set_status(GSKNN_ERR_ARG, "invalid sizes (ldc must be >= m)");
  if (!Xq || !Xq2 || !qidx || !Xc || !Xc2 || !cidx || !C)
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  int qlo, qhi, clo, chi;
  if (!index_range(qidx, nq, &qlo, &qhi) || !index_range(cidx, nc, &clo, &chi))
    return set_status(GSKNN_ERR_INDEX, "negative point index");
  cudaStream_t st = host_stream();
  const size_t qrows = (size_t)(qhi - qlo + 1), crows = (size_t)(chi - clo + 1);
  void *pq, *pq2, *pc, *pc2, *pqi, *pci, *pC, *stv, *ws;
  CU(scratch(SLOT_HQTAB, qrows * d * sizeof(T), st, &pq));
  CU(scratch(SLOT_HQNRM, qrows * sizeof(T), st, &pq2));
  CU(scratch(SLOT_HCTAB, crows * d * sizeof(T), st, &pc));
  CU(scratch(SLOT_HCNRM, crows * sizeof(T), st, &pc2));
  CU(scratch(SLOT_HQIDX, (size_t)nq * 4, st, &pqi));
  CU(scratch(SLOT_HCIDX, (size_t)nc * 4, st, &pci));
  CU(scratch(SLOT_HD, (size_t)nq * nc * sizeof(T), st, &pC));
  CU(scratch(SLOT_STATUS, 256, st, &stv));
  CU(cudaMemcpyAsync(pq, Xq + (size_t)qlo * d, qrows * d * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pq2, Xq2 + qlo, qrows * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pc, Xc + (size_t)clo * d, crows * d * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pc2, Xc2 + clo, crows * sizeof(T), cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pqi, qidx, (size_t)nq * 4, cudaMemcpyHostToDevice, st));
  CU(cudaMemcpyAsync(pci, cidx, (size_t)nc * 4, cudaMemcpyHostToDevice, st));
  int *status = static_cast<int *>(stv);
  CU(cudaMemsetAsync(status, 0, sizeof(int), st));
  const LargePlan P = large_plan<T>(nq, nc, d, 1, 0);
  CU(scratch(SLOT_KERNEL, P.bytes, st, &ws));
  {
    TraceScope ts("dist_block", st, 3);  // two packing launches and the distance block
    CU(block_run<T>(P, nq, nc, d, static_cast<const T *>(pq) - (size_t)qlo * d,
                    static_cast<const T *>(pq2) - qlo, (long long)qhi + 1,
                    static_cast<const int *>(pqi), static_cast<const T *>(pc) - (size_t)clo * d,
                    static_cast<const T *>(pc2) - clo, (long long)chi + 1,
                    static_cast<const int *>(pci), static_cast<T *>(pC), nc, ws, status, st));
  }
  int rc = device_status(st);
  if (rc != GSKNN_OK) return rc;
  CU(cudaMemcpy2DAsync(C, (size_t)ldc * sizeof(T), pC, (size_t)nc * sizeof(T),
                       (size_t)nc * sizeof(T), (size_t)nq, cudaMemcpyDeviceToHost, st));
  CU(cudaStreamSynchronize(st));
  return set_status(GSKNN_OK, nullptr);
}

}  // namespace gsknn

using namespace gsknn;

// ==========================================================================================
// C ABI
// ==========================================================================================
extern "C" {

int gsknn_last_error(void) { return t_status; }
const char *gsknn_last_error_string(void) { return t_msg; }

int gsknn_set_mode(int mode) {
  if (mode < GSKNN_MODE_AUTO || mode > GSKNN_MODE_BF16X3)
    return set_status(GSKNN_ERR_ARG, "unknown mode %d", mode);
  g_mode = mode;
  return set_status(GSKNN_OK, nullptr);
}
int gsknn_get_mode(void) { return g_mode; }

int gsknn_s_device(int m, int n, int d, int k, const float *XA, const float *XA2, long long nA,
                   const int *alpha, const float *XB, const float *XB2, long long nB,
                   const int *beta, float *D, int *I, int ldD, void *stream) {
  return knn_device<float>(n, m, d, k, XB, XB2, nB, beta, XA, XA2, nA, alpha, D, I, ldD,
                           (cudaStream_t)stream);
}

int gsknn_d_device(int m, int n, int d, int k, const double *XA, const double *XA2,
                   long long nA, const int *alpha, const double *XB, const double *XB2,
                   long long nB, const int *beta, double *D, int *I, int ldD, void *stream) {
  return knn_device<double>(n, m, d, k, XB, XB2, nB, beta, XA, XA2, nA, alpha, D, I, ldD,
                            (cudaStream_t)stream);
}

int gsknn_s_device_metric(int type, int m, int n, int d, int k, const float *XA,
                          const float *XA2, long long nA, const int *alpha, const float *XB,
                          const float *XB2, long long nB, const int *beta, float *D, int *I,
                          int ldD, void *stream) {
  if (type != KNN_2NORM && type != KNN_1NORM)
    return set_status(GSKNN_ERR_ARG, "type must be KNN_2NORM or KNN_1NORM");
  return knn_device<float>(n, m, d, k, XB, XB2, nB, beta, XA, XA2, nA, alpha, D, I, ldD,
                           (cudaStream_t)stream, type == KNN_1NORM ? 1 : 0);
}

int gsknn_d_device_metric(int type, int m, int n, int d, int k, const double *XA,
                          const double *XA2, long long nA, const int *alpha, const double *XB,
                          const double *XB2, long long nB, const int *beta, double *D, int *I,
                          int ldD, void *stream) {
  if (type != KNN_2NORM && type != KNN_1NORM)
    return set_status(GSKNN_ERR_ARG, "type must be KNN_2NORM or KNN_1NORM");
  return knn_device<double>(n, m, d, k, XB, XB2, nB, beta, XA, XA2, nA, alpha, D, I, ldD,
                            (cudaStream_t)stream, type == KNN_1NORM ? 1 : 0);
}

int gsknn_stream_status(void *stream) { return device_status((cudaStream_t)stream); }

int gsknn_tc_distances(int mode, int m, int n, int d, int k, const float *XA, const float *XA2,
                       long long nA, const int *alpha, const float *XB, const float *XB2,
                       long long nB, const int *beta, float *D, int *I, int ldD, float *C,
                       long long ldc, float *margin, void *stream) {
  if (mode != GSKNN_MODE_TF32 && mode != GSKNN_MODE_BF16 && mode != GSKNN_MODE_BF16X3)
    return set_status(GSKNN_ERR_ARG, "gsknn_tc_distances: mode must be a tensor-core mode");
  if (C && ldc < m) return set_status(GSKNN_ERR_ARG, "gsknn_tc_distances: ldc < m");
  return knn_device_tc(mode, n, m, d, k, XB, XB2, nB, beta, XA, XA2, nA, alpha, D, I, ldD,
                       (cudaStream_t)stream, C, ldc, margin);
}

void gsknn_trace_enable(int on) {
  std::lock_guard<std::mutex> lk(g_tmu);
  g_trace = on != 0;
}

int gsknn_trace_read(char *buf, int len) {
  std::lock_guard<std::mutex> lk(g_tmu);
  struct Acc { int n = 0; double ms = 0.0; };
  std::map<std::string, Acc> acc;
  int total = 0;
  for (auto &r : g_recs) {
    cudaEventSynchronize(r.b);
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, r.a, r.b) == cudaSuccess) {
      Acc &x = acc[r.name];
      x.n += r.nk;
      x.ms += ms;
    }
    g_evpool.push_back(r.a);
    g_evpool.push_back(r.b);
    total++;
  }
  g_recs.clear();
  std::string out = "{";
  bool first = true;
  for (auto &kv : acc) {
    char tmp[256];
    snprintf(tmp, sizeof(tmp), "%s\"%s\": {\"launches\": %d, \"ms\": %.6f}", first ? "" : ", ",
             kv.first.c_str(), kv.second.n, kv.second.ms);
    out += tmp;
    first = false;
  }
  out += "}";
  if (buf && len > 0) snprintf(buf, (size_t)len, "%s", out.c_str());
  return total;
}

void gsknn_release_workspace(void) {
  int dev = 0;
  cudaGetDevice(&dev);
  release_all_for_device(dev);
}

// ---- reference entry points (frame/gsknn.c) ----
void sgsknn_var1(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                 float *XB2, int *beta, float *D, int *I) {
  knn_host<float>(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, D, I, r);
}

void dgsknn_var1(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
                 double *XB2, int *beta, double *D, int *I) {
  knn_host<double>(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, D, I, r);
}

void sgsknn(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
            float *XB2, int *beta, heap_t *heap) {
  if (!heap) {
    set_status(GSKNN_ERR_ARG, "null heap");
    return;
  }
  knn_host<float>(n, m, k, r, XB, XB2, beta, XA, XA2, alpha, heap->D_s, heap->I, heap->ldk, 0,
                  heap->type == KNN_1NORM ? 1 : 0);
}

void dgsknn(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
            double *XB2, int *beta, heap_t *heap) {
  if (!heap) {
    set_status(GSKNN_ERR_ARG, "null heap");
    return;
  }
  if (r > KNN_VAR_THRES) {
    dgsknn_var3(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, heap);
    return;
  }
  knn_host<double>(n, m, k, r, XB, XB2, beta, XA, XA2, alpha, heap->D, heap->I, heap->ldk, 0,
                   heap->type == KNN_1NORM ? 1 : 0);
}

// frame/gsknn.c:597-659. The heap's own layout decides the selection: 4-ary with the header
// when heapCreate_d built it that way (heap->d == 4), binary otherwise (attached heaps).
void dgsknn_var3(int m, int n, int k, int r, double *XA, double *XA2, int *amap, double *XB,
                 double *XB2, int *bmap, heap_t *heap) {
  if (!heap) {
    set_status(GSKNN_ERR_ARG, "null heap");
    return;
  }
  knn_host<double>(n, m, k, r, XB, XB2, bmap, XA, XA2, amap, heap->D, heap->I, heap->ldk,
                   heap->d == 4 ? 2 : 1, heap->type == KNN_1NORM ? 1 : 0);
}

void dgssq2nrm(int m, int n, int k, double *XA, double *XA2, int *amap, double *XB,
               double *XB2, int *bmap, double *C, int ldc) {
  sq2nrm_host<double>(n, m, k, XB, XB2, bmap, XA, XA2, amap, C, ldc);
}

// frame/gsknn_ref.c:63-162: D/I are n rows of r (binary heaps), candidates on the alpha side.
void sgsknn_ref(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                float *XB2, int *beta, float *D, int *I) {
  if (r == 0) {
    set_status(GSKNN_EARLY_RETURN, "early return: r is 0");
    return;
  }
  knn_host<float>(n, m, k, r, XB, XB2, beta, XA, XA2, alpha, D, I, r, 1);
}

void dgsknn_ref(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
                double *XB2, int *beta, double *D, int *I) {
  if (r == 0) {
    set_status(GSKNN_EARLY_RETURN, "early return: r is 0");
    return;
  }
  knn_host<double>(n, m, k, r, XB, XB2, beta, XA, XA2, alpha, D, I, r, 1);
}

// frame/gsknn_ref_stl.cpp:81-214: the same reference algorithm with an STL heap per row.
void sgsknn_ref_stl(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                    float *XB2, int *beta, float *D, int *I) {
  sgsknn_ref(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, D, I);
}

void dgsknn_ref_stl(int m, int n, int k, int r, double *XA, double *XA2, int *alpha,
                    double *XB, double *XB2, int *beta, double *D, int *I) {
  dgsknn_ref(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, D, I);
}

}  // extern "C"
