// knn_stream.cu -- the batching form with the point table and the heaps in host memory.
//
// For point sets beyond HBM (or a table memory-mapped from disk, gsknn_table.cpp): the points
// and the N x k heaps stay on the host, and each pass streams through a device staging table of
// `group_points` rows. A tree's leaves partition the points, so a tree is cut into groups of
// whole leaves that fit the staging table. For every group:
//   1. host threads gather its rows, norms and heap rows into pinned staging;
//   2. one copy each moves them to the device;
//   3. the batching pipeline (knn_batch.cu) runs on the staging table, its rows standing for the
//      group's global points, so lists and heaps carry global ids;
//   4. the updated heap rows come back and host threads scatter them into place.
// Groups of one tree touch disjoint points, so the gather of the next group and the scatter of
// the previous one overlap the device work of the current one (two pinned staging sets). Trees
// run one after another, so a point's heap sees the leaves of every tree. The result equals the
// resident job's after the same passes: the k nearest distinct leaf-mates per point, merged with
// the incoming heap.
#include "gsknn.h"
#include "knn_internal.h"

#include <algorithm>
#include <chrono>
#include <cstring>
#include <map>
#include <thread>
#include <vector>

namespace gsknn {

struct StreamJob {
  int N, d, k, ldD, P, leaf_min;
  long long max_rows;  // padded rows the staging job accepts
  const float *X, *X2;
  float *D;
  int *I;
  cudaStream_t st = nullptr;
  gsknn_batch_t *job = nullptr;
  void *dmem = nullptr;
  float *dX = nullptr, *dX2 = nullptr, *dD = nullptr;
  int *dI = nullptr;
  uint32_t *dgid = nullptr;
  struct Stage {
    void *mem = nullptr;
    float *X = nullptr, *X2 = nullptr, *D = nullptr;
    int *I = nullptr;
    uint32_t *gid = nullptr;
    std::vector<int> lptr, lpts, ltree;
    int n = 0;
  } stage[2];
  // last pass
  int groups = 0;
  double h2d = 0, d2h = 0, host_ms = 0;
};

static unsigned stream_threads() {
  unsigned nt = std::thread::hardware_concurrency();
  if (nt == 0) nt = 1;
  return nt > 32 ? 32 : nt;
}

// f(i) for i in [0, n) over the host threads (one thread for small n)
template <class F>
static void par_for(size_t n, size_t min_per_thread, F f) {
  unsigned nt = stream_threads();
  if (n < min_per_thread * 2) nt = 1;
  auto work = [&](unsigned w) {
    const size_t a = n * w / nt, b = n * (w + 1) / nt;
    for (size_t i = a; i < b; i++) f(i);
  };
  std::vector<std::thread> pool;
  for (unsigned w = 1; w < nt; w++) pool.emplace_back(work, w);
  work(0);
  for (auto &t : pool) t.join();
}

// Group g of a tree: leaves [l0, l1) of `order` (indices into the pass's leaf arrays).
static void gather_group(StreamJob *J, StreamJob::Stage &S, const std::vector<int> &order, int l0,
                         int l1, const int *leaf_ptr, const int *leaf_pts) {
  S.lptr.assign(1, 0);
  S.lpts.clear();
  S.ltree.clear();
  std::vector<int> G;
  for (int t = l0; t < l1; t++) {
    const int l = order[t];
    for (int e = leaf_ptr[l]; e < leaf_ptr[l + 1]; e++) {
      S.lpts.push_back((int)G.size());
      G.push_back(leaf_pts[e]);
    }
    S.lptr.push_back((int)G.size());
    S.ltree.push_back(0);
  }
  S.n = (int)G.size();
  const int d = J->d, k = J->k, ldD = J->ldD;
  par_for((size_t)S.n, 4096, [&](size_t i) {
    const size_t g = (size_t)G[i];
    std::memcpy(S.X + i * d, J->X + g * d, (size_t)d * 4);
    S.X2[i] = J->X2[g];
    std::memcpy(S.D + i * k, J->D + g * ldD, (size_t)k * 4);
    std::memcpy(S.I + i * k, J->I + g * ldD, (size_t)k * 4);
    S.gid[i] = (uint32_t)g;
  });
}

static void scatter_group(StreamJob *J, const StreamJob::Stage &S) {
  const int k = J->k, ldD = J->ldD;
  par_for((size_t)S.n, 4096, [&](size_t i) {
    const size_t g = (size_t)S.gid[i];
    std::memcpy(J->D + g * ldD, S.D + i * k, (size_t)k * 4);
    std::memcpy(J->I + g * ldD, S.I + i * k, (size_t)k * 4);
  });
}

// Copies in, the pass, copies out, on the job's stream (asynchronous).
static int enqueue_group(StreamJob *J, StreamJob::Stage &S) {
  const size_t n = (size_t)S.n, d = (size_t)J->d, k = (size_t)J->k;
  cudaError_t e = cudaMemcpyAsync(J->dX, S.X, n * d * 4, cudaMemcpyHostToDevice, J->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(J->dX2, S.X2, n * 4, cudaMemcpyHostToDevice, J->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(J->dD, S.D, n * k * 4, cudaMemcpyHostToDevice, J->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(J->dI, S.I, n * k * 4, cudaMemcpyHostToDevice, J->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(J->dgid, S.gid, n * 4, cudaMemcpyHostToDevice, J->st);
  if (e != cudaSuccess)
    return set_status(GSKNN_ERR_CUDA, "streaming form: copy failed: %s", cudaGetErrorString(e));
  const int rc = gsknn_batch_pass(J->job, S.lptr.data(), S.lpts.data(), S.ltree.data(),
                                  (int)S.ltree.size());
  if (rc != GSKNN_OK) return rc;
  e = cudaMemcpyAsync(S.D, J->dD, n * k * 4, cudaMemcpyDeviceToHost, J->st);
  if (e == cudaSuccess) e = cudaMemcpyAsync(S.I, J->dI, n * k * 4, cudaMemcpyDeviceToHost, J->st);
  if (e != cudaSuccess)
    return set_status(GSKNN_ERR_CUDA, "streaming form: copy failed: %s", cudaGetErrorString(e));
  J->h2d += (double)n * (d * 4 + 4 + 2 * k * 4 + 4);
  J->d2h += (double)n * 2 * k * 4;
  J->groups++;
  return GSKNN_OK;
}

static void free_stream(StreamJob *J) {
  if (J->st) cudaStreamSynchronize(J->st);
  if (J->job) gsknn_batch_destroy(J->job);
  for (auto &S : J->stage)
    if (S.mem) cudaFreeHost(S.mem);
  if (J->dmem) cudaFree(J->dmem);
  if (J->st) cudaStreamDestroy(J->st);
  delete J;
}

}  // namespace gsknn

using gsknn::StreamJob;

extern "C" {

gsknn_stream_t *gsknn_stream_create(int N, int d, int k, const float *X, const float *X2,
                                    float *D, int *I, int ldD, int group_points, int leaf_min,
                                    int shape) {
  using namespace gsknn;
  if (N <= 0 || d <= 0 || k <= 0 || ldD < k || group_points <= 0 || leaf_min <= 0 || !X ||
      !X2 || !D || !I) {
    set_status(GSKNN_ERR_ARG, "gsknn_stream_create: invalid sizes or null pointer");
    return nullptr;
  }
  if (shape >= 3) {  // the tensor-core batching shape works on table rows, not global ids
    set_status(GSKNN_ERR_UNSUPPORTED, "gsknn_stream_create: CUDA-core tile shapes only");
    return nullptr;
  }
  StreamJob *J = new StreamJob();
  J->N = N; J->d = d; J->k = k; J->ldD = ldD; J->leaf_min = leaf_min;
  J->P = std::min(group_points, N);
  J->X = X; J->X2 = X2; J->D = D; J->I = I;
  // the staging job's padded-row capacity (gsknn_batch_create: every leaf pads to whole tiles
  // of at most 128 rows)
  const long long leaves = ((long long)J->P + leaf_min - 1) / leaf_min;
  J->max_rows = (((long long)J->P + 128 * leaves) + 63) / 64 * 64;
  const size_t P = (size_t)J->P;
  size_t off = 0;
  auto take = [&](size_t n) { size_t o = off; off = (off + n + 255) & ~(size_t)255; return o; };
  const size_t oX = take(P * d * 4), oX2 = take(P * 4), oD = take(P * k * 4), oI = take(P * k * 4),
               oG = take(P * 4);
  bool ok = cudaStreamCreateWithFlags(&J->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaMalloc(&J->dmem, off) == cudaSuccess;
  if (ok) {
    char *b = static_cast<char *>(J->dmem);
    J->dX = reinterpret_cast<float *>(b + oX);
    J->dX2 = reinterpret_cast<float *>(b + oX2);
    J->dD = reinterpret_cast<float *>(b + oD);
    J->dI = reinterpret_cast<int *>(b + oI);
    J->dgid = reinterpret_cast<uint32_t *>(b + oG);
    for (auto &S : J->stage) {
      if (cudaHostAlloc(&S.mem, off, cudaHostAllocDefault) != cudaSuccess) {
        ok = false;
        break;
      }
      char *h = static_cast<char *>(S.mem);
      S.X = reinterpret_cast<float *>(h + oX);
      S.X2 = reinterpret_cast<float *>(h + oX2);
      S.D = reinterpret_cast<float *>(h + oD);
      S.I = reinterpret_cast<int *>(h + oI);
      S.gid = reinterpret_cast<uint32_t *>(h + oG);
    }
  }
  if (!ok) {
    cudaGetLastError();
    free_stream(J);
    set_status(GSKNN_ERR_NOMEM, "gsknn_stream_create: staging memory could not be allocated");
    return nullptr;
  }
  J->job = gsknn_batch_create(J->P, d, k, J->dX, J->dX2, J->dD, J->dI, k, 1, leaf_min, shape,
                              J->st);
  if (!J->job) {
    const int code = gsknn_last_error();
    free_stream(J);
    set_status(code ? code : GSKNN_ERR_CUDA, "gsknn_stream_create: staging job: %s",
               gsknn_last_error_string());
    return nullptr;
  }
  batch_set_global_ids(J->job, J->dgid);
  set_status(GSKNN_OK, nullptr);
  return reinterpret_cast<gsknn_stream_t *>(J);
}

int gsknn_stream_pass(gsknn_stream_t *job, const int *leaf_ptr, const int *leaf_pts,
                      const int *leaf_tree, int nleaves) {
  using namespace gsknn;
  StreamJob *J = reinterpret_cast<StreamJob *>(job);
  if (!J || !leaf_ptr || !leaf_pts || !leaf_tree || nleaves < 0)
    return set_status(GSKNN_ERR_ARG, "gsknn_stream_pass: invalid argument");
  if (nleaves == 0) return set_status(GSKNN_EARLY_RETURN, "gsknn_stream_pass: no leaves");
  // check the leaves and order them by tree (stable: each tree's leaves in the given order)
  std::map<int, std::vector<int>> trees;
  for (int l = 0; l < nleaves; l++) {
    const int L = leaf_ptr[l + 1] - leaf_ptr[l];
    if (L < 0) return set_status(GSKNN_ERR_ARG, "leaf_ptr must be non-decreasing");
    if (L > J->P)
      return set_status(GSKNN_ERR_UNSUPPORTED, "a leaf of %d points exceeds group_points %d", L,
                        J->P);
    if (leaf_tree[l] < 0) return set_status(GSKNN_ERR_ARG, "leaf_tree entries must be >= 0");
    for (int e = leaf_ptr[l]; e < leaf_ptr[l + 1]; e++)
      if (leaf_pts[e] < 0 || leaf_pts[e] >= J->N)
        return set_status(GSKNN_ERR_INDEX, "a leaf lists a point outside [0, N)");
    if (L > 0) trees[leaf_tree[l]].push_back(l);
  }
  J->groups = 0;
  J->h2d = J->d2h = 0;
  const auto t0 = std::chrono::steady_clock::now();
  for (auto &tr : trees) {
    const std::vector<int> &order = tr.second;
    // cut the tree into groups of whole leaves: points within the staging table and padded
    // rows within the staging job
    std::vector<std::pair<int, int>> groups;
    int a = 0;
    long long pts = 0, padded = 0;
    for (int t = 0; t < (int)order.size(); t++) {
      const int L = leaf_ptr[order[t] + 1] - leaf_ptr[order[t]];
      const long long pl = (L + 127) / 128 * 128;
      if (t > a && (pts + L > J->P || padded + pl > J->max_rows)) {
        groups.push_back({a, t});
        a = t;
        pts = padded = 0;
      }
      pts += L;
      padded += pl;
    }
    groups.push_back({a, (int)order.size()});
    // pipeline: gather group g + 1 while group g runs on the device
    int cur = 0;
    gather_group(J, J->stage[cur], order, groups[0].first, groups[0].second, leaf_ptr, leaf_pts);
    int rc = enqueue_group(J, J->stage[cur]);
    if (rc != GSKNN_OK) return rc;
    for (size_t g = 1; g < groups.size(); g++) {
      StreamJob::Stage &nx = J->stage[cur ^ 1];
      gather_group(J, nx, order, groups[g].first, groups[g].second, leaf_ptr, leaf_pts);
      if (cudaStreamSynchronize(J->st) != cudaSuccess)
        return set_status(GSKNN_ERR_CUDA, "streaming form: device work failed");
      // group g's heap rows have landed in its staging set: start group g + 1, then put them
      // in place while it runs
      rc = enqueue_group(J, nx);
      if (rc != GSKNN_OK) return rc;
      scatter_group(J, J->stage[cur]);
      cur ^= 1;
    }
    rc = gsknn_batch_sync(J->job);
    if (rc != GSKNN_OK) return rc;
    if (cudaStreamSynchronize(J->st) != cudaSuccess)
      return set_status(GSKNN_ERR_CUDA, "streaming form: device work failed");
    scatter_group(J, J->stage[cur]);
  }
  J->host_ms =
      std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  return set_status(GSKNN_OK, nullptr);
}

int gsknn_stream_info(const gsknn_stream_t *job, int *groups, double *h2d_bytes,
                      double *d2h_bytes, double *pass_ms) {
  const StreamJob *J = reinterpret_cast<const StreamJob *>(job);
  if (!J) return gsknn::set_status(GSKNN_ERR_ARG, "gsknn_stream_info: null job");
  if (groups) *groups = J->groups;
  if (h2d_bytes) *h2d_bytes = J->h2d;
  if (d2h_bytes) *d2h_bytes = J->d2h;
  if (pass_ms) *pass_ms = J->host_ms;
  return GSKNN_OK;
}

void gsknn_stream_destroy(gsknn_stream_t *job) {
  if (job) gsknn::free_stream(reinterpret_cast<StreamJob *>(job));
}

}  // extern "C"
