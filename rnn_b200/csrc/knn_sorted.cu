// knn_sorted.cu -- the sorted-output adapters around the fused kNN.
//
// The reference's tree code consumes kNN results as ascending (distance, id) lists:
// dgsrnn_directKQuery (frame/old/dgsrnn_directKQuery.cpp:14-135) runs the fused kNN of m queries
// against n references on identity maps with its own norms and pops every heap row into an
// ascending std::pair<double, long> list; dgsrnn_directKQuery_var2 (same file, 141-222) takes
// the caller's maps and norms and copies the heap rows out as they are. Pairs are not C ABI, so
// here the lists are two arrays (distances, 64-bit ids). A device row sort turns heap rows that
// stay on the GPU into the same ascending lists.
#include "gsknn.h"
#include "knn_common.cuh"
#include "knn_internal.h"

#include <algorithm>
#include <limits>
#include <thread>
#include <vector>

namespace gsknn {

// One warp per row: the row's k entries sorted ascending by (distance, id as unsigned) in place,
// so -1 padding sorts last among equal distances; E*32 >= k.
template <typename T, int E>
__global__ void __launch_bounds__(256) sort_rows(T *__restrict__ D, int *__restrict__ I, int n,
                                                 int k, int ldk) {
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (q >= n) return;
  T d[E];
  uint32_t id[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    d[e] = t < k ? D[(size_t)q * ldk + t] : Num<T>::inf();
    id[e] = t < k ? (uint32_t)I[(size_t)q * ldk + t] : NO_ID;
  }
  warp_sort<T, E>(d, id, lane);
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (t < k) {
      D[(size_t)q * ldk + t] = d[e];
      I[(size_t)q * ldk + t] = (int)id[e];
    }
  }
}

template <typename T>
static cudaError_t launch_sort_rows(T *D, int *I, int n, int k, int ldk, cudaStream_t st) {
  const int blocks = (n + 7) / 8;
  if (k <= 32) sort_rows<T, 1><<<blocks, 256, 0, st>>>(D, I, n, k, ldk);
  else if (k <= 64) sort_rows<T, 2><<<blocks, 256, 0, st>>>(D, I, n, k, ldk);
  else if (k <= 128) sort_rows<T, 4><<<blocks, 256, 0, st>>>(D, I, n, k, ldk);
  else if (k <= 256) sort_rows<T, 8><<<blocks, 256, 0, st>>>(D, I, n, k, ldk);
  else sort_rows<T, 16><<<blocks, 256, 0, st>>>(D, I, n, k, ldk);
  return cudaGetLastError();
}

template <typename T>
static int heap_sort_device(T *D, int *I, int n, int k, int ldk, void *stream) {
  if (n == 0 || k == 0) return set_status(GSKNN_EARLY_RETURN, "early return: n or k is 0");
  if (n < 0 || k < 0 || ldk < k || !D || !I)
    return set_status(GSKNN_ERR_ARG, "invalid sizes or null pointer");
  if (k > 512) return set_status(GSKNN_ERR_UNSUPPORTED, "row sort supports k <= 512, got %d", k);
  const cudaError_t e = launch_sort_rows<T>(D, I, n, k, ldk, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return set_status(GSKNN_ERR_CUDA, "row sort launch failed: %s", cudaGetErrorString(e));
  return set_status(GSKNN_OK, nullptr);
}

// Squared 2-norms of the rows of a row-major table, accumulated in double as the adapter does
// (dgsrnn_directKQuery.cpp:60-79), over the host's cores.
template <typename T>
static void row_norms(const T *X, long rows, long dim, T *out) {
  const long per = 1L << 14;
  const int nt = (int)std::max(1L, std::min<long>((rows + per - 1) / per,
                                                  (long)std::thread::hardware_concurrency()));
  auto work = [&](int t) {
    const long lo = rows * t / nt, hi = rows * (t + 1) / nt;
    for (long i = lo; i < hi; i++) {
      double s = 0.0;
      for (long p = 0; p < dim; p++) s += (double)X[i * dim + p] * (double)X[i * dim + p];
      out[i] = (T)s;
    }
  };
  std::vector<std::thread> pool;
  for (int t = 1; t < nt; t++) pool.emplace_back(work, t);
  work(0);
  for (auto &th : pool) th.join();
}

// The fused kNN of m queries (heap rows) against n references on host tables with the given
// maps and norms, into heap rows initialised as the adapter does (largest finite value, -1).
template <typename T>
static int knn_rows(int m, int n, int dim, int k, const T *query, const T *XA2, const int *amap,
                    const T *ref, const T *XB2, const int *bmap, std::vector<T> &D,
                    std::vector<int> &I) {
  D.assign((size_t)m * k, std::numeric_limits<T>::max());
  I.assign((size_t)m * k, -1);
  // *_var1 roles: queries (heap rows) first, then the references
  if (sizeof(T) == 8)
    dgsknn_var1(m, n, dim, k, (double *)query, (double *)XA2, (int *)amap, (double *)ref,
                (double *)XB2, (int *)bmap, (double *)D.data(), I.data());
  else
    sgsknn_var1(m, n, dim, k, (float *)query, (float *)XA2, (int *)amap, (float *)ref,
                (float *)XB2, (int *)bmap, (float *)D.data(), I.data());
  return gsknn_last_error();
}

template <typename T>
static int direct_kquery(const T *ref, const T *query, long n, long m, long k, long dim,
                         T *dist, long *id) {
  if (n == 0 || m == 0 || k == 0 || dim == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: n, m, k or dim is 0");
  if (n < 0 || m < 0 || k < 0 || dim < 0 || !ref || !query || !dist || !id)
    return set_status(GSKNN_ERR_ARG, "negative size or null pointer");
  if (n > 0x7fffffffL || m > 0x7fffffffL || k > 0x7fffffffL || dim > 0x7fffffffL ||
      m * k > 0x7fffffffL)
    return set_status(GSKNN_ERR_UNSUPPORTED, "sizes beyond int range");
  std::vector<T> r2((size_t)n), q2((size_t)m);
  row_norms(ref, n, dim, r2.data());
  row_norms(query, m, dim, q2.data());
  std::vector<int> amap((size_t)m), bmap((size_t)n);
  for (long i = 0; i < m; i++) amap[(size_t)i] = (int)i;
  for (long j = 0; j < n; j++) bmap[(size_t)j] = (int)j;
  std::vector<T> D;
  std::vector<int> I;
  const int rc = knn_rows<T>((int)m, (int)n, (int)dim, (int)k, query, q2.data(), amap.data(), ref,
                             r2.data(), bmap.data(), D, I);
  if (rc != GSKNN_OK) return rc;
  // the library writes every row descending (the k-th first): reversed, it is the ascending
  // list the adapter's heap pops produce (dgsrnn_directKQuery.cpp:112-124)
  for (long i = 0; i < m; i++)
    for (long t = 0; t < k; t++) {
      const size_t s = (size_t)(i * k + (k - 1 - t));
      dist[i * k + t] = D[s];
      id[i * k + t] = (long)I[s];
    }
  return set_status(GSKNN_OK, nullptr);
}

template <typename T>
static int direct_kquery_maps(int m, int n, int dim, int k, const T *query, const T *XA2,
                              const int *amap, const T *ref, const T *XB2, const int *bmap,
                              T *dist, long *id) {
  if (m == 0 || n == 0 || dim == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, dim or k is 0");
  if (m < 0 || n < 0 || dim < 0 || k < 0 || !query || !XA2 || !amap || !ref || !XB2 || !bmap ||
      !dist || !id)
    return set_status(GSKNN_ERR_ARG, "negative size or null pointer");
  if ((long)m * k > 0x7fffffffL) return set_status(GSKNN_ERR_UNSUPPORTED, "m * k beyond int range");
  std::vector<T> D;
  std::vector<int> I;
  const int rc = knn_rows<T>(m, n, dim, k, query, XA2, amap, ref, XB2, bmap, D, I);
  if (rc != GSKNN_OK) return rc;
  // heap order, copied out as dgsrnn_directKQuery_var2 does (dgsrnn_directKQuery.cpp:208-214)
  for (size_t s = 0; s < (size_t)m * k; s++) {
    dist[s] = D[s];
    id[s] = (long)I[s];
  }
  return set_status(GSKNN_OK, nullptr);
}

}  // namespace gsknn

extern "C" {

int gsknn_heap_sort_s_device(float *D, int *I, int n, int k, int ldk, void *stream) {
  return gsknn::heap_sort_device<float>(D, I, n, k, ldk, stream);
}

int gsknn_heap_sort_d_device(double *D, int *I, int n, int k, int ldk, void *stream) {
  return gsknn::heap_sort_device<double>(D, I, n, k, ldk, stream);
}

int gsknn_direct_kquery_d(const double *ref, const double *query, long n, long m, long k,
                          long dim, double *dist, long *id) {
  return gsknn::direct_kquery<double>(ref, query, n, m, k, dim, dist, id);
}

int gsknn_direct_kquery_s(const float *ref, const float *query, long n, long m, long k, long dim,
                          float *dist, long *id) {
  return gsknn::direct_kquery<float>(ref, query, n, m, k, dim, dist, id);
}

int gsknn_direct_kquery_maps_d(int m, int n, int dim, int k, const double *query,
                               const double *XA2, const int *amap, const double *ref,
                               const double *XB2, const int *bmap, double *dist, long *id) {
  return gsknn::direct_kquery_maps<double>(m, n, dim, k, query, XA2, amap, ref, XB2, bmap, dist,
                                           id);
}

int gsknn_direct_kquery_maps_s(int m, int n, int dim, int k, const float *query,
                               const float *XA2, const int *amap, const float *ref,
                               const float *XB2, const int *bmap, float *dist, long *id) {
  return gsknn::direct_kquery_maps<float>(m, n, dim, k, query, XA2, amap, ref, XB2, bmap, dist,
                                          id);
}

}  // extern "C"
