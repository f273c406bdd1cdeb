// knn_batch.cu -- the batching form: all-nearest-neighbour search over the leaves of
// randomized trees (alpha = beta = leaf point list), every leaf of a pass in one persistent
// launch, the pass captured once in a CUDA graph and replayed, heaps merged across passes.
//
// The reference runs such searches as one dgsknn call per leaf from its tree drivers; here one
// pass (the leaves of T trees over the same N points) is three kernels:
//   batch_pack      leaf rows gathered into k-major panels, every leaf padded to whole tiles
//                   (padding rows carry NaN norms and never become neighbours)
//   batch_knn_simt  persistent CTAs take work items (one query tile of one leaf against all of
//                   that leaf's candidate tiles) from an atomic counter, longest items first,
//                   and run the CUDA-core tile body (knn_simt_body.cuh); each query row's sorted
//                   list goes to a per-(tree, point) slot stamped with the pass number
//   batch_merge     one warp per point: the point's heap row and its lists from this pass's
//                   trees are merged with duplicates removed (the same neighbour found by
//                   several trees, or already in the heap from an earlier pass) and the k
//                   smallest are written back in descending order (a valid max-heap row)
// Arithmetic is the plain FP32 form of sgsknn: FP32 dot products in dimension order,
// d = (-2<q,c> + |c|^2) + |q|^2 clamped at 0, ties to the lower id.
//
// Tile shapes (BT = query tile = candidate tile rows) are chosen per (d, k, mean leaf size) by
// an autotuner that times every shape on the first pass it sees (results of the trial runs are
// discarded) and remembers the winner for the process.
#include "knn_common.cuh"
#include "knn_internal.h"
#include "knn_simt_body.cuh"
#include "gsknn.h"

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace gsknn {
namespace batch {

constexpr int DK = 16;

// ---- tile shapes: 0 = 128 x 128 tiles (8x8 per thread, 256 threads), 1 = 64 x 64 tiles
// (8x4 per thread, 128 threads), 2 = 64 x 64 tiles (4x4 per thread, 256 threads)
template <int KP, int SHAPE> struct Shape;
template <int KP> struct Shape<KP, 0> { using C = SimtCfg<float, KP, 2, 2, 4, 2, DK, 3>; };
template <int KP> struct Shape<KP, 1> { using C = SimtCfg<float, KP, 2, 1, 2, 2, DK, 3>; };
template <int KP> struct Shape<KP, 2> { using C = SimtCfg<float, KP, 1, 1, 4, 2, DK, 3>; };
constexpr int NSHAPES = 3;   // CUDA-core tile shapes
constexpr int SHAPE_TC = 3;  // the tensor-core shape (split BF16 + FP64 re-rank per tree)
inline int shape_bt(int shape) { return shape == 0 ? 128 : 64; }
inline bool shape_ok(int shape, int kp) { return kp <= 64 || shape != 0; }

struct Meta {          // per-pass counts, written by the host before each replay
  int ntiles;          // packed tiles this pass
  int nitems;          // work items this pass
  int pass_id;         // stamp of this pass's lists
  int pad;
};

// Pack the rows of pidx (point id, or -1 for padding) into panels [tile][nkc][DK][BT]; a
// fixed grid strides over this pass's (tile, dimension chunk) blocks.
__global__ void __launch_bounds__(256) batch_pack(const float *__restrict__ X,
                                                  const float *__restrict__ X2, int d, int N,
                                                  const int *__restrict__ pidx,
                                                  const Meta *__restrict__ meta, int BT, int nkc,
                                                  float *__restrict__ P,
                                                  float *__restrict__ norms,
                                                  uint32_t *__restrict__ ids,
                                                  uint32_t *__restrict__ rows,
                                                  const uint32_t *__restrict__ gid,
                                                  int *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float *s = reinterpret_cast<float *>(smem_raw);  // [DK][BT + 1]
  const int nblk = meta->ntiles * nkc;
  const int tid = threadIdx.x;
  for (int blk = blockIdx.x; blk < nblk; blk += gridDim.x) {
    const int tile = blk / nkc, kc = blk % nkc;
    for (int e = tid; e < BT * DK; e += blockDim.x) {
      const int r = e / DK, p = e % DK;
      const int gp = kc * DK + p;
      const int row = pidx[tile * BT + r];
      float v = 0.0f;
      if (row >= 0 && row < N && gp < d) v = X[(size_t)row * d + gp];
      s[p * (BT + 1) + r] = v;
    }
    __syncthreads();
    float *dst = P + ((size_t)(tile * nkc + kc) * DK) * BT;
    for (int e = tid; e < BT * DK; e += blockDim.x) {
      const int p = e / BT, r = e % BT;
      dst[(size_t)p * BT + r] = s[p * (BT + 1) + r];
    }
    if (kc == 0) {
      for (int r = tid; r < BT; r += blockDim.x) {
        const int gr = tile * BT + r;
        const int row = pidx[gr];
        float nv = Num<float>::nan();
        uint32_t id = NO_ID, lr = NO_ID;
        if (row >= 0 && row < N) {
          nv = X2[row];
          lr = (uint32_t)row;
          id = gid ? gid[row] : lr;
        } else if (row != -1) {
          atomicExch(status, GSKNN_ERR_INDEX);
        }
        norms[gr] = nv;
        ids[gr] = id;   // the id lists carry (global when gid is given)
        rows[gr] = lr;  // the heap row of the table (NO_ID: padding)
      }
    }
    __syncthreads();  // the staging tile is reused by the next block
  }
}

struct BatchArgs {
  const float *P, *norms;
  const uint32_t *ids;   // candidate ids written to the lists
  const uint32_t *rows;  // heap rows of the packed rows
  const int4 *items;   // (query tile, first candidate tile, end candidate tile, tree)
  const Meta *meta;
  int *next;           // work-item counter (zeroed before the launch)
  int nkc, k, N;
  const float *D;      // global heap (initial thresholds)
  int ldD;
  float *outD;         // lists [T][N][k]
  uint32_t *outI;
  int *stamp;          // [T][N]
};

template <class C>
__global__ void __launch_bounds__(C::NTHR) batch_knn_simt(BatchArgs a) {
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ int s_item;
  const int nitems = a.meta->nitems, pass_id = a.meta->pass_id;
  while (true) {
    if (threadIdx.x == 0) s_item = atomicAdd(a.next, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= nitems) break;
    const int4 w = a.items[it];
    SimtBlock<float> b;
    b.Apan = a.P + (size_t)w.x * a.nkc * C::DK * C::BQ;
    b.Bpack = a.P;
    b.qn = a.norms + (size_t)w.x * C::BQ;
    b.cn = a.norms;
    b.cid = a.ids;
    b.nkc = a.nkc;
    b.k = a.k;
    b.t_begin = w.y;
    b.t_end = w.z;
    b.nrows = C::BQ;
    b.rowid = a.rows + (size_t)w.x * C::BQ;
    b.row0 = 0;
    b.Din = a.D;
    b.ldD = a.ldD;
    b.outD = a.outD;
    b.outI = a.outI;
    b.out0 = (long long)w.w * a.N;
    simt_block<C>(smem, b);
    for (int r = threadIdx.x; r < C::BQ; r += C::NTHR) {
      const uint32_t id = b.rowid[r];
      if (id != NO_ID) a.stamp[(size_t)w.w * a.N + id] = pass_id;
    }
    __syncthreads();  // the next item re-initialises the shared lists and s_item
  }
}

// L <- the N smallest distinct keys of (L U B); both ascending, N = 32*E; duplicates are
// equal (distance, id) pairs (the same neighbour reached twice by the same arithmetic).
template <int E>
__device__ __forceinline__ void merge_unique(float (&ld)[E], uint32_t (&li)[E],
                                             const float (&bd)[E], const uint32_t (&bi)[E],
                                             int lane) {
  float cd[2 * E];
  uint32_t ci[2 * E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    cd[e] = ld[e];
    ci[e] = li[e];
    // B reversed behind L: ascending then descending, a bitonic sequence of 2N keys
    cd[E + e] = __shfl_sync(FULL_MASK, bd[E - 1 - e], 31 - lane);
    ci[E + e] = __shfl_sync(FULL_MASK, bi[E - 1 - e], 31 - lane);
  }
  warp_bitonic_merge<float, 2 * E>(cd, ci, lane);
  // element i = e*32 + lane; its predecessor is (e, lane-1) or (e-1, 31)
  bool dup[2 * E];
#pragma unroll
  for (int e = 0; e < 2 * E; e++) {
    const float ud = __shfl_up_sync(FULL_MASK, cd[e], 1);
    const uint32_t ui = __shfl_up_sync(FULL_MASK, ci[e], 1);
    const float wd = __shfl_sync(FULL_MASK, cd[e > 0 ? e - 1 : 0], 31);
    const uint32_t wi = __shfl_sync(FULL_MASK, ci[e > 0 ? e - 1 : 0], 31);
    const bool has_prev = lane > 0 || e > 0;
    const float pd = lane > 0 ? ud : wd;
    const uint32_t pi = lane > 0 ? ui : wi;
    dup[e] = has_prev && ci[e] != NO_ID && ci[e] == pi && cd[e] == pd;
  }
  bool any = false;
#pragma unroll
  for (int e = 0; e < 2 * E; e++) {
    if (dup[e]) {
      cd[e] = Num<float>::inf();
      ci[e] = NO_ID;
      any = true;
    }
  }
  if (__any_sync(FULL_MASK, any)) warp_sort<float, 2 * E>(cd, ci, lane);
#pragma unroll
  for (int e = 0; e < E; e++) {
    ld[e] = cd[e];
    li[e] = ci[e];
  }
}

template <int E>
__global__ void __launch_bounds__(256) batch_merge(float *__restrict__ D, int *__restrict__ I,
                                                   int ldD, int N, int k, int T,
                                                   const float *__restrict__ outD,
                                                   const uint32_t *__restrict__ outI,
                                                   const int *__restrict__ stamp,
                                                   const Meta *__restrict__ meta) {
  const int lane = threadIdx.x & 31;
  const int p = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (p >= N) return;
  const int pass_id = meta->pass_id;
  float ld[E];
  uint32_t li[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    ld[e] = t < k ? D[(size_t)p * ldD + t] : Num<float>::inf();
    li[e] = t < k ? (uint32_t)I[(size_t)p * ldD + t] : NO_ID;
  }
  warp_sort<float, E>(ld, li, lane);
  for (int tr = 0; tr < T; tr++) {
    if (stamp[(size_t)tr * N + p] != pass_id) continue;  // not in this tree this pass
    const size_t base = ((size_t)tr * N + p) * k;
    float bd[E];
    uint32_t bi[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int t = e * 32 + lane;
      bd[e] = t < k ? outD[base + t] : Num<float>::inf();
      bi[e] = t < k ? outI[base + t] : NO_ID;
    }
    merge_unique<E>(ld, li, bd, bi, lane);
  }
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (t < k) {
      D[(size_t)p * ldD + (k - 1 - t)] = ld[e];
      I[(size_t)p * ldD + (k - 1 - t)] = (int)li[e];
    }
  }
}

// ---- host side -----------------------------------------------------------------------------
// Preparation (kernel attribute, occupancy -> persistent grid) runs outside stream capture;
// the launch itself is what a pass records.
template <class C>
static cudaError_t prep_leaves(int sms, int *grid) {
  cudaError_t e = cudaFuncSetAttribute(batch_knn_simt<C>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_knn_simt<C>, C::NTHR,
                                                    C::SMEM);
  if (e != cudaSuccess) return e;
  *grid = std::max(1, per_sm) * sms;
  return cudaSuccess;
}

template <class C>
static cudaError_t launch_leaves(const BatchArgs &a, int grid, cudaStream_t st) {
  batch_knn_simt<C><<<grid, C::NTHR, C::SMEM, st>>>(a);
  return cudaGetLastError();
}

// prep (grid_out != nullptr) or launch (grid) the leaf kernel of (kp, shape)
template <int KP, int S>
static cudaError_t leaves_op(const BatchArgs *a, int sms, int grid, int *grid_out,
                             cudaStream_t st) {
  using C = typename Shape<KP, S>::C;
  return grid_out ? prep_leaves<C>(sms, grid_out) : launch_leaves<C>(*a, grid, st);
}

template <int KP>
static cudaError_t leaves_kp(int shape, const BatchArgs *a, int sms, int grid, int *grid_out,
                             cudaStream_t st) {
  switch (shape) {
    case 0:
      if constexpr (KP <= 64) return leaves_op<KP, 0>(a, sms, grid, grid_out, st);
      return cudaErrorInvalidValue;
    case 1: return leaves_op<KP, 1>(a, sms, grid, grid_out, st);
    case 2: return leaves_op<KP, 2>(a, sms, grid, grid_out, st);
  }
  return cudaErrorInvalidValue;
}

static cudaError_t leaves_any(int kp, int shape, const BatchArgs *a, int sms, int grid,
                              int *grid_out, cudaStream_t st) {
  switch (kp) {
    case 32: return leaves_kp<32>(shape, a, sms, grid, grid_out, st);
    case 64: return leaves_kp<64>(shape, a, sms, grid, grid_out, st);
    case 128: return leaves_kp<128>(shape, a, sms, grid, grid_out, st);
    case 256: return leaves_kp<256>(shape, a, sms, grid, grid_out, st);
  }
  return cudaErrorInvalidValue;
}

static cudaError_t launch_merge(int kp, float *D, int *I, int ldD, int N, int k, int T,
                                const float *outD, const uint32_t *outI, const int *stamp,
                                const Meta *meta, cudaStream_t st) {
  const int blocks = (N + 7) / 8;
  switch (kp) {
    case 32: batch_merge<1><<<blocks, 256, 0, st>>>(D, I, ldD, N, k, T, outD, outI, stamp, meta); break;
    case 64: batch_merge<2><<<blocks, 256, 0, st>>>(D, I, ldD, N, k, T, outD, outI, stamp, meta); break;
    case 128: batch_merge<4><<<blocks, 256, 0, st>>>(D, I, ldD, N, k, T, outD, outI, stamp, meta); break;
    case 256: batch_merge<8><<<blocks, 256, 0, st>>>(D, I, ldD, N, k, T, outD, outI, stamp, meta); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

// process-wide autotuner memory: (d, kp, mean leaf size rounded to a power of two) -> shape
static std::mutex g_tune_mu;
static std::map<std::tuple<int, int, int, int>, int> g_tuned;

static int size_class(double mean_leaf) {
  int c = 1;
  while (c < mean_leaf && c < (1 << 20)) c <<= 1;
  return c;
}

}  // namespace batch

// One all-nearest-neighbour job: N points, T trees per pass, a global heap on the device.
struct BatchJob {
  int N, d, k, kp, ldD, T, leaf_min, nkc;
  const float *X, *X2;
  float *D;
  int *I;
  cudaStream_t user;   // the caller's stream: passes are ordered after its prior work, and
                       // its later work after the pass
  cudaStream_t st;     // the job's own stream (captured and replayed; the legacy default
                       // stream cannot be captured)
  cudaEvent_t ev_in, ev_out;
  int sms;
  int shape;           // tile shape (-1 until tuned or set)
  bool tuned_here;
  float tune_ms[batch::NSHAPES];
  int max_tiles;       // packed rows / 64 of the largest plan over every shape
  long long max_rows;  // T*N points plus up to 128 rows of padding per leaf
  int grid[batch::NSHAPES];  // persistent grid per prepared shape (0: not prepared)
  int pass_id;
  // device buffers
  void *dbuf;
  size_t dbytes;
  float *P, *norms, *outD;
  uint32_t *ids, *rows, *outI;
  const uint32_t *gid;  // global id of each table row (null: the row index itself)
  int *pidx, *stamp, *next, *status;
  int4 *items;
  batch::Meta *meta;
  // pinned staging of the plan
  int *h_pidx;
  int4 *h_items;
  batch::Meta *h_meta;
  cudaEvent_t staged;  // the previous pass's plan has been copied out of the staging buffers
  // graph of one pass (pack, leaves, merge) for the tuned shape
  cudaGraph_t graph;
  cudaGraphExec_t exec;
  int graph_shape;
  // last pass
  int last_tiles, last_items;
  double last_evals;
  // tensor-core shape: one leaf panel per tree, the trees run one after another, each query
  // tile against its own leaf's candidate tiles, the exact re-rank merging into the heap
  int tc_tile;                  // candidate tile width of the panels (0: not available)
  TcLeafPlan tcl;               // plan of the allocated workspace (tcl.ok: allocated)
  void *tc_ws;
  // GSKNN_TC_COUNTERS=1: the leaf passes' epilogue and re-rank counters (device, 16 words),
  // printed and reset at each sync, with the panel rows and query-tile CTAs they cover
  unsigned long long *tc_counters;
  long long tc_cnt_rows, tc_cnt_ctas;
  int *tc_pidx;                 // device: every tree's panel rows (point or -1)
  int4 *tc_qtab;                // device: every tree's query-tile table
  int2 *tc_rtab;                // device: candidate tile range of every panel query tile
  int *h_tc_pidx;               // pinned staging of the three
  int4 *h_tc_qtab;
  int2 *h_tc_rtab;
  long long tc_cap_rows;        // capacity (rows over all trees) of the arrays above
  long long *h_tc_tree;         // per tree: rows, query tiles, and the offsets of the three
  bool tc_setup_done;           // the workspace holds the row map and the shift
  float *tD;                    // scratch heap for timing the tensor-core shape
  int *tI;
  float tune_tc_ms;
};

}  // namespace gsknn

using gsknn::BatchJob;
namespace gb = gsknn::batch;

static int set_err(int code, const char *msg) { return gsknn::set_status(code, "%s", msg); }

#define BCU(x)                                                             \
  do {                                                                     \
    cudaError_t e_ = (x);                                                  \
    if (e_ != cudaSuccess) {                                               \
      char m_[256];                                                        \
      std::snprintf(m_, sizeof(m_), "CUDA error in batching form: %s (%s)", \
                    cudaGetErrorString(e_), #x);                           \
      return set_err(GSKNN_ERR_CUDA, m_);                                  \
    }                                                                      \
  } while (0)

// Plan of one pass for tile rows BT: pidx (leaf rows padded to whole tiles), items (one per
// query tile, longest candidate range first). Returns tiles, items via the pointers.
static int build_plan(BatchJob *b, int BT, const int *leaf_ptr, const int *leaf_pts,
                      const int *leaf_tree, int nleaves, int *ntiles, int *nitems,
                      double *evals) {
  int tiles = 0;
  for (int l = 0; l < nleaves; l++) {
    const int L = leaf_ptr[l + 1] - leaf_ptr[l];
    if (L < 0) return set_err(GSKNN_ERR_ARG, "leaf_ptr must be non-decreasing");
    if (leaf_tree[l] < 0 || leaf_tree[l] >= b->T)
      return set_err(GSKNN_ERR_ARG, "leaf_tree entries must lie in [0, trees_per_pass)");
    tiles += (L + BT - 1) / BT;
  }
  if ((long long)tiles * BT > b->max_rows)
    return set_err(GSKNN_ERR_UNSUPPORTED,
                   "pass larger than the job was created for (too many leaves or points)");
  std::vector<int4> items;
  items.reserve(tiles);
  int t0 = 0;
  double ev = 0.0;
  for (int l = 0; l < nleaves; l++) {
    const int L = leaf_ptr[l + 1] - leaf_ptr[l];
    const int nt = (L + BT - 1) / BT;
    int *dst = b->h_pidx + (size_t)t0 * BT;
    for (int r = 0; r < nt * BT; r++) dst[r] = r < L ? leaf_pts[leaf_ptr[l] + r] : -1;
    for (int q = 0; q < nt; q++) items.push_back(make_int4(t0 + q, t0, t0 + nt, leaf_tree[l]));
    ev += (double)L * L;
    t0 += nt;
  }
  std::stable_sort(items.begin(), items.end(),
                   [](const int4 &x, const int4 &y) { return x.z - x.y > y.z - y.y; });
  std::memcpy(b->h_items, items.data(), items.size() * sizeof(int4));
  *ntiles = tiles;
  *nitems = (int)items.size();
  *evals = ev;
  return GSKNN_OK;
}

// Enqueue one pass (pack, leaves, optionally merge) for `shape` on the job's stream.
static cudaError_t prepare_shape(BatchJob *b, int shape) {
  if (b->grid[shape] > 0) return cudaSuccess;
  return gb::leaves_any(b->kp, shape, nullptr, b->sms, 0, &b->grid[shape], b->st);
}

static cudaError_t enqueue_pass(BatchJob *b, int shape, bool merge) {
  const int BT = gb::shape_bt(shape);
  cudaError_t e = cudaMemsetAsync(b->next, 0, sizeof(int), b->st);
  if (e != cudaSuccess) return e;
  const size_t psm = (size_t)gb::DK * (BT + 1) * 4;
  gb::batch_pack<<<b->sms * 8, 256, psm, b->st>>>(
      b->X, b->X2, b->d, b->N, b->pidx, b->meta, BT, b->nkc, b->P, b->norms, b->ids, b->rows,
      b->gid, b->status);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  gb::BatchArgs a{};
  a.P = b->P; a.norms = b->norms; a.ids = b->ids; a.rows = b->rows; a.items = b->items;
  a.meta = b->meta;
  a.next = b->next; a.nkc = b->nkc; a.k = b->k; a.N = b->N; a.D = b->D; a.ldD = b->ldD;
  a.outD = b->outD; a.outI = b->outI; a.stamp = b->stamp;
  e = gb::leaves_any(b->kp, shape, &a, b->sms, b->grid[shape], nullptr, b->st);
  if (e != cudaSuccess || !merge) return e;
  return gb::launch_merge(b->kp, b->D, b->I, b->ldD, b->N, b->k, b->T, b->outD, b->outI,
                          b->stamp, b->meta, b->st);
}

// Copy the staged plan of the pass to the device (ordered before the pass on the stream).
static cudaError_t upload_plan(BatchJob *b, int BT, int ntiles, int nitems) {
  cudaError_t e = cudaMemcpyAsync(b->pidx, b->h_pidx, (size_t)ntiles * BT * 4,
                                  cudaMemcpyHostToDevice, b->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->items, b->h_items, (size_t)nitems * sizeof(int4),
                        cudaMemcpyHostToDevice, b->st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(b->meta, b->h_meta, sizeof(gb::Meta), cudaMemcpyHostToDevice, b->st);
  if (e == cudaSuccess) e = cudaEventRecord(b->staged, b->st);
  return e;
}

// ---- tensor-core shape -----------------------------------------------------------------------
// Per tree of the pass: its leaves laid out at multiples of the tile width, the query tiles that
// hold real rows (each with its leaf's candidate tile range) and, for every panel query tile,
// the range (the leaf brute force's lookup). Fills the pinned staging and the per-tree table.
static int build_tc_plan(BatchJob *b, const int *leaf_ptr, const int *leaf_pts,
                         const int *leaf_tree, int nleaves, double *evals, long long *need_rows,
                         int *max_tree_rows) {
  const int NT = b->tc_tile;
  std::vector<long long> rows(b->T, 0), nq(b->T, 0);
  double ev = 0.0;
  for (int l = 0; l < nleaves; l++) {
    const int L = leaf_ptr[l + 1] - leaf_ptr[l];
    if (L < 0) return set_err(GSKNN_ERR_ARG, "leaf_ptr must be non-decreasing");
    const int t = leaf_tree[l];
    if (t < 0 || t >= b->T)
      return set_err(GSKNN_ERR_ARG, "leaf_tree entries must lie in [0, trees_per_pass)");
    if (L == 0) continue;
    rows[t] += (long long)(L + NT - 1) / NT * NT;
    nq[t] += (L + 127) / 128;
    ev += (double)L * L;
  }
  long long tot = 0, mx = 0;
  for (int t = 0; t < b->T; t++) {
    tot += rows[t];
    mx = std::max(mx, rows[t]);
  }
  *need_rows = tot;
  *max_tree_rows = (int)std::min<long long>(mx, 1LL << 30);
  *evals = ev;
  if (tot > b->tc_cap_rows) return GSKNN_OK;  // the caller grows the arrays and calls again
  long long po = 0, qo = 0;
  for (int t = 0; t < b->T; t++) {
    long long *tr = b->h_tc_tree + 6 * t;
    tr[0] = rows[t];
    tr[1] = 0;
    tr[2] = po;       // panel rows offset
    tr[3] = qo;       // query-tile table offset
    tr[4] = po / 128; // range table offset
    tr[5] = 0;        // rows laid out so far
    po += rows[t];
    qo += nq[t];
  }
  for (int l = 0; l < nleaves; l++) {
    const int L = leaf_ptr[l + 1] - leaf_ptr[l];
    if (L == 0) continue;
    long long *tr = b->h_tc_tree + 6 * leaf_tree[l];
    const long long r0 = tr[5];
    const int span = (L + NT - 1) / NT * NT;
    int *dst = b->h_tc_pidx + tr[2] + r0;
    for (int r = 0; r < span; r++) dst[r] = r < L ? leaf_pts[leaf_ptr[l] + r] : -1;
    const int tb = (int)(r0 / NT), te = tb + span / NT;
    for (long long q = r0 / 128; q * 128 < r0 + L; q++)
      b->h_tc_qtab[tr[3] + tr[1]++] = make_int4((int)q, tb, te, 0);
    for (long long q = r0 / 128; q * 128 < r0 + span; q++)
      b->h_tc_rtab[tr[4] + q] = make_int2(tb, te);
    tr[5] += span;
  }
  return GSKNN_OK;
}

static void free_tc(BatchJob *b) {
  if (b->tc_ws) cudaFree(b->tc_ws);
  if (b->tc_counters) cudaFree(b->tc_counters);
  b->tc_counters = nullptr;
  if (b->tc_pidx) cudaFree(b->tc_pidx);
  if (b->h_tc_pidx) cudaFreeHost(b->h_tc_pidx);
  if (b->h_tc_qtab) cudaFreeHost(b->h_tc_qtab);
  if (b->h_tc_rtab) cudaFreeHost(b->h_tc_rtab);
  b->tc_ws = nullptr;
  b->tc_pidx = nullptr;
  b->h_tc_pidx = nullptr;
  b->h_tc_qtab = nullptr;
  b->h_tc_rtab = nullptr;
  b->tc_cap_rows = 0;
  b->tcl.ok = false;
  b->tc_setup_done = false;
}

// Workspace and plan arrays for `rows` panel rows over all trees, `tree_rows` for one tree (with
// a margin, so that later passes rarely need to grow them).
static int ensure_tc(BatchJob *b, long long rows, int tree_rows) {
  if (b->tcl.ok && rows <= b->tc_cap_rows && tree_rows <= b->tcl.rows_cap) return GSKNN_OK;
  BCU(cudaStreamSynchronize(b->st));
  BCU(cudaEventSynchronize(b->staged));
  free_tc(b);
  const long long cap = (rows + rows / 8 + 128 * b->T + 127) / 128 * 128;
  const long long tcap = ((long long)tree_rows + tree_rows / 8 + 127) / 128 * 128;
  b->tcl = gsknn::tc_leaf_plan(b->N, (int)std::min<long long>(tcap, 1LL << 30), b->d, b->k,
                               b->sms);
  if (!b->tcl.ok) return set_err(GSKNN_ERR_UNSUPPORTED, "tensor-core shape: no tile plan");
  const size_t pb = (size_t)cap * 4, qb = (size_t)(cap / 128) * sizeof(int4),
               rb = (size_t)(cap / 128) * sizeof(int2);
  if (cudaMalloc(&b->tc_ws, b->tcl.bytes) != cudaSuccess ||
      cudaMalloc((void **)&b->tc_pidx, pb + qb + rb + 512) != cudaSuccess ||
      cudaHostAlloc((void **)&b->h_tc_pidx, pb, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void **)&b->h_tc_qtab, qb, cudaHostAllocDefault) != cudaSuccess ||
      cudaHostAlloc((void **)&b->h_tc_rtab, rb, cudaHostAllocDefault) != cudaSuccess) {
    cudaGetLastError();
    free_tc(b);
    return set_err(GSKNN_ERR_NOMEM, "tensor-core shape: device memory exhausted");
  }
  char *base = reinterpret_cast<char *>(b->tc_pidx);
  b->tc_qtab = reinterpret_cast<int4 *>(base + ((pb + 255) & ~(size_t)255));
  b->tc_rtab = reinterpret_cast<int2 *>(base + ((pb + 255) & ~(size_t)255) +
                                        ((qb + 255) & ~(size_t)255));
  b->tc_cap_rows = cap;
  return GSKNN_OK;
}

// Upload the staged tensor-core plan and enqueue every tree's pass on the heap D / I.
static int enqueue_tc_pass(BatchJob *b, float *D, int *I) {
  long long prow = 0, pq = 0;
  for (int t = 0; t < b->T; t++) {
    prow += b->h_tc_tree[6 * t];
    pq += b->h_tc_tree[6 * t + 1];
  }
  BCU(cudaMemcpyAsync(b->tc_pidx, b->h_tc_pidx, (size_t)prow * 4, cudaMemcpyHostToDevice,
                      b->st));
  BCU(cudaMemcpyAsync(b->tc_qtab, b->h_tc_qtab, (size_t)pq * sizeof(int4),
                      cudaMemcpyHostToDevice, b->st));
  BCU(cudaMemcpyAsync(b->tc_rtab, b->h_tc_rtab, (size_t)(prow / 128) * sizeof(int2),
                      cudaMemcpyHostToDevice, b->st));
  BCU(cudaEventRecord(b->staged, b->st));
  static const bool want_counters = std::getenv("GSKNN_TC_COUNTERS") != nullptr;
  if (want_counters && !b->tc_counters) {
    BCU(cudaMalloc(&b->tc_counters, 16 * sizeof(unsigned long long)));
    BCU(cudaMemsetAsync(b->tc_counters, 0, 16 * sizeof(unsigned long long), b->st));
  }
  for (int t = 0; t < b->T; t++) {
    const long long *tr = b->h_tc_tree + 6 * t;
    if (tr[1] == 0) continue;
    BCU(gsknn::tc_leaf_pass(b->tcl, b->tc_ws, b->X, b->X2, b->N, b->d, b->k,
                            b->tc_pidx + tr[2], (int)tr[0], b->tc_qtab + tr[3], (int)tr[1],
                            b->tc_rtab + tr[4], D, I, b->ldD, b->status, b->st,
                            !b->tc_setup_done, b->tc_counters));
    b->tc_setup_done = true;
    b->tc_cnt_rows += tr[0];
    b->tc_cnt_ctas += tr[1];
  }
  return GSKNN_OK;
}

// Plan, grow and enqueue one tensor-core pass.
static int tc_pass(BatchJob *b, const int *leaf_ptr, const int *leaf_pts, const int *leaf_tree,
                   int nleaves, float *D, int *I, double *evals) {
  if (b->gid) return set_err(GSKNN_ERR_UNSUPPORTED, "tensor-core shape: not for global ids");
  BCU(cudaEventSynchronize(b->staged));  // the staging of the previous upload is free
  long long need = 0;
  int tmax = 0;
  int rc = build_tc_plan(b, leaf_ptr, leaf_pts, leaf_tree, nleaves, evals, &need, &tmax);
  if (rc != GSKNN_OK) return rc;
  if (!b->tcl.ok || need > b->tc_cap_rows || tmax > b->tcl.rows_cap) {
    rc = ensure_tc(b, need, tmax);
    if (rc != GSKNN_OK) return rc;
    rc = build_tc_plan(b, leaf_ptr, leaf_pts, leaf_tree, nleaves, evals, &need, &tmax);
    if (rc != GSKNN_OK) return rc;
  }
  return enqueue_tc_pass(b, D, I);
}

namespace gsknn {
// Rows of the job's table stand for the global points gid[row] (device array, N entries): the
// lists and the heap carry those ids, while leaves, stamps and heap rows index the table.
void batch_set_global_ids(void *job, const uint32_t *gid) {
  reinterpret_cast<BatchJob *>(job)->gid = gid;
}
}  // namespace gsknn

extern "C" {

gsknn_batch_t *gsknn_batch_create(int N, int d, int k, const float *X, const float *X2,
                                  float *D, int *I, int ldD, int trees_per_pass, int leaf_min,
                                  int shape, void *stream) {
  if (N <= 0 || d <= 0 || k <= 0 || trees_per_pass <= 0 || leaf_min <= 0 || ldD < k || !X ||
      !X2 || !D || !I) {
    set_err(GSKNN_ERR_ARG, "gsknn_batch_create: invalid sizes or null pointer");
    return nullptr;
  }
  if (k > 256) {
    set_err(GSKNN_ERR_UNSUPPORTED, "gsknn_batch_create: k > 256 is not supported");
    return nullptr;
  }
  if (shape > gb::SHAPE_TC) {
    set_err(GSKNN_ERR_ARG, "gsknn_batch_create: unknown tile shape");
    return nullptr;
  }
  BatchJob *b = new BatchJob();
  std::memset(b, 0, sizeof(BatchJob));
  b->N = N; b->d = d; b->k = k; b->ldD = ldD; b->T = trees_per_pass; b->leaf_min = leaf_min;
  b->kp = 32;
  while (b->kp < k) b->kp <<= 1;
  if (shape >= 0 && shape < gb::NSHAPES && !gb::shape_ok(shape, b->kp)) {
    delete b;
    set_err(GSKNN_ERR_UNSUPPORTED, "gsknn_batch_create: 128-row tiles need k <= 64");
    return nullptr;
  }
  b->X = X; b->X2 = X2; b->D = D; b->I = I;
  b->user = static_cast<cudaStream_t>(stream);
  b->shape = shape;
  b->nkc = (d + gb::DK - 1) / gb::DK;
  int dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, dev);
  b->tc_tile = gsknn::tc_leaf_tile(d, k, b->sms);
  b->tune_tc_ms = -1.f;
  if (shape == gb::SHAPE_TC && b->tc_tile == 0) {
    delete b;
    set_err(GSKNN_ERR_UNSUPPORTED, "gsknn_batch_create: no tensor-core tile plan for d and k");
    return nullptr;
  }
  b->h_tc_tree = new long long[6 * (size_t)trees_per_pass]();
  // every leaf pads to whole tiles: at most 127 rows each at 128-row tiles
  const long long leaves = (long long)trees_per_pass * ((N + leaf_min - 1) / leaf_min);
  const long long max_rows = (long long)trees_per_pass * N + 128 * leaves;
  const long long mt = (max_rows + 63) / 64;
  if (mt * 64 > (1LL << 31) - 1) {
    delete b;
    set_err(GSKNN_ERR_UNSUPPORTED, "gsknn_batch_create: problem too large");
    return nullptr;
  }
  b->max_tiles = (int)mt;
  b->max_rows = mt * 64;
  const size_t rows = (size_t)b->max_rows;
  const size_t TN = (size_t)trees_per_pass * N;
  size_t off = 0;
  auto take = [&](size_t n) { size_t o = off; off = (off + n + 255) & ~(size_t)255; return o; };
  const size_t oP = take(rows * (size_t)b->nkc * gb::DK * 4);
  const size_t oN = take(rows * 4), oId = take(rows * 4), oRow = take(rows * 4),
               oPidx = take(rows * 4);
  const size_t oOD = take(TN * k * 4), oOI = take(TN * k * 4), oSt = take(TN * 4);
  const size_t oIt = take((size_t)b->max_tiles * sizeof(int4));
  const size_t oMeta = take(sizeof(gb::Meta)), oNext = take(4), oStat = take(4);
  b->dbytes = off;
  if (cudaMalloc(&b->dbuf, off) != cudaSuccess) {
    cudaGetLastError();
    delete b;
    set_err(GSKNN_ERR_NOMEM, "gsknn_batch_create: device memory exhausted");
    return nullptr;
  }
  char *base = static_cast<char *>(b->dbuf);
  b->P = reinterpret_cast<float *>(base + oP);
  b->norms = reinterpret_cast<float *>(base + oN);
  b->ids = reinterpret_cast<uint32_t *>(base + oId);
  b->rows = reinterpret_cast<uint32_t *>(base + oRow);
  b->pidx = reinterpret_cast<int *>(base + oPidx);
  b->outD = reinterpret_cast<float *>(base + oOD);
  b->outI = reinterpret_cast<uint32_t *>(base + oOI);
  b->stamp = reinterpret_cast<int *>(base + oSt);
  b->items = reinterpret_cast<int4 *>(base + oIt);
  b->meta = reinterpret_cast<gb::Meta *>(base + oMeta);
  b->next = reinterpret_cast<int *>(base + oNext);
  b->status = reinterpret_cast<int *>(base + oStat);
  bool ok = cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_in, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventCreateWithFlags(&b->ev_out, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventRecord(b->ev_in, b->user) == cudaSuccess &&
            cudaStreamWaitEvent(b->st, b->ev_in, 0) == cudaSuccess &&
            cudaMemsetAsync(b->stamp, 0, TN * 4, b->st) == cudaSuccess &&
            cudaMemsetAsync(b->status, 0, 4, b->st) == cudaSuccess &&
            cudaHostAlloc((void **)&b->h_pidx, rows * 4, cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void **)&b->h_items, (size_t)b->max_tiles * sizeof(int4),
                          cudaHostAllocDefault) == cudaSuccess &&
            cudaHostAlloc((void **)&b->h_meta, sizeof(gb::Meta), cudaHostAllocDefault) ==
                cudaSuccess &&
            cudaEventCreateWithFlags(&b->staged, cudaEventDisableTiming) == cudaSuccess &&
            cudaEventRecord(b->staged, b->st) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    gsknn_batch_destroy(reinterpret_cast<gsknn_batch_t *>(b));
    set_err(GSKNN_ERR_CUDA, "gsknn_batch_create: staging set-up failed");
    return nullptr;
  }
  b->graph_shape = -1;
  gsknn::set_status(GSKNN_OK, nullptr);
  return reinterpret_cast<gsknn_batch_t *>(b);
}

int gsknn_batch_pass(gsknn_batch_t *job, const int *leaf_ptr, const int *leaf_pts,
                     const int *leaf_tree, int nleaves) {
  BatchJob *b = reinterpret_cast<BatchJob *>(job);
  if (!b || !leaf_ptr || !leaf_pts || !leaf_tree || nleaves < 0)
    return set_err(GSKNN_ERR_ARG, "gsknn_batch_pass: invalid argument");
  if (nleaves == 0) return set_err(GSKNN_EARLY_RETURN, "gsknn_batch_pass: no leaves");
  // the staging buffers are reused: wait until the previous pass's plan has been copied out
  BCU(cudaEventSynchronize(b->staged));
  b->pass_id++;
  // order the pass after the caller's work on its stream (e.g. the heap's initialisation)
  BCU(cudaEventRecord(b->ev_in, b->user));
  BCU(cudaStreamWaitEvent(b->st, b->ev_in, 0));
  // tune on this pass's leaves if no shape is known for (d, k, leaf size)
  const double mean_leaf = (double)(leaf_ptr[nleaves] - leaf_ptr[0]) / nleaves;
  // (the tensor-core shape is not open to jobs with global ids, so they tune apart)
  const auto key = std::make_tuple(b->d, b->kp, gb::size_class(mean_leaf), b->gid ? 1 : 0);
  if (b->shape < 0) {
    std::lock_guard<std::mutex> lk(gb::g_tune_mu);
    auto it = gb::g_tuned.find(key);
    if (it != gb::g_tuned.end()) b->shape = it->second;
  }
  if (b->shape < 0) {
    // time every shape on this pass (lists only, no merge: the heap is untouched)
    cudaEvent_t e0, e1;
    BCU(cudaEventCreate(&e0));
    BCU(cudaEventCreate(&e1));
    float best = 0.f;
    int best_s = -1;
    // the tensor-core shape writes the heap as it goes: it is timed on a scratch copy
    b->tune_tc_ms = -1.f;
    if (b->tc_tile > 0 && !b->gid) {
      const size_t hb = (size_t)b->N * b->ldD * 4;
      if (!b->tD) {
        if (cudaMalloc((void **)&b->tD, hb) != cudaSuccess ||
            cudaMalloc((void **)&b->tI, hb) != cudaSuccess) {
          cudaGetLastError();
          return set_err(GSKNN_ERR_NOMEM, "gsknn_batch_pass: no memory to tune");
        }
      }
      double ev = 0;
      for (int rep = 0; rep < 2; rep++) {  // warm-up (workspace, modules), then timed
        BCU(cudaMemcpyAsync(b->tD, b->D, hb, cudaMemcpyDeviceToDevice, b->st));
        BCU(cudaMemcpyAsync(b->tI, b->I, hb, cudaMemcpyDeviceToDevice, b->st));
        BCU(cudaEventRecord(e0, b->st));
        const int rc = tc_pass(b, leaf_ptr, leaf_pts, leaf_tree, nleaves, b->tD, b->tI, &ev);
        if (rc != GSKNN_OK) return rc;
        BCU(cudaEventRecord(e1, b->st));
        BCU(cudaEventSynchronize(e1));
        float ms = 0.f;
        BCU(cudaEventElapsedTime(&ms, e0, e1));
        b->tune_tc_ms = ms;
      }
      best = b->tune_tc_ms;
      best_s = gb::SHAPE_TC;
    }
    for (int s = 0; s < gb::NSHAPES; s++) {
      b->tune_ms[s] = -1.f;
      if (!gb::shape_ok(s, b->kp)) continue;
      int tiles = 0, items = 0;
      double ev = 0;
      const int rc = build_plan(b, gb::shape_bt(s), leaf_ptr, leaf_pts, leaf_tree, nleaves,
                                &tiles, &items, &ev);
      if (rc != GSKNN_OK) return rc;
      b->h_meta->ntiles = tiles;
      b->h_meta->nitems = items;
      b->h_meta->pass_id = b->pass_id;
      BCU(upload_plan(b, gb::shape_bt(s), tiles, items));
      BCU(prepare_shape(b, s));
      BCU(enqueue_pass(b, s, false));  // warm-up (module load, caches)
      BCU(cudaMemsetAsync(b->next, 0, sizeof(int), b->st));
      BCU(cudaEventRecord(e0, b->st));
      BCU(enqueue_pass(b, s, false));
      BCU(cudaEventRecord(e1, b->st));
      BCU(cudaEventSynchronize(e1));
      float ms = 0.f;
      BCU(cudaEventElapsedTime(&ms, e0, e1));
      b->tune_ms[s] = ms;
      if (best_s < 0 || ms < best) { best = ms; best_s = s; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->shape = best_s;
    b->tuned_here = true;
    std::lock_guard<std::mutex> lk(gb::g_tune_mu);
    gb::g_tuned[key] = best_s;
  }
  if (b->shape == gb::SHAPE_TC) {
    double ev = 0;
    const int rc = tc_pass(b, leaf_ptr, leaf_pts, leaf_tree, nleaves, b->D, b->I, &ev);
    if (rc != GSKNN_OK) return rc;
    BCU(cudaEventRecord(b->ev_out, b->st));
    BCU(cudaStreamWaitEvent(b->user, b->ev_out, 0));
    long long q = 0, rows = 0;
    for (int t = 0; t < b->T; t++) {
      rows += b->h_tc_tree[6 * t];
      q += b->h_tc_tree[6 * t + 1];
    }
    b->last_tiles = (int)(rows / 128);
    b->last_items = (int)q;
    b->last_evals = ev;
    gsknn::set_status(GSKNN_OK, nullptr);
    return GSKNN_OK;
  }
  const int BT = gb::shape_bt(b->shape);
  int tiles = 0, items = 0;
  double ev = 0;
  const int rc = build_plan(b, BT, leaf_ptr, leaf_pts, leaf_tree, nleaves, &tiles, &items, &ev);
  if (rc != GSKNN_OK) return rc;
  b->h_meta->ntiles = tiles;
  b->h_meta->nitems = items;
  b->h_meta->pass_id = b->pass_id;
  BCU(upload_plan(b, BT, tiles, items));
  BCU(prepare_shape(b, b->shape));
  if (b->graph_shape != b->shape) {
    // capture the pass once (buffers and launch shapes are fixed; the counts live on the
    // device), then replay it for every pass
    if (b->exec) { cudaGraphExecDestroy(b->exec); b->exec = nullptr; }
    if (b->graph) { cudaGraphDestroy(b->graph); b->graph = nullptr; }
    BCU(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
    cudaError_t e = enqueue_pass(b, b->shape, true);
    cudaGraph_t g = nullptr;
    cudaError_t e2 = cudaStreamEndCapture(b->st, &g);
    BCU(e);
    BCU(e2);
    b->graph = g;
    BCU(cudaGraphInstantiate(&b->exec, b->graph, 0));
    b->graph_shape = b->shape;
  }
  BCU(cudaGraphLaunch(b->exec, b->st));
  // and the caller's later work after the pass
  BCU(cudaEventRecord(b->ev_out, b->st));
  BCU(cudaStreamWaitEvent(b->user, b->ev_out, 0));
  b->last_tiles = tiles;
  b->last_items = items;
  b->last_evals = ev;
  gsknn::set_status(GSKNN_OK, nullptr);
  return GSKNN_OK;
}

int gsknn_batch_sync(gsknn_batch_t *job) {
  BatchJob *b = reinterpret_cast<BatchJob *>(job);
  if (!b) return set_err(GSKNN_ERR_ARG, "gsknn_batch_sync: null job");
  BCU(cudaStreamSynchronize(b->st));
  if (b->tc_counters && b->tc_cnt_rows > 0) {
    unsigned long long h[16] = {};
    BCU(cudaMemcpy(h, b->tc_counters, sizeof(h), cudaMemcpyDeviceToHost));
    BCU(cudaMemset(b->tc_counters, 0, sizeof(h)));
    const double rows = (double)b->tc_cnt_rows, warps = (double)b->tc_cnt_ctas * 8;
    std::fprintf(stderr,
                 "gsknn batch tc: panel rows=%lld logged/row=%.1f inserts/row=%.1f "
                 "slow-chunks/warp=%.1f chunks/warp=%.1f rerank-scanned/row=%.1f "
                 "exact/row=%.1f\n",
                 b->tc_cnt_rows, (double)h[0] / rows, (double)h[1] / rows, (double)h[3] / warps,
                 (double)h[4] / warps, (double)h[5] / rows, (double)h[6] / rows);
    b->tc_cnt_rows = b->tc_cnt_ctas = 0;
  }
  int st = 0;
  BCU(cudaMemcpy(&st, b->status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st == GSKNN_ERR_INDEX)
    return set_err(GSKNN_ERR_INDEX, "a leaf lists a point outside [0, N)");
  gsknn::set_status(GSKNN_OK, nullptr);
  return GSKNN_OK;
}

int gsknn_batch_info(const gsknn_batch_t *job, int *shape, int *tile_rows, int *grid,
                     int *tiles, int *items, double *evals, float *tune_ms) {
  const BatchJob *b = reinterpret_cast<const BatchJob *>(job);
  if (!b) return set_err(GSKNN_ERR_ARG, "gsknn_batch_info: null job");
  const bool tc = b->shape == gb::SHAPE_TC;
  if (shape) *shape = b->shape;
  if (tile_rows) *tile_rows = tc ? b->tc_tile : b->shape >= 0 ? gb::shape_bt(b->shape) : 0;
  if (grid) *grid = tc ? b->last_items : b->shape >= 0 ? b->grid[b->shape] : 0;
  if (tiles) *tiles = b->last_tiles;
  if (items) *items = b->last_items;
  if (evals) *evals = b->last_evals;
  if (tune_ms) {
    for (int s = 0; s < gb::NSHAPES; s++) tune_ms[s] = b->tuned_here ? b->tune_ms[s] : -1.f;
    tune_ms[gb::SHAPE_TC] = b->tuned_here ? b->tune_tc_ms : -1.f;
  }
  return GSKNN_OK;
}

void gsknn_batch_destroy(gsknn_batch_t *job) {
  BatchJob *b = reinterpret_cast<BatchJob *>(job);
  if (!b) return;
  if (b->st) cudaStreamSynchronize(b->st);
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->ev_in) cudaEventDestroy(b->ev_in);
  if (b->ev_out) cudaEventDestroy(b->ev_out);
  if (b->st) cudaStreamDestroy(b->st);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->staged) cudaEventDestroy(b->staged);
  if (b->h_pidx) cudaFreeHost(b->h_pidx);
  if (b->h_items) cudaFreeHost(b->h_items);
  if (b->h_meta) cudaFreeHost(b->h_meta);
  if (b->dbuf) cudaFree(b->dbuf);
  free_tc(b);
  if (b->tD) cudaFree(b->tD);
  if (b->tI) cudaFree(b->tI);
  delete[] b->h_tc_tree;
  delete b;
}

void gsknn_batch_forget_tuning(void) {
  std::lock_guard<std::mutex> lk(gb::g_tune_mu);
  gb::g_tuned.clear();
}

}  // extern "C"
