// knn_tc.cu -- the precision form of the fused kNN: tensor-core (tcgen05) distances in TF32,
// BF16 or split BF16 (hi*hi + hi*lo + lo*hi), with FP32 accumulation in TMEM, followed by an
// FP64 re-rank of every candidate whose approximate distance lies within a rigorous rounding
// bound of the query's k-th approximate distance. The result is the exact FP64 top-k (ties to
// the lower id) of the caller's float inputs, merged into the caller's heaps.
//
// Kernels (one call):
//   tc_center,    shift vector mu = mean of a strided sample of candidate rows (partial sums
//   tc_center_fin per slice, then their fixed-order total and mu.mu)
//   tc_pack       one warp per row: gather, centre, round to the MMA format into a row-major
//                 [rows][d_pad] panel (TMA source), effective norm X2 - 2 mu.x + mu.mu (the
//                 centred norm, built on the caller's norm) in FP64, centred norm bound, ids;
//                 running maxima for the bound
//   tc_knn        warp 0 TMA producer, warp 1 MMA issuer (TMEM owner), warps 2-9 epilogue (two
//                 per TMEM lane quarter, each taking half of every tile's columns) with one
//                 query row per thread: approximate d' = qn' + cn' - 2<q~,c~> (with the norm
//                 column, cn' enters through one extra MMA against an all-ones A tile and the
//                 accumulator holds w = -v/2); per row and epilogue part a max-heap of the
//                 ceil(k/2) smallest d' of its own columns in shared memory; any two such heaps
//                 hold k candidates, so the second smallest root a row can see (its own, the
//                 other part's, and the roots up to three other splits published) bounds the
//                 k-th from above (threshold = that + 2E); a per-query log in HBM of every
//                 candidate under the threshold
//   tc_rerank     one warp per query: exact FP64 distances of the logged band, sorted merge with
//                 the incoming heap row, descending write-back (a valid max-heap);
//                 tc_rerank_hold (BF16, k <= 64) holds the band above the approximate k-th back,
//                 tc_rerank_leaf (batching form) sorts and writes a row only if it changes
//   tc_fallback   queries whose log overflowed: exact FP64 brute force over all candidates
//
// Error bound (per query q, all candidates c; u = unit roundoff of the MMA input format,
// M = max |c~|, CN = max |cn'|, D = padded dimension):
//   |d'(q,c) - d(q,c)| <= E_q = 1.25 * [ 2 (2u + u^2 + D 2^-23 (1+u)^2) |q~| M
//                                         + 3 * 2^-24 (CN + |qn'| + 2 |q~| M) ]
// For the split format the input term 2u + u^2 is replaced by 3.2 u^2 (u = 2^-8) and the
// accumulation term counts 3D products. With the norm column the accumulation counts 3 more
// terms, and E gains 1.25 (n 2^-23 + 2^-24) CN for the norm parts it sums (n accumulated terms).
#include "knn_common.cuh"
#include "knn_internal.h"
#include "tc_ptx.cuh"

#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>

namespace gsknn {
namespace tc {

constexpr int TC_M = 128;            // queries per CTA (TMEM lanes)
constexpr int CHUNK_BYTES = 128;     // K bytes per TMA box / swizzle atom row
constexpr int A_CHUNK = TC_M * CHUNK_BYTES;  // 16 KB
// Warp 0 TMA producer, warp 1 MMA issuer, then NEPI epilogue warps: NPART per TMEM lane quarter,
// part j of a quarter taking the j-th of NPART equal column ranges of every tile. Every part keeps
// a small heap of its own columns per row (the partition bound, see TcParams::proot).
constexpr int NEPI = TC_EPI_WARPS;
constexpr int NPART = TC_EPI_PARTS;
constexpr int NTHREADS = 32 * (2 + NEPI);
// accumulator columns per TMEM wait: 64 (two loads) while the registers allow, else 32
constexpr int EPI_STEP = NPART <= 2 ? 64 : 32;
constexpr uint32_t LOG_OVF = 1u << 30;
// The epilogue frees a TMEM accumulator as soon as its reads have landed, while it still uses
// the tile's candidate norms; the norms therefore get one slot more than the two accumulators
// (the slot the MMA warp refills belongs to a tile every epilogue warp has finished).
constexpr int CN_SLOTS = 3;

// ------------------------------------------------------------------------------------------
// shift vector
// ------------------------------------------------------------------------------------------
// The shift is the mean of a strided sample of the candidate rows, summed in a fixed order in
// two steps so that it is the same bits on every run:
//   tc_center   grid (dimension groups of 32, CENTER_SLICES slices of the sample), 32 warps per
//               block: lane = dimension, warps stride over the slice's rows (coalesced 128-byte
//               row segments), a block reduction in warp order, one partial sum per (slice,
//               dimension) and one row count per slice;
//   tc_center_fin  one block: mu = (sum of the partials in slice order) / rows, and mu.mu in FP64.
constexpr int CENTER_SLICES = 16;

__global__ void __launch_bounds__(1024) tc_center(const float *__restrict__ X, int d,
                                                  long long nrows, const int *__restrict__ idx,
                                                  int count, int nsample,
                                                  double *__restrict__ part,
                                                  int *__restrict__ part_n) {
  __shared__ double ps[32][33];
  __shared__ int pc[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int p = blockIdx.x * 32 + lane;
  const int t_lo = (int)((long long)nsample * blockIdx.y / CENTER_SLICES);
  const int t_hi = (int)((long long)nsample * (blockIdx.y + 1) / CENTER_SLICES);
  double s = 0.0;
  int used = 0;
  // eight sample rows per round: their index and row loads are independent and issue together
  for (int t0 = t_lo + warp; t0 < t_hi; t0 += 32 * 8) {
    float v[8];
    bool ok[8];
#pragma unroll
    for (int u = 0; u < 8; u++) {
      const int t = t0 + 32 * u;
      long long row = -1;
      if (t < t_hi) row = idx[(long long)t * count / nsample];
      ok[u] = row >= 0 && row < nrows;
      v[u] = ok[u] && p < d ? X[row * d + p] : 0.0f;
    }
#pragma unroll
    for (int u = 0; u < 8; u++) {
      if (ok[u]) {
        if (p < d) s += (double)v[u];
        used++;
      }
    }
  }
  ps[warp][lane] = s;
  if (lane == 0) pc[warp] = used;
  __syncthreads();
  if (warp == 0) {
    double tot = 0.0;
    int n = 0;
    for (int w = 0; w < 32; w++) {
      tot += ps[w][lane];
      n += pc[w];
    }
    if (p < d) part[(size_t)blockIdx.y * d + p] = tot;
    if (blockIdx.x == 0 && lane == 0) part_n[blockIdx.y] = n;
  }
}

__global__ void __launch_bounds__(256) tc_center_fin(const double *__restrict__ part,
                                                     const int *__restrict__ part_n, int d,
                                                     float *__restrict__ mu,
                                                     double *__restrict__ mu2) {
  __shared__ double red[8];
  int n = 0;
  for (int sl = 0; sl < CENTER_SLICES; sl++) n += part_n[sl];
  double s2 = 0.0;
  for (int p = threadIdx.x; p < d; p += blockDim.x) {
    double tot = 0.0;
    for (int sl = 0; sl < CENTER_SLICES; sl++) tot += part[(size_t)sl * d + p];
    const float m = n ? (float)(tot / n) : 0.0f;
    mu[p] = m;
    s2 += (double)m * (double)m;
  }
  for (int o = 16; o; o >>= 1) s2 += __shfl_xor_sync(FULL_MASK, s2, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s2;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    *mu2 = t;
  }
}

// ------------------------------------------------------------------------------------------
// packing
// ------------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

// Norm column of candidate row r (32 bytes, the K of one MMA): -cn/2 as the exact sum of three
// parts in the MMA input format (BF16: 3 x 8 significant bits; TF32: 3 x 11 >= the 24 of the
// float cn), then zeros. Against an all-ones A column the MMA adds -cn/2 to <q~, c~>, so the
// accumulator holds w = <q~, c~> - cn/2 = -v/2. A padding row holds -inf (w = -inf, v = +inf:
// never admitted).
__device__ __forceinline__ void write_norm_row(int fmt, void *npanel, int r, bool real, float cn) {
  uint4 lo4 = make_uint4(0u, 0u, 0u, 0u), hi4 = make_uint4(0u, 0u, 0u, 0u);
  const float x = -0.5f * cn;
  if (fmt == 0) {
    uint32_t h = 0xFF800000u, m = 0u, l = 0u;
    if (real) {
      h = to_tf32(x);
      const float r1 = x - __uint_as_float(h);
      m = to_tf32(r1);
      l = to_tf32(r1 - __uint_as_float(m));
    }
    lo4 = make_uint4(h, m, l, 0u);
  } else {
    uint32_t h = 0xFF80u, m = 0u, l = 0u;
    if (real) {
      const __nv_bfloat16 bh = __float2bfloat16_rn(x);
      const float r1 = x - __bfloat162float(bh);
      const __nv_bfloat16 bm = __float2bfloat16_rn(r1);
      const __nv_bfloat16 bl = __float2bfloat16_rn(r1 - __bfloat162float(bm));
      h = __bfloat16_as_ushort(bh);
      m = __bfloat16_as_ushort(bm);
      l = __bfloat16_as_ushort(bl);
    }
    lo4 = make_uint4(h | (m << 16), l, 0u, 0u);
  }
  uint4 *dst = reinterpret_cast<uint4 *>(static_cast<char *>(npanel) + (size_t)r * 32);
  dst[0] = lo4;
  dst[1] = hi4;
}

// fmt: 0 = TF32 (4-byte panel), 1 = BF16, 2 = split BF16 (hi and lo panels)
// Optional forms: `dcount` (device) replaces `count` and limits the panel to the tiles it needs;
// `rowmap` packs point idx[rowmap[r]] as row r; `gate` (device) skips all work when it reads 0;
// a null `enorm` writes the panels only (norms, bounds, ids and statistics are left alone);
// `pad_ok` packs index -1 as an empty padding row instead of reporting it; `npanel` (candidates)
// receives each row's norm column (write_norm_row).
__global__ void __launch_bounds__(256) tc_pack(
    int fmt, const float *__restrict__ X, const float *__restrict__ X2, int d, int d_pad,
    long long nrows, const int *__restrict__ idx, int count, int rows_pad,
    const float *__restrict__ mu, const double *__restrict__ mu2, int is_cand, void *panel,
    void *panel_lo, float *__restrict__ enorm, float *__restrict__ cnrm,
    uint32_t *__restrict__ ids, unsigned *__restrict__ stats, int *__restrict__ status,
    const int *__restrict__ dcount = nullptr, const int *__restrict__ rowmap = nullptr,
    const int *__restrict__ gate = nullptr, int pad_ok = 0, void *npanel = nullptr) {
  const int lane = threadIdx.x & 31;
  if (gate && *gate == 0) return;
  if (dcount) {
    count = *dcount;
    const int used = ((count + TC_M - 1) / TC_M) * TC_M;
    if (used < rows_pad) rows_pad = used;
  }
  // one row per warp, grid-stride; the candidate bound statistics are kept per warp and reach
  // the global maxima once per warp (not once per row: same-address atomics serialize)
  unsigned mx_nrm = 0u, mx_en = 0u;
  const int wstride = gridDim.x * (blockDim.x >> 5);
  for (int r = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); r < rows_pad;
       r += wstride) {
    long long row = -1;
    if (r < count) {
      row = idx[rowmap ? rowmap[r] : r];
      if (pad_ok && row == -1) {
        // a padding row of a leaf panel (the batching form): silently empty
      } else if (row < 0 || row >= nrows) {
        if (lane == 0) atomicExch(status, GSKNN_ERR_INDEX);
        row = -1;
      }
    }
    double s2 = 0.0, smx = 0.0;
    for (int p = lane; p < d_pad; p += 32) {
      float y = 0.0f;
      if (row >= 0 && p < d) {
        const float x = X[row * d + p];
        const float m = mu[p];
        y = x - m;
        smx += (double)m * (double)x;
        s2 += (double)y * (double)y;
      }
      const size_t o = (size_t)r * d_pad + p;
      if (fmt == 0) {
        reinterpret_cast<uint32_t *>(panel)[o] = to_tf32(y);
      } else if (fmt == 1) {
        reinterpret_cast<__nv_bfloat16 *>(panel)[o] = __float2bfloat16_rn(y);
      } else {
        const __nv_bfloat16 hi = __float2bfloat16_rn(y);
        const __nv_bfloat16 lo = __float2bfloat16_rn(y - __bfloat162float(hi));
        reinterpret_cast<__nv_bfloat16 *>(panel)[o] = hi;
        reinterpret_cast<__nv_bfloat16 *>(panel_lo)[o] = lo;
      }
    }
    for (int o = 16; o; o >>= 1) {
      s2 += __shfl_xor_sync(FULL_MASK, s2, o);
      smx += __shfl_xor_sync(FULL_MASK, smx, o);
    }
    if (lane == 0 && npanel) {
      // the same effective norm as below (the epilogue's cn), as the MMA's norm column
      const float enf = row >= 0 ? (float)((double)X2[row] - 2.0 * smx + *mu2) : 0.0f;
      write_norm_row(fmt, npanel, r, row >= 0, enf);
    }
    if (lane == 0 && enorm) {
      if (row >= 0) {
        // |x - mu|^2 expressed through the caller's norm: X2 - 2 mu.x + mu.mu
        const double en = (double)X2[row] - 2.0 * smx + *mu2;
        const float enf = (float)en;
        // centred norm of the stored (FP32-rounded) shift, rounded up
        const float nrm = (float)(sqrt(s2) * (1.0 + 1e-6)) * (1.0f + 1e-6f);
        enorm[r] = enf;
        cnrm[r] = nrm;
        if (ids) ids[r] = (uint32_t)row;
        // non-negative floats order like their bit patterns
        mx_nrm = max(mx_nrm, __float_as_uint(nrm));
        mx_en = max(mx_en, __float_as_uint(fabsf(enf) * (1.0f + 1e-6f)));
      } else {
        enorm[r] = Num<float>::nan();
        cnrm[r] = 0.0f;
        if (ids) ids[r] = NO_ID;
      }
    }
  }
  if (lane == 0 && enorm && is_cand && (mx_nrm | mx_en)) {
    atomicMax(&stats[0], mx_nrm);
    atomicMax(&stats[1], mx_en);
  }
}

// Blocks of a tc_pack launch over `rows` panel rows: one warp per row up to 16 CTAs of 8 warps
// per SM, grid-stride beyond.
static inline unsigned tc_pack_grid(long long rows) {
  const long long want = (rows + 7) / 8;
  return (unsigned)std::max(1LL, std::min(want, 148LL * 16));
}

// ------------------------------------------------------------------------------------------
// the tensor-core kernel
// ------------------------------------------------------------------------------------------
struct TcParams {
  int Q, k, nkc, ntiles_r, N, NST, logcap;
  int a_terms, b_terms, fmt;
  uint32_t idesc;
  const float *cn;
  const uint32_t *cid;
  const float *qn;
  const float *qnrm;
  const unsigned *stats;
  const float *Din;
  int ldD;
  float coefA, coefB, coefC;
  uint2 *log;
  int *logcnt;
  // Partition bound. A query's candidates fall into P = NPART * S partitions (split, part). Each
  // keeps a heap of the hk = ceil(k / NPART) smallest approximate distances among its own
  // candidates seen so far, and publishes its root at proot[query * P + split * NPART + part]
  // (bits of max(root, 0); all bits set while the heap is not full). Any NPART heaps hold at
  // least k real candidates, so the NPART-th smallest root among any partitions of the query --
  // those of its own CTA, and of up to W - 1 other splits as far as they have run -- bounds the
  // query's k-th from above.
  unsigned *proot;
  int hk, W, S;
  float *margin;
  int *status;
  float *dbg;
  long long dbg_ld;
  long long dbg_ncols;
  unsigned long long *counters;  // optional diagnostics (5 counters), may be null
  // optional (escalation pass): the query count on the device (Q is then the capacity and the
  // stride of the per-query arrays) and the heap row of each query
  const int *dQ;
  const int *rowmap;
  // optional (batching form): one entry per CTA -- (query tile, first candidate tile, end
  // candidate tile) -- in place of the (query tile, split) grid; rows whose rowmap entry is -1
  // are padding
  const int4 *qtab;
  // a full log marks the query overflowed at once, without compacting it (a later pass in a
  // narrower format finishes such queries)
  int no_compact;
};

struct SmemLayout {
  uint32_t a_off, b_off, an_off, bn_off, heap_off, cn_off, bar_off, tmem_off, total;
};

// Norm column (fold): an all-ones A tile and two slots of candidate norm tiles, 32-byte rows.
constexpr int NORM_ROW = 32;

// Partition bound (see TcParams::proot): heap entries per row and part, and the splits whose
// published roots a row reads (its own and up to three more).
__host__ __device__ inline int tc_heap_k(int k) { return (k + NPART - 1) / NPART; }
__host__ __device__ inline int tc_window(int S) { return S < 4 ? S : 4; }

// heap_row: heap entries per row over all epilogue parts; fold: the norm column areas
__host__ __device__ inline SmemLayout tc_smem_layout(int nkc, int a_terms, int b_terms, int N,
                                                     int NST, int heap_row, bool fold = false) {
  SmemLayout L;
  uint32_t off = 0;
  L.a_off = off;
  off += (uint32_t)a_terms * nkc * A_CHUNK;
  L.b_off = off;
  off += (uint32_t)NST * b_terms * N * CHUNK_BYTES;
  L.an_off = off;  // 1024-aligned: every area above is a multiple of 1 KB
  off += fold ? (uint32_t)TC_M * NORM_ROW : 0u;
  L.bn_off = off;
  off += fold ? 2u * N * NORM_ROW : 0u;
  L.heap_off = off;
  off += (uint32_t)heap_row * TC_M * 4;
  off = (off + 15) & ~15u;
  L.cn_off = off;  // candidate norms of the tiles in flight, copied by the MMA warp
  off += (uint32_t)CN_SLOTS * N * 4;
  off = (off + 7) & ~7u;
  L.bar_off = off;
  // full, empty, tfull[2], tempty[2], afull, cnfull, nfull[2], nempty[2]
  off += (uint32_t)(2 * NST + 9 + CN_SLOTS) * 8;
  L.tmem_off = off;
  off += 16;
  L.total = off + 1024;  // alignment slack
  return L;
}

struct EpiState {
  // root: this part's heap root; o1 <= o2: the two smallest roots among the other partitions
  // the row reads (as last published); pub: what this part last published
  // Tv: the filter bound on v = d' - qn'; Tw = -Tv/2 the same bound on w = -v/2 (norm column)
  float qn, E2, thr0, root, o1, o2, pub, thr, Tv, Tw;
  int cnt;
  int ovf;
  // optional diagnostics: logged candidates, heap inserts, convergent-loop iterations, chunks
  // that took the slow path
  unsigned n_ev, n_ins, n_it, n_sc;
};

// Any two partitions' heaps hold at least k real candidates, so the second smallest root among
// this part's and the others' bounds the query's k-th smallest approximate distance from above.
__device__ __forceinline__ void refresh_threshold(EpiState &s) {
  static_assert(NPART == 2, "the bound takes the NPART-th smallest root");
  float t = fminf(fmaxf(s.root, s.o1), s.o2) + s.E2;
  s.thr = t < s.thr0 ? t : s.thr0;
  // padding rows past the last query never admit; nor does a row whose log overflowed (the
  // query is finished by a later pass), so its chunks stop taking the slow path
  if (s.thr == -Num<float>::inf() || s.ovf) {
    s.Tv = -Num<float>::inf();
    s.Tw = Num<float>::inf();
    return;
  }
  // filter in the v = d' - qn' space with slack for the rounding of the subtraction
  s.Tv = (s.thr - s.qn) + (fabsf(s.thr) + fabsf(s.qn)) * 2.4e-7f + 1e-30f;
  s.Tw = -0.5f * s.Tv;  // exact: v <= Tv  <=>  w >= Tw
}

// Replace the heap root by x (< root) and sift down; returns the new root. Heap of k floats,
// element i of this thread's query at heap[i * TC_M + row] (bank-conflict free across a warp).
__device__ __forceinline__ float heap_replace_root(float *heap, int row, int k, float x) {
  int s = 0;
  while (true) {
    int c = 2 * s + 1;
    if (c >= k) break;
    float cv = heap[c * TC_M + row];
    if (c + 1 < k) {
      const float c2 = heap[(c + 1) * TC_M + row];
      if (c2 > cv) { cv = c2; c = c + 1; }
    }
    if (!(cv > x)) break;
    heap[s * TC_M + row] = cv;
    s = c;
  }
  heap[s * TC_M + row] = x;
  return heap[row];
}

// Drops log entries above the current threshold; returns the new count. Reads in batches of
// 16 before writing (writes never pass the read position), so the loads overlap.
__device__ __noinline__ int log_compact(uint2 *lg, int cnt, float thr) {
  int w = 0;
  for (int e = 0; e < cnt; e += 16) {
    uint2 buf[16];
#pragma unroll
    for (int j = 0; j < 16; j++) buf[j] = e + j < cnt ? lg[e + j] : make_uint2(0x7f800000u, 0u);
#pragma unroll
    for (int j = 0; j < 16; j++)
      if (__uint_as_float(buf[j].x) <= thr) lg[w++] = buf[j];
  }
  return w;
}

constexpr int PEND = 8;  // heap inserts a lane may defer before the warp flushes them

// Defer the heap insert of `dp` (when `ins`) into a small register ring, filled through
// compile-time indices so it stays in registers.
__device__ __forceinline__ void epi_defer(float dp, bool ins, float (&pend)[PEND], int &np) {
#pragma unroll
  for (int j = 0; j < PEND; j++) pend[j] = (ins && j == np) ? dp : pend[j];
  np += ins ? 1 : 0;
}

// One candidate of the exact slow path: log it (when `act` and under the threshold) and defer
// its heap insert. Branch-free: every lane of the warp runs it, with predicates instead of
// divergent branches.
__device__ __forceinline__ void epi_candidate(EpiState &s, float v, uint32_t id, bool act,
                                              uint2 *lg, int logcap, float (&pend)[PEND],
                                              int &np) {
  const float dp = v + s.qn;
  const bool take = act && dp <= s.thr;
  s.n_ev += take ? 1u : 0u;
  const bool room = s.cnt < logcap;
  if (take && !s.ovf && room) lg[s.cnt] = make_uint2(__float_as_uint(dp), id);
  s.cnt += (take && !s.ovf && room) ? 1 : 0;
  s.ovf |= (take && !room) ? 1 : 0;
  epi_defer(dp, take && dp < s.root, pend, np);
}

// Apply the deferred inserts (all lanes of the warp together, so their sift-downs overlap),
// publish the new root to the other partitions and tighten the threshold.
__device__ __forceinline__ void epi_flush(EpiState &s, float *heap, int row, int k,
                                          float (&pend)[PEND], int &np, unsigned *pslot) {
#pragma unroll
  for (int j = 0; j < PEND; j++) {
    if (j < np && pend[j] < s.root) {
      s.n_ins++;
      s.root = heap_replace_root(heap, row, k, pend[j]);
    }
  }
  np = 0;
  // published as non-negative float bits (a larger value bounds as well), which order like
  // unsigned integers; only this partition writes its slot
  const float pv = fmaxf(s.root, 0.0f);
  if (pv < s.pub) {
    __stcg(pslot, __float_as_uint(pv));
    s.pub = pv;
  }
  refresh_threshold(s);
}

// FOLD: the candidate norms enter through the MMA (the norm column, write_norm_row), so the
// accumulator holds w = -v/2 and the epilogue filters it directly; else the epilogue forms
// v = cn - 2<q~, c~> from the norms it reads into shared memory.
template <int FMT, bool FOLD>
__global__ void __launch_bounds__(NTHREADS, 1)
    tc_knn(const __grid_constant__ CUtensorMap tA, const __grid_constant__ CUtensorMap tAlo,
           const __grid_constant__ CUtensorMap tB, const __grid_constant__ CUtensorMap tBlo,
           const __grid_constant__ CUtensorMap tBn, const TcParams p) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // escalation pass: launched for the largest possible query count, the tiles past the count
  // on the device exit before any set-up
  const int Qn = p.dQ ? *p.dQ : p.Q;
  // grid: (query tile, split), query tiles fastest, so that a query's later splits mostly start
  // after its first ones finished and take their final roots as a tight bound from the first
  // tile; or one block per qtab entry
  if (!p.qtab && (int)blockIdx.x * TC_M >= Qn) return;
  const uint32_t raw = su32(smem_raw);
  unsigned char *smem = smem_raw + ((1024u - (raw & 1023u)) & 1023u);
  const SmemLayout L =
      tc_smem_layout(p.nkc, p.a_terms, p.b_terms, p.N, p.NST, NPART * p.hk, FOLD);
  unsigned char *sA = smem + L.a_off;
  unsigned char *sB = smem + L.b_off;
  unsigned char *sAn = smem + L.an_off;
  unsigned char *sBn = smem + L.bn_off;
  float *heap = reinterpret_cast<float *>(smem + L.heap_off);
  uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L.bar_off);
  uint64_t *full = bars;
  uint64_t *empty = bars + p.NST;
  uint64_t *tfull = bars + 2 * p.NST;
  uint64_t *tempty = bars + 2 * p.NST + 2;
  uint64_t *afull = bars + 2 * p.NST + 4;
  uint64_t *cnfull = bars + 2 * p.NST + 5;
  uint64_t *nfull = cnfull + CN_SLOTS;  // norm tile of slot b landed
  uint64_t *nempty = nfull + 2;         // norm tile of slot b read by the tile's MMAs
  float *cn_s = reinterpret_cast<float *>(smem + L.cn_off);
  uint32_t *tmem_holder = reinterpret_cast<uint32_t *>(smem + L.tmem_off);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  int qt = blockIdx.x, t_begin, t_end;
  const int split = blockIdx.y;
  if (p.qtab) {
    const int4 w = p.qtab[blockIdx.x];
    qt = w.x;
    t_begin = w.y;
    t_end = w.z;
  } else {
    // balanced ranges: every split gets floor or ceil of ntiles_r / S tiles
    t_begin = (int)((long long)split * p.ntiles_r / p.S);
    t_end = (int)((long long)(split + 1) * p.ntiles_r / p.S);
  }
  if (t_end > p.ntiles_r) t_end = p.ntiles_r;
  const int ntile = t_end > t_begin ? t_end - t_begin : 0;
  const int N = p.N;
  const uint32_t b_stage_bytes = (uint32_t)p.b_terms * N * CHUNK_BYTES;

  if (threadIdx.x == 0) {
    for (int s = 0; s < p.NST; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&tfull[b], 1);
      mbar_init(&tempty[b], NEPI);
    }
    mbar_init(afull, 1);
    for (int c = 0; c < CN_SLOTS; c++) mbar_init(&cnfull[c], 1);
    for (int b = 0; b < 2; b++) {
      mbar_init(&nfull[b], 1);
      mbar_init(&nempty[b], 1);
    }
    mbar_fence_init();
  }
  if (warp == 1) {
    tmem_alloc(tmem_holder, (uint32_t)(2 * N));
    tmem_relinquish();
  }
  // the per-row heaps start at +inf before any epilogue warp reads a root (each part of a lane
  // quarter reads the other's root as part of its bound)
  for (int i = threadIdx.x; i < NPART * p.hk * TC_M; i += NTHREADS) heap[i] = Num<float>::inf();
  if (FOLD) {
    // the all-ones A side of the norm column (every 16-byte chunk alike, so any swizzle of it is
    // the same bytes), made visible to the tensor core's operand reads
    const uint32_t one = FMT == 0 ? 0x3F800000u : 0x3F803F80u;
    uint32_t *an = reinterpret_cast<uint32_t *>(sAn);
    for (int i = threadIdx.x; i < TC_M * NORM_ROW / 4; i += NTHREADS) an[i] = one;
    fence_proxy_async_smem();
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem_base = *tmem_holder;
  bool failed = false;

  if (warp == 0) {
    // ---------------- TMA producer ----------------
    if (lane == 0 && ntile > 0) {
      prefetch_tmap(&tA);
      prefetch_tmap(&tB);
      const int celems = FMT == 0 ? 32 : 64;
      mbar_expect_tx(afull, (uint32_t)(p.a_terms * p.nkc * A_CHUNK));
      for (int kc = 0; kc < p.nkc; kc++) {
        tma_load_2d(sA + kc * A_CHUNK, &tA, kc * celems, qt * TC_M, afull);
        if (FMT == 2)
          tma_load_2d(sA + (p.nkc + kc) * A_CHUNK, &tAlo, kc * celems, qt * TC_M, afull);
      }
      int it = 0;
      if (FOLD) prefetch_tmap(&tBn);
      for (int lt = 0; lt < ntile && !failed; lt++) {
        const int tile = t_begin + lt;
        if (FOLD) {
          // the tile's norm column, into slot lt & 1 once the MMAs of tile lt - 2 read it
          const int nb = lt & 1;
          if (!mbar_wait(&nempty[nb], ((uint32_t)(lt >> 1) & 1u) ^ 1u)) { failed = true; break; }
          mbar_expect_tx(&nfull[nb], (uint32_t)(N * NORM_ROW));
          tma_load_2d(sBn + (uint32_t)nb * N * NORM_ROW, &tBn, 0, tile * N, &nfull[nb]);
        }
        for (int kc = 0; kc < p.nkc; kc++, it++) {
          const int s = it % p.NST;
          const uint32_t round = (uint32_t)(it / p.NST);
          if (!mbar_wait(&empty[s], (round & 1u) ^ 1u)) { failed = true; break; }
          mbar_expect_tx(&full[s], b_stage_bytes);
          unsigned char *dst = sB + (uint32_t)s * b_stage_bytes;
          tma_load_2d(dst, &tB, kc * celems, tile * N, &full[s]);
          if (FMT == 2)
            tma_load_2d(dst + N * CHUNK_BYTES, &tBlo, kc * celems, tile * N, &full[s]);
        }
      }
    }
  } else if (warp == 1) {
    // ---------------- MMA issuer ----------------
    if (lane == 0 && ntile > 0) {
      const long long t_start = p.counters ? clock64() : 0;
      long long w_tempty = 0, w_full = 0;
      if (!mbar_wait(afull, 0)) failed = true;
      tc_fence_after();
      const uint32_t a_base = su32(sA), b_base = su32(sB);
      int it = 0;
      for (int lt = 0; lt < ntile && !failed; lt++) {
        const int b = lt & 1;
        const uint32_t use = (uint32_t)(lt >> 1);
        long long t0 = p.counters ? clock64() : 0;
        if (!mbar_wait(&tempty[b], (use & 1u) ^ 1u)) { failed = true; break; }
        if (p.counters) w_tempty += clock64() - t0;
        // every epilogue warp has released tile lt - 2, so all of them are done with tile lt - 3
        // and its norm slot: fetch this tile's candidate norms there
        const uint32_t tmem_d = tmem_base + (uint32_t)(b * N);
        if (FOLD) {
          // the norm column first: w = -cn/2, then the products accumulate onto it
          if (!mbar_wait(&nfull[b], use & 1u)) { failed = true; break; }
          tc_fence_after();
          const uint64_t ad = sdesc_k_sw32(su32(sAn));
          const uint64_t bd = sdesc_k_sw32(su32(sBn) + (uint32_t)b * N * NORM_ROW);
          if (FMT == 0) mma_tf32(tmem_d, ad, bd, p.idesc, 0u);
          else mma_f16(tmem_d, ad, bd, p.idesc, 0u);
        } else {
          const int c = lt % CN_SLOTS;
          mbar_expect_tx(&cnfull[c], (uint32_t)(N * 4));
          bulk_g2s(cn_s + c * N, p.cn + (size_t)(t_begin + lt) * N, (uint32_t)(N * 4),
                   &cnfull[c]);
          tc_fence_after();
        }
        for (int kc = 0; kc < p.nkc; kc++, it++) {
          const int s = it % p.NST;
          const uint32_t round = (uint32_t)(it / p.NST);
          t0 = p.counters ? clock64() : 0;
          if (!mbar_wait(&full[s], round & 1u)) { failed = true; break; }
          if (p.counters) w_full += clock64() - t0;
          tc_fence_after();
          const uint32_t a_chunk = a_base + (uint32_t)kc * A_CHUNK;
          const uint32_t b_chunk = b_base + (uint32_t)s * b_stage_bytes;
#pragma unroll
          for (int ks = 0; ks < 4; ks++) {
            const uint32_t off = (uint32_t)ks * 32u;
            const uint64_t ad = sdesc_k_sw128(a_chunk + off);
            const uint64_t bd = sdesc_k_sw128(b_chunk + off);
            const uint32_t first = (!FOLD && kc == 0 && ks == 0) ? 0u : 1u;
            if (FMT == 0) {
              mma_tf32(tmem_d, ad, bd, p.idesc, first);
            } else {
              mma_f16(tmem_d, ad, bd, p.idesc, first);
              if (FMT == 2) {
                const uint64_t alo = sdesc_k_sw128(a_chunk + (uint32_t)p.nkc * A_CHUNK + off);
                const uint64_t blo = sdesc_k_sw128(b_chunk + (uint32_t)N * CHUNK_BYTES + off);
                mma_f16(tmem_d, ad, blo, p.idesc, 1u);
                mma_f16(tmem_d, alo, bd, p.idesc, 1u);
              }
            }
          }
          mma_commit(&empty[s]);
        }
        if (!failed) {
          if (FOLD) mma_commit(&nempty[b]);
          mma_commit(&tfull[b]);
        }
      }
      if (p.counters) {
        atomicAdd(&p.counters[7], (unsigned long long)w_full);
        atomicAdd(&p.counters[8], (unsigned long long)w_tempty);
        atomicAdd(&p.counters[10], (unsigned long long)(clock64() - t_start));
      }
    }
  } else {
    // ---------------- epilogue: one query row per thread ----------------
    const int lq = warp & 3;            // TMEM lane quarter this warp may access
    const int part = (warp - 2) >> 2;   // column range of the tile (and heap) of this warp
    const int row = lq * 32 + lane;
    const int gq = qt * TC_M + row;
    const bool valid = gq < Qn && (!p.rowmap || p.rowmap[gq] >= 0);
    float *const myheap = heap + part * p.hk * TC_M;
    const float *const otherheap = heap + (NPART - 1 - part) * p.hk * TC_M;
    const int P = NPART * p.S;  // partitions of a query
    EpiState s;
    s.cnt = 0;
    s.ovf = 0;
    s.o1 = Num<float>::inf();
    s.o2 = Num<float>::inf();
    s.pub = Num<float>::inf();
    s.n_ev = s.n_ins = s.n_it = s.n_sc = 0;
    unsigned *const pslot = p.proot + (size_t)(valid ? gq : 0) * P + NPART * split + part;
    const unsigned *const prow = p.proot + (size_t)(valid ? gq : 0) * P;
    float pend[PEND];
    int np = 0;
#pragma unroll
    for (int j = 0; j < PEND; j++) pend[j] = Num<float>::inf();
    s.root = Num<float>::inf();
    s.qn = 0.0f;
    s.E2 = 0.0f;
    s.thr0 = Num<float>::inf();
    if (valid) {
      s.qn = p.qn[gq];
      const float M = __uint_as_float(p.stats[0]);
      const float CN = __uint_as_float(p.stats[1]);
      const float qa = p.qnrm[gq];
      const float E =
          p.coefA * qa * M + p.coefB * (CN + fabsf(s.qn) + 2.0f * qa * M) + p.coefC * CN;
      s.E2 = 2.0f * E;
      if (p.Din) {
        float mx = -Num<float>::inf();
        const float *rowD = p.Din + (size_t)(p.rowmap ? p.rowmap[gq] : gq) * p.ldD;
        for (int j = 0; j < p.k; j++) mx = fmaxf(mx, rowD[j]);
        if (mx > -Num<float>::inf()) s.thr0 = mx + s.E2;
      }
      refresh_threshold(s);
      if (split == 0 && part == 0) p.margin[gq] = s.E2;
    } else {
      // padding row: its log and shared-bound pointers alias query 0, so it must never admit a
      // candidate; the -inf ceiling survives every threshold refresh
      s.thr0 = -Num<float>::inf();
      s.thr = -Num<float>::inf();
      s.Tv = -Num<float>::inf();
      s.Tw = Num<float>::inf();
    }
    const int lslot = NPART * split + part;  // this warp's log among the NPART*S logs of the query
    uint2 *lg = p.log + ((size_t)lslot * p.Q + (valid ? gq : 0)) * p.logcap;
    // One 32-column chunk: approximate distances, a cheap min-filter, and for the rare chunks
    // with survivors a warp-convergent pass in which every lane with pending candidates handles
    // one of them per iteration (selected from its registers by index).
    // Fast part of a 32-column chunk: d' - qn' (the v space) over the accumulator values in
    // place, and their minimum (a tree of depth 5). Two chunks' fast parts run back to back in
    // one basic block so their independent arithmetic overlaps.
    // With the norm column (FOLD) the registers already hold w = -v/2 and the fast part is the
    // maximum alone.
    auto fast = [&](uint32_t (&r)[32], const float *cnt, int c0) -> float {
      if constexpr (FOLD) {
        float m11[11];
#pragma unroll
        for (int j = 0; j < 10; j++)
          m11[j] = fmax3(__uint_as_float(r[3 * j]), __uint_as_float(r[3 * j + 1]),
                         __uint_as_float(r[3 * j + 2]));
        m11[10] = fmaxf(__uint_as_float(r[30]), __uint_as_float(r[31]));
        const float n0 = fmax3(m11[0], m11[1], m11[2]), n1 = fmax3(m11[3], m11[4], m11[5]);
        const float n2 = fmax3(m11[6], m11[7], m11[8]), n3 = fmaxf(m11[9], m11[10]);
        return fmaxf(fmax3(n0, n1, n2), n3);
      }
      const float4 *cn4 = reinterpret_cast<const float4 *>(cnt + c0);
#pragma unroll
      for (int j = 0; j < 8; j++) {
        const float4 c4 = cn4[j];
        float v0, v1, v2, v3;
        fma2(v0, v1, __uint_as_float(r[4 * j + 0]), __uint_as_float(r[4 * j + 1]), -2.0f, c4.x,
             c4.y);
        fma2(v2, v3, __uint_as_float(r[4 * j + 2]), __uint_as_float(r[4 * j + 3]), -2.0f, c4.z,
             c4.w);
        r[4 * j + 0] = __float_as_uint(v0);
        r[4 * j + 1] = __float_as_uint(v1);
        r[4 * j + 2] = __float_as_uint(v2);
        r[4 * j + 3] = __float_as_uint(v3);
      }
      // minimum: three-input tree of depth 4 (32 -> 11 -> 4 -> 1)
      float m11[11];
#pragma unroll
      for (int j = 0; j < 10; j++)
        m11[j] = fmin3(__uint_as_float(r[3 * j]), __uint_as_float(r[3 * j + 1]),
                       __uint_as_float(r[3 * j + 2]));
      m11[10] = fminf(__uint_as_float(r[30]), __uint_as_float(r[31]));
      const float n0 = fmin3(m11[0], m11[1], m11[2]), n1 = fmin3(m11[3], m11[4], m11[5]);
      const float n2 = fmin3(m11[6], m11[7], m11[8]), n3 = fminf(m11[9], m11[10]);
      return fminf(fmin3(n0, n1, n2), n3);
    };
    // whether a chunk's extreme value (minimum v, or maximum w with the norm column) admits
    auto hit = [&](float m) { return FOLD ? m >= s.Tw : m <= s.Tv; };
    auto dbg_write = [&](const uint32_t (&r)[32], size_t cbase, int c0) {
      for (int i = 0; i < 32; i++) {
        const long long col = (long long)cbase + c0 + i;
        const float v = FOLD ? -2.0f * __uint_as_float(r[i]) : __uint_as_float(r[i]);
        if (col < p.dbg_ncols) p.dbg[(size_t)gq * p.dbg_ld + col] = v + s.qn;
      }
    };
    // Slow part, for a chunk in which some lane has a candidate under its threshold: a
    // warp-convergent pass in which every lane with pending candidates logs one of them per
    // iteration (selected from its registers by index) and defers its heap insert.
    auto slow = [&](const uint32_t (&r)[32], size_t cbase, int c0) {
      // (a compaction that frees less than half of the log marks it overflowed: repeated
      // compactions that each free a few entries would cost a full read of the log per chunk)
      if (__any_sync(FULL_MASK, s.cnt > p.logcap - 32)) {
        if (s.cnt > p.logcap - 32 && !s.ovf) {
          if (!p.no_compact) s.cnt = log_compact(lg, s.cnt, s.thr);
          if (s.cnt > p.logcap / 2) {
            s.ovf = 1;
            refresh_threshold(s);
          }
        }
      }
      // pass mask as an OR tree (depth 5), built by every lane
      uint32_t m16[16];
#pragma unroll
      for (int j = 0; j < 16; j++) {
        if constexpr (FOLD)
          m16[j] = (__uint_as_float(r[2 * j]) >= s.Tw ? 1u << (2 * j) : 0u) |
                   (__uint_as_float(r[2 * j + 1]) >= s.Tw ? 1u << (2 * j + 1) : 0u);
        else
          m16[j] = (__uint_as_float(r[2 * j]) <= s.Tv ? 1u << (2 * j) : 0u) |
                   (__uint_as_float(r[2 * j + 1]) <= s.Tv ? 1u << (2 * j + 1) : 0u);
      }
#pragma unroll
      for (int w = 8; w >= 1; w >>= 1)
#pragma unroll
        for (int j = 0; j < w; j++) m16[j] = m16[2 * j] | m16[2 * j + 1];
      uint32_t mask = m16[0];
      s.n_sc++;
      while (__any_sync(FULL_MASK, mask != 0)) {
        s.n_it++;
        const bool act = mask != 0;
        const int i = (__ffs(mask) - 1) & 31;
        mask &= mask - 1;
        // v[i] for a runtime i: a 5-level select tree on the bits of i
        float t16[16];
#pragma unroll
        for (int j = 0; j < 16; j++) t16[j] = __uint_as_float((i & 16) ? r[j + 16] : r[j]);
#pragma unroll
        for (int w = 8, bit = 8; w >= 1; w >>= 1, bit >>= 1)
#pragma unroll
          for (int j = 0; j < w; j++) t16[j] = (i & bit) ? t16[j + w] : t16[j];
        const float vsel = FOLD ? -2.0f * t16[0] : t16[0];
        epi_candidate(s, vsel, (uint32_t)(cbase + c0 + i), act && valid, lg, p.logcap, pend, np);
        if (__any_sync(FULL_MASK, np == PEND)) epi_flush(s, myheap, row, p.hk, pend, np, pslot);
      }
    };
    // the two smallest roots up to W - 1 other splits have published (all bits set, which
    // orders last: a heap not full yet); the loads for the next tile are issued a tile ahead
    // so their latency hides behind the tile's work
    auto read_window = [&](unsigned &m1, unsigned &m2) {
      m1 = m2 = 0xFFFFFFFFu;
      for (int w = 1; w < p.W; w++) {
        int sp = split + w;
        if (sp >= p.S) sp -= p.S;
        const uint2 v = __ldcg(reinterpret_cast<const uint2 *>(prow + NPART * sp));
        m2 = min(m2, max(m1, v.x));
        m1 = min(m1, v.x);
        m2 = min(m2, max(m1, v.y));
        m1 = min(m1, v.y);
      }
    };
    auto as_bound = [](unsigned u) {
      return u == 0xFFFFFFFFu ? Num<float>::inf() : __uint_as_float(u);
    };
    unsigned win1 = 0xFFFFFFFFu, win2 = 0xFFFFFFFFu;
    if (valid) read_window(win1, win2);
    const long long t_start = p.counters ? clock64() : 0;
    long long w_tfull = 0;
    for (int lt = 0; lt < ntile && !failed; lt++) {
      const int b = lt & 1, c = lt % CN_SLOTS;
      const uint32_t use = (uint32_t)(lt >> 1), cuse = (uint32_t)(lt / CN_SLOTS);
      if (valid) {
        // the other part of this lane quarter (same rows, other columns) keeps its heap in
        // shared memory: its root is read directly (one 4-byte word, written whole)
        const float a = *reinterpret_cast<volatile const float *>(&otherheap[row]);
        const float w1 = as_bound(win1), w2 = as_bound(win2);
        const float o1 = fminf(a, w1), o2 = fminf(fmaxf(a, w1), w2);
        if (o1 < s.o1 || o2 < s.o2) {
          s.o1 = fminf(s.o1, o1);
          s.o2 = fminf(s.o2, o2);
          refresh_threshold(s);
        }
        read_window(win1, win2);
      }
      const long long t0 = p.counters ? clock64() : 0;
      if (!mbar_wait(&tfull[b], use & 1u)) { failed = true; break; }
      if (!FOLD && !mbar_wait(&cnfull[c], cuse & 1u)) { failed = true; break; }
      if (p.counters) w_tfull += clock64() - t0;
      tc_fence_after();
      const uint32_t taddr = tmem_base + ((uint32_t)(lq * 32) << 16) + (uint32_t)(b * N);
      const float *cnt = cn_s + c * N;
      const int tile = t_begin + lt;
      const size_t cbase = (size_t)tile * N;
      // this warp's N/NPART columns, EPI_STEP at a time (one or two 32-column chunks per TMEM
      // wait); the accumulator is freed for the MMA warp once the tile's last loads of every
      // epilogue warp have landed (the norms stay in their own slot)
      const int cb = part * (N / NPART), ce = cb + N / NPART;
      if (!p.dbg && __all_sync(FULL_MASK, !valid || s.ovf)) {
        // every row of this warp is padding or finished by a later pass: release the
        // accumulator without reading it (after its tile landed, so the release counts for
        // this tile)
        tc_fence_before();
        __syncwarp();
        if (lane == 0) mbar_arrive(&tempty[b]);
        continue;
      }
      for (int c0 = cb; c0 < ce; c0 += EPI_STEP) {
        if constexpr (EPI_STEP == 64) {
          uint32_t ra[32], rb[32];
          __syncwarp();
          tmem_ld32(taddr + (uint32_t)c0, ra);
          tmem_ld32(taddr + (uint32_t)c0 + 32u, rb);
          tmem_wait_ld();
          reg_fence32(ra);
          reg_fence32(rb);
          if (c0 + 64 >= ce) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
          }
          const float ma = fast(ra, cnt, c0);
          const float mb = fast(rb, cnt, c0 + 32);
          if (p.dbg && valid) {
            dbg_write(ra, cbase, c0);
            dbg_write(rb, cbase, c0 + 32);
          }
          if (__any_sync(FULL_MASK, hit(ma))) slow(ra, cbase, c0);
          if (__any_sync(FULL_MASK, hit(mb))) slow(rb, cbase, c0 + 32);
        } else {
          uint32_t ra[32];
          __syncwarp();
          tmem_ld32(taddr + (uint32_t)c0, ra);
          tmem_wait_ld();
          reg_fence32(ra);
          if (c0 + 32 >= ce) {
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[b]);
          }
          const float ma = fast(ra, cnt, c0);
          if (p.dbg && valid) dbg_write(ra, cbase, c0);
          if (__any_sync(FULL_MASK, hit(ma))) slow(ra, cbase, c0);
        }
      }
    }
    epi_flush(s, myheap, row, p.hk, pend, np, pslot);
    if (valid) p.logcnt[(size_t)lslot * p.Q + gq] = s.cnt | (s.ovf ? (int)LOG_OVF : 0);
    if (p.counters) {
      atomicAdd(&p.counters[0], (unsigned long long)s.n_ev);
      atomicAdd(&p.counters[1], (unsigned long long)s.n_ins);
      if (lane == 0) {
        atomicAdd(&p.counters[2], (unsigned long long)s.n_it);
        atomicAdd(&p.counters[3], (unsigned long long)s.n_sc);
        atomicAdd(&p.counters[4], (unsigned long long)ntile * (N / 64));
        atomicAdd(&p.counters[9], (unsigned long long)w_tfull);
        atomicAdd(&p.counters[11], (unsigned long long)(clock64() - t_start));
      }
    }
  }
  if (failed) atomicExch(p.status, GSKNN_ERR_TIMEOUT);
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == 1) tmem_dealloc(tmem_base, (uint32_t)(2 * N));
}

// ------------------------------------------------------------------------------------------
// FP64 re-rank of the logged band
// ------------------------------------------------------------------------------------------
struct RerankParams {
  int Q, k, S, logcap, d;
  const uint2 *log;
  const int *logcnt;
  const unsigned *proot;  // partition roots of tc_knn ([query][S]; S counts NPART per split)
  const float *margin;
  const float *Xq, *Xq2, *Xc, *Xc2;
  const int *qidx;
  const uint32_t *cid;  // packed candidate position -> point id
  float *D;
  int *I;
  int ldD;
  int *fallback_list;
  int *fallback_count;
  unsigned long long *counters;  // optional: [5] entries scanned, [6] exact distances
  const int *dQ;      // optional: query count on the device (Q is then the stride)
  const int *rowmap;  // optional: heap row (and query position in qidx) of each query; -1: none
  // batching form: candidates already in the incoming heap row (by id) are not entered twice,
  // and overflowed queries go to the fallback list as their own positions q
  int dedup;
};

// Exact squared distance of the oracle: (-2 <q,c> + |c|^2) + |q|^2 in FP64 from float inputs,
// clamped at zero; the dot product is split across the warp.
// The same distance computed by one thread: the FP64 dot product accumulates the (exact)
// float x float products in dimension order, as the oracle does (frame/dgsknn_ref_impl.h).
__device__ __forceinline__ double exact_dist_lane(const float *q, const float *c, int d,
                                                  double cc, double qq) {
  double acc = 0.0;
  const uintptr_t qc = reinterpret_cast<uintptr_t>(q) | reinterpret_cast<uintptr_t>(c);
  if ((d & 3) == 0 && (qc & 15) == 0) {
    const float4 *q4 = reinterpret_cast<const float4 *>(q);
    const float4 *c4 = reinterpret_cast<const float4 *>(c);
    for (int i = 0; i < (d >> 2); i++) {
      const float4 a = __ldg(q4 + i), b = __ldg(c4 + i);
      acc = fma((double)a.x, (double)b.x, acc);
      acc = fma((double)a.y, (double)b.y, acc);
      acc = fma((double)a.z, (double)b.z, acc);
      acc = fma((double)a.w, (double)b.w, acc);
    }
  } else {
    for (int pp = 0; pp < d; pp++) acc = fma((double)q[pp], (double)c[pp], acc);
  }
  const double v = fma(-2.0, acc, cc) + qq;
  return v < 0.0 ? 0.0 : v;
}

__device__ __forceinline__ double exact_dist_warp(const float *q, const float *c, int d,
                                                  double cc, double qq, int lane) {
  double acc = 0.0;
  for (int pp = lane; pp < d; pp += 32) acc = fma((double)q[pp], (double)c[pp], acc);
#pragma unroll
  for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(FULL_MASK, acc, o);
  double v = fma(-2.0, acc, cc) + qq;
  return v < 0.0 ? 0.0 : v;
}

template <int E>
__device__ __forceinline__ void write_heap_row(float *D, int *I, int ldD, int q, int k,
                                               const double (&ld)[E], const uint32_t (&li)[E],
                                               int lane) {
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (t < k) {
      D[(size_t)q * ldD + (k - 1 - t)] = (float)ld[e];
      I[(size_t)q * ldD + (k - 1 - t)] = (int)li[e];
    }
  }
}

// (sort = false leaves the list in the row's own order; sort it before merging into it)
template <int E>
__device__ __forceinline__ void load_heap_row(const float *D, const int *I, int ldD, int q, int k,
                                              double (&ld)[E], uint32_t (&li)[E], int lane,
                                              bool sort = true) {
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (t < k) {
      ld[e] = (double)D[(size_t)q * ldD + t];
      li[e] = (uint32_t)I[(size_t)q * ldD + t];
    } else {
      ld[e] = Num<double>::inf();
      li[e] = NO_ID;
    }
  }
  if (sort) warp_sort<double, E>(ld, li, lane);
}

// thr <- min(thr, k-th of the ascending exact list + E), rounded up: a candidate with d' above it
// has d > that k-th and cannot enter the list.
template <int E>
__device__ __forceinline__ void tighten_thr(const double (&ld)[E], int k, float Eq, float &thr) {
  double t = ld[0];
#pragma unroll
  for (int e2 = 0; e2 < E; e2++)
    if (e2 == (k - 1) / 32) t = ld[e2];
  const double dk = __shfl_sync(FULL_MASK, t, (k - 1) & 31);
  if (dk < 1e38) thr = fminf(thr, __fadd_ru(__double2float_ru(dk), Eq));
}

// Whether `id` (NO_ID: never) is one of the ids the warp holds in `li` (E per lane).
template <int E>
__device__ __forceinline__ bool id_in_row(uint32_t id, const uint32_t (&li)[E]) {
  bool hit = false;
#pragma unroll
  for (int e = 0; e < E; e++)
    for (int src = 0; src < 32; src++) hit |= __shfl_sync(FULL_MASK, li[e], src) == id;
  return hit && id != NO_ID;
}

constexpr int RR_BAND = 128;  // band entries (d' above the approximate k-th) a warp holds back

// HOLD: entries above the approximate k-th are held back and filtered against the threshold the
// nearly final exact k-th gives (pays where the band is wide: BF16); else one pass in log order.
// LAZY (the batching form's leaf pass): the incoming row stays unsorted until a candidate can
// enter it, and a row nothing entered is not written back.
template <int E, bool HOLD, bool LAZY>
__device__ __forceinline__ void rerank_body(const RerankParams &p) {
  __shared__ uint32_t rr_stage[8][64];
  __shared__ uint2 rr_band[8][HOLD ? RR_BAND : 1];
  const int lane = threadIdx.x & 31;
  const int q = blockIdx.x * 8 + (threadIdx.x >> 5);
  if (q >= (p.dQ ? *p.dQ : p.Q)) return;
  const int hr = p.rowmap ? p.rowmap[q] : q;  // heap row and query position
  if (hr < 0) return;                          // a padding row of a leaf panel
  // overflowed logs: the query goes to the next pass (a narrower format, or brute force)
  bool ovf = false;
  for (int s = 0; s < p.S; s++) ovf |= (p.logcnt[(size_t)s * p.Q + q] & (int)LOG_OVF) != 0;
  // the second smallest final root over the query's partitions (any two heaps hold k entries;
  // all bits set, ordering last: a heap that never filled)
  float T;
  {
    const unsigned *pr = p.proot + (size_t)q * p.S;
    unsigned m1 = 0xFFFFFFFFu, m2 = 0xFFFFFFFFu;
    for (int s = 0; s < p.S; s++) {
      const unsigned u = pr[s];
      m2 = min(m2, max(m1, u));
      m1 = min(m1, u);
    }
    T = m2 == 0xFFFFFFFFu ? Num<float>::inf() : __uint_as_float(m2);
  }
  if (ovf) {
    if (lane == 0) p.fallback_list[atomicAdd(p.fallback_count, 1)] = p.dedup ? q : hr;
    return;
  }
  const float E2 = p.margin[q];
  // Pass 1: the exact k-th smallest approximate distance over all of the query's logs. Every
  // candidate among the k smallest approximate distances was logged (its d' was below every
  // threshold in force), so this is the global approximate k-th, usually far below the bound T
  // the splits ended with. When all the logs together hold at most 32 entries (short lists:
  // leaves of the batching form), pass 2 takes them in one batch of exact distances whatever
  // the bound, so pass 1 is skipped and T stays the partition bound.
  int total = 0;
  for (int s = 0; s < p.S; s++) total += p.logcnt[(size_t)s * p.Q + q];
  if (total > 32) {
    float kd[E];
    uint32_t ki[E];
#pragma unroll
    for (int e = 0; e < E; e++) { kd[e] = Num<float>::inf(); ki[e] = NO_ID; }
    float kth = T;
    for (int s = 0; s < p.S; s++) {
      const int cnt = p.logcnt[(size_t)s * p.Q + q];
      const uint2 *lg = p.log + ((size_t)s * p.Q + q) * p.logcap;
      // one batch of log entries is loaded ahead, so that its latency overlaps the vote and
      // merge of the current batch
      float dv_next = lane < cnt ? __uint_as_float(lg[lane].x) : Num<float>::inf();
      for (int base = 0; base < cnt; base += 32) {
        const int e = base + lane;
        const float dv = dv_next;
        dv_next = e + 32 < cnt ? __uint_as_float(lg[e + 32].x) : Num<float>::inf();
        if (!__any_sync(FULL_MASK, dv <= kth)) continue;
        float b1[1] = {dv};
        uint32_t i1[1] = {(uint32_t)e};
        warp_sort<float, 1>(b1, i1, lane);
        warp_merge_32<float, E>(kd, ki, b1[0], i1[0], lane);
        float t = kd[0];
#pragma unroll
        for (int e2 = 0; e2 < E; e2++)
          if (e2 == (p.k - 1) / 32) t = kd[e2];
        kth = fminf(kth, __shfl_sync(FULL_MASK, t, (p.k - 1) & 31));
      }
    }
    T = kth;
  }
  // A candidate in the final top-k has d' <= d_k + E <= T + 2E. Its exact distance is also at
  // most the k-th of any k real candidates with exact distances (the incoming row and those
  // computed so far), so d' <= that k-th + E: the threshold tightens as the exact list fills.
  float thr = T + E2;
  const float Eq = 0.5f * E2;
  double ld[E];
  uint32_t li[E];
  // LAZY: the incoming row stays unsorted until some candidate can enter it: a batch whose
  // exact distances all exceed the list's k-th (the row's largest distance, until the first
  // merge) changes nothing, and a row nothing entered is not written back.
  load_heap_row<E>(p.D, p.I, p.ldD, hr, p.k, ld, li, lane, !LAZY);
  bool sorted = !LAZY;
  double lim = Num<double>::inf();
  if (HOLD) {
    tighten_thr<E>(ld, p.k, Eq, thr);
  } else {
    // the incoming row's largest distance bounds the k-th (as the list's k-th would)
    float mx = -Num<float>::inf();
    for (int j = lane; j < p.k; j += 32) mx = fmaxf(mx, p.D[(size_t)hr * p.ldD + j]);
    for (int o = 16; o; o >>= 1) mx = fmaxf(mx, __shfl_xor_sync(FULL_MASK, mx, o));
    if (mx > -Num<float>::inf() && mx < 1e38f) thr = fminf(thr, __fadd_ru(mx, Eq));
    lim = (double)mx;
  }
  uint32_t li0[E];  // the incoming row's ids (the batching form's duplicate check)
#pragma unroll
  for (int e = 0; e < E; e++) li0[e] = li[e];
  const long long qrow = p.qidx[hr];
  const float *qv = p.Xq + qrow * p.d;
  const double qq = (double)p.Xq2[qrow];
  // Pass 2: entries under the threshold are compacted into a per-warp staging list; every 32 of
  // them each lane computes one exact distance (independent row gathers across the lanes), then
  // the batch is sorted and merged into the exact list. With HOLD, entries at or under T (the k
  // smallest d') go first; those above T are held back in shared memory (as far as it holds
  // them) and filtered afterwards against the threshold the nearly final exact k-th gives.
  uint32_t *stg = rr_stage[threadIdx.x >> 5];
  int nb = 0;
  auto flush = [&](int count) {
    double dist = Num<double>::inf();
    uint32_t id = NO_ID;
    if (lane < count) id = p.cid[stg[lane]];
    // batching form: an id already in the incoming row is not entered again, and costs no
    // row gather
    if (p.dedup && id_in_row<E>(id, li0)) id = NO_ID;
    if (id != NO_ID)
      dist = exact_dist_lane(qv, p.Xc + (long long)id * p.d, p.d, (double)p.Xc2[id], qq);
    if (p.counters && lane == 0) atomicAdd(&p.counters[6], (unsigned long long)count);
    if (LAZY) {
      // nothing in this batch can enter (ties are settled by the merge itself)
      if (!__any_sync(FULL_MASK, id != NO_ID && dist <= lim)) return;
      if (!sorted) {
        warp_sort<double, E>(ld, li, lane);
        sorted = true;
      }
    }
    double b1[1] = {dist};
    uint32_t i1[1] = {id};
    warp_sort<double, 1>(b1, i1, lane);
    warp_merge_32<double, E>(ld, li, b1[0], i1[0], lane);
    if (LAZY) {
      double t = ld[0];
#pragma unroll
      for (int e2 = 0; e2 < E; e2++)
        if (e2 == (p.k - 1) / 32) t = ld[e2];
      lim = __shfl_sync(FULL_MASK, t, (p.k - 1) & 31);
    }
  };
  if constexpr (!HOLD) {
    for (int s = 0; s < p.S; s++) {
      const int cnt = p.logcnt[(size_t)s * p.Q + q];
      const uint2 *lg = p.log + ((size_t)s * p.Q + q) * p.logcap;
      if (p.counters && lane == 0) atomicAdd(&p.counters[5], (unsigned long long)cnt);
      for (int base = 0; base < cnt; base += 32) {
        const int e = base + lane;
        uint2 ent = make_uint2(0u, NO_ID);
        bool take = false;
        if (e < cnt) {
          ent = lg[e];
          take = __uint_as_float(ent.x) <= thr;
        }
        const unsigned m = __ballot_sync(FULL_MASK, take);
        if (take) stg[nb + __popc(m & ((1u << lane) - 1u))] = ent.y;
        nb += __popc(m);
        __syncwarp();
        if (nb >= 32) {
          flush(32);
          __syncwarp();
          const uint32_t rest = lane < nb - 32 ? stg[32 + lane] : 0u;
          __syncwarp();
          if (lane < nb - 32) stg[lane] = rest;
          nb -= 32;
          __syncwarp();
        }
      }
    }
  } else {
    uint2 *bnd = rr_band[threadIdx.x >> 5];
    int nbd = 0;
    // sources in order: the NPART * S logs, then (HOLD) the held band; one flush site
    for (int s = 0; s < p.S + (HOLD ? 1 : 0); s++) {
      const bool from_log = s < p.S;
      const int cnt = from_log ? p.logcnt[(size_t)s * p.Q + q] : nbd;
      const uint2 *lg = from_log ? p.log + ((size_t)s * p.Q + q) * p.logcap : bnd;
      if (p.counters && lane == 0 && from_log)
        atomicAdd(&p.counters[5], (unsigned long long)cnt);
      for (int base = 0; base < cnt; base += 32) {
        const int e = base + lane;
        uint2 ent = make_uint2(0u, NO_ID);
        bool take = false, band = false;
        if (e < cnt) {
          ent = lg[e];
          const float dv = __uint_as_float(ent.x);
          take = dv <= thr;
          band = HOLD && from_log && take && dv > T;
        }
        if (HOLD && from_log) {
          const unsigned mb = __ballot_sync(FULL_MASK, band);
          if (nbd + __popc(mb) <= RR_BAND) {
            if (band) bnd[nbd + __popc(mb & ((1u << lane) - 1u))] = ent;
            nbd += __popc(mb);
            take = take && !band;
          }
          __syncwarp();
        }
        const unsigned m = __ballot_sync(FULL_MASK, take);
        if (take) stg[nb + __popc(m & ((1u << lane) - 1u))] = ent.y;
        nb += __popc(m);
        __syncwarp();
        if (nb >= 32) {
          flush(32);
          if (HOLD) tighten_thr<E>(ld, p.k, Eq, thr);
          __syncwarp();
          const uint32_t rest = lane < nb - 32 ? stg[32 + lane] : 0u;
          __syncwarp();
          if (lane < nb - 32) stg[lane] = rest;
          nb -= 32;
          __syncwarp();
        }
      }
    }
  }
  if (nb > 0) flush(nb);
  if (sorted) write_heap_row<E>(p.D, p.I, p.ldD, hr, p.k, ld, li, lane);
}

template <int E>
__global__ void __launch_bounds__(256) tc_rerank(RerankParams p) {
  rerank_body<E, false, false>(p);
}

template <int E>
__global__ void __launch_bounds__(256) tc_rerank_leaf(RerankParams p) {
  rerank_body<E, false, true>(p);
}

// The held variant is capped at 64 registers (four CTAs per SM): this latency-bound kernel loses
// more to fewer resident warps than to a few spills.
template <int E>
__global__ void __launch_bounds__(256, 4) tc_rerank_hold(RerankParams p) {
  rerank_body<E, true, false>(p);
}

// ------------------------------------------------------------------------------------------
// exact brute force for queries whose log overflowed (rare; one CTA per query)
// ------------------------------------------------------------------------------------------
struct FallbackParams {
  int k, d, nc;
  const float *Xq, *Xq2, *Xc, *Xc2;
  const int *qidx, *cidx;
  long long nrows_c;
  float *D;
  int *I;
  int ldD;
  const int *list;
  const int *count;
};

template <int E>
__global__ void __launch_bounds__(256) tc_fallback(FallbackParams p) {
  __shared__ double sd[8][32 * E];
  __shared__ uint32_t si[8][32 * E];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int n = *p.count;
  for (int w = blockIdx.x; w < n; w += gridDim.x) {
    const int q = p.list[w];
    const long long qrow = p.qidx[q];
    const float *qv = p.Xq + qrow * p.d;
    const double qq = (double)p.Xq2[qrow];
    double ld[E];
    uint32_t li[E];
#pragma unroll
    for (int e = 0; e < E; e++) { ld[e] = Num<double>::inf(); li[e] = NO_ID; }
    double kth = Num<double>::inf();
    // each warp scans a strided share of the candidates, one candidate per lane at a time
    for (int base = warp * 32; base < p.nc; base += 256) {
      const int c = base + lane;
      double dist = Num<double>::inf();
      uint32_t id = NO_ID;
      if (c < p.nc) {
        const long long row = p.cidx[c];
        if (row >= 0 && row < p.nrows_c) {
          const float *cv = p.Xc + row * p.d;
          double acc = 0.0;
          for (int pp = 0; pp < p.d; pp++) acc = fma((double)qv[pp], (double)cv[pp], acc);
          dist = fma(-2.0, acc, (double)p.Xc2[row]) + qq;
          if (dist < 0.0) dist = 0.0;
          id = (uint32_t)row;
        }
      }
      if (__any_sync(FULL_MASK, dist <= kth)) {
        double b1[1] = {dist};
        uint32_t i1[1] = {id};
        warp_sort<double, 1>(b1, i1, lane);
        warp_merge_32<double, E>(ld, li, b1[0], i1[0], lane);
        double t = ld[0];
#pragma unroll
        for (int e = 0; e < E; e++)
          if (e == (p.k - 1) / 32) t = ld[e];
        kth = __shfl_sync(FULL_MASK, t, (p.k - 1) & 31);
      }
    }
#pragma unroll
    for (int e = 0; e < E; e++) {
      sd[warp][e * 32 + lane] = ld[e];
      si[warp][e * 32 + lane] = li[e];
    }
    __syncthreads();
    if (warp == 0) {
      double md[E];
      uint32_t mi[E];
      load_heap_row<E>(p.D, p.I, p.ldD, q, p.k, md, mi, lane);
      for (int w2 = 0; w2 < 8; w2++) {
        double bd[E];
        uint32_t bi[E];
#pragma unroll
        for (int e = 0; e < E; e++) {
          bd[e] = sd[w2][e * 32 + lane];
          bi[e] = si[w2][e * 32 + lane];
        }
        warp_merge_lists<double, E>(md, mi, bd, bi, lane);
      }
      write_heap_row<E>(p.D, p.I, p.ldD, q, p.k, md, mi, lane);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------------------------
// batching form: exact brute force of overflowed queries over their own leaf
// ------------------------------------------------------------------------------------------
struct LeafFallbackParams {
  int k, d, N;                 // N: candidate tile width of the panel
  const float *X, *X2;         // the point table
  const int *rowmap;           // panel row -> point (heap row)
  const uint32_t *ids;         // panel row -> point id (NO_ID: padding)
  const int2 *rtab;            // panel query tile -> (first, end) candidate tile of its leaf
  float *D;
  int *I;
  int ldD;
  const int *list;             // panel rows
  const int *count;
};

// One warp per listed query: the exact FP64 distances to every point of its leaf, merged with
// the incoming heap row (ids already there are not entered twice).
template <int E>
__global__ void __launch_bounds__(256) tc_fallback_leaf(LeafFallbackParams p) {
  const int lane = threadIdx.x & 31;
  const int n = *p.count;
  for (int w = blockIdx.x * 8 + (threadIdx.x >> 5); w < n; w += gridDim.x * 8) {
    const int q = p.list[w];
    const int hr = p.rowmap[q];
    const int2 r = p.rtab[q / TC_M];
    const float *qv = p.X + (long long)hr * p.d;
    const double qq = (double)p.X2[hr];
    double ld[E];
    uint32_t li[E];
    load_heap_row<E>(p.D, p.I, p.ldD, hr, p.k, ld, li, lane);
    uint32_t li0[E];
#pragma unroll
    for (int e = 0; e < E; e++) li0[e] = li[e];
    for (int base = r.x * p.N; base < r.y * p.N; base += 32) {  // warp-uniform trip count
      const int c = base + lane;
      uint32_t id = NO_ID;
      double dist = Num<double>::inf();
      if (c < r.y * p.N) {
        id = p.ids[c];
        if (id != NO_ID)
          dist = exact_dist_lane(qv, p.X + (long long)id * p.d, p.d, (double)p.X2[id], qq);
      }
      if (id_in_row<E>(id, li0)) {
        dist = Num<double>::inf();
        id = NO_ID;
      }
      double b1[1] = {dist};
      uint32_t i1[1] = {id};
      warp_sort<double, 1>(b1, i1, lane);
      warp_merge_32<double, E>(ld, li, b1[0], i1[0], lane);
    }
    write_heap_row<E>(p.D, p.I, p.ldD, hr, p.k, ld, li, lane);
  }
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    void *ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) ==
            cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiledFn>(ptr);
  }
  return fn;
}

// Row-major [rows][d_pad] panel of elem-byte elements; box = 128 bytes x box_rows rows, 128B
// swizzle (the K-major layout tcgen05 descriptors expect).
static cudaError_t make_panel_map(CUtensorMap *m, void *base, int elem, int d_pad, int rows,
                                  int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  cuuint64_t gdim[2] = {(cuuint64_t)d_pad, (cuuint64_t)rows};
  cuuint64_t gstride[1] = {(cuuint64_t)d_pad * elem};
  cuuint32_t box[2] = {(cuuint32_t)(CHUNK_BYTES / elem), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16,
                  2, base, gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Norm panel [rows][32 bytes] (write_norm_row), box of box_rows rows, 32-byte swizzle.
static cudaError_t make_norm_map(CUtensorMap *m, void *base, int elem, int rows, int box_rows) {
  EncodeTiledFn fn = encode_fn();
  if (!fn) return cudaErrorNotSupported;
  cuuint64_t gdim[2] = {(cuuint64_t)(NORM_ROW / elem), (cuuint64_t)rows};
  cuuint64_t gstride[1] = {(cuuint64_t)NORM_ROW};
  cuuint32_t box[2] = {(cuuint32_t)(NORM_ROW / elem), (cuuint32_t)box_rows};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(m, elem == 4 ? CU_TENSOR_MAP_DATA_TYPE_UINT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16,
                  2, base, gdim, gstride, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Launches tc_knn in the plan's format, with the norm column when `npanel` (the candidates' norm
// panel) is given and its areas fit; sets the matching error-bound coefficients in tp.
template <typename Grid>
static cudaError_t launch_tc_knn(const TcPlan &P, void *npanel, int npanel_rows, Grid grid,
                                 const CUtensorMap &mA, const CUtensorMap &mAlo,
                                 const CUtensorMap &mB, const CUtensorMap &mBlo, TcParams &tp,
                                 cudaStream_t st) {
  const bool fold = npanel && P.smem_fold;
  CUtensorMap mBn = mB;
  if (fold) {
    const cudaError_t e = make_norm_map(&mBn, npanel, P.elem, npanel_rows, P.N);
    if (e != cudaSuccess) return e;
  }
  tp.coefA = fold ? P.coefA_fold : P.coefA;
  tp.coefB = P.coefB;
  tp.coefC = fold ? P.coefC_fold : P.coefC;
  const unsigned smem = fold ? P.smem_fold : P.smem;
  cudaError_t e = cudaSuccess;
  auto go = [&](auto kern) {
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e == cudaSuccess) kern<<<grid, NTHREADS, smem, st>>>(mA, mAlo, mB, mBlo, mBn, tp);
  };
  if (P.fmt == 0) fold ? go(tc_knn<0, true>) : go(tc_knn<0, false>);
  else if (P.fmt == 1) fold ? go(tc_knn<1, true>) : go(tc_knn<1, false>);
  else fold ? go(tc_knn<2, true>) : go(tc_knn<2, false>);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e;
}

}  // namespace tc

static size_t al256(size_t x) { return (x + 255) & ~(size_t)255; }

int tc_format_of_mode(int mode) {
  return mode == GSKNN_TC_BF16 ? 1 : mode == GSKNN_TC_BF16X3 ? 2 : 0;
}

// Prepared-candidate area: mu, mu2, stats, panel(s), norms, norm bounds, ids.
struct CandLayout {
  size_t o_mu, o_mu2, o_cpart, o_stats, o_pb, o_pb_lo, o_pn, o_cn, o_cnrm, o_cid, bytes;
  int fmt, elem, d_pad, r_pad;
};

static CandLayout cand_layout(int nc, int d, int mode) {
  using namespace tc;
  CandLayout L{};
  L.fmt = tc_format_of_mode(mode);
  L.elem = L.fmt == 0 ? 4 : 2;
  const int celems = CHUNK_BYTES / L.elem;
  L.d_pad = ((d + celems - 1) / celems) * celems;
  L.r_pad = ((nc + 255) / 256) * 256;  // whole tiles of 256 and of 128 candidates
  size_t off = 0;
  auto take = [&](size_t b) { size_t o = off; off = al256(off + b); return o; };
  L.o_mu = take((size_t)d * 4);
  L.o_mu2 = take(8);
  L.o_cpart = take((size_t)CENTER_SLICES * d * 8 + CENTER_SLICES * 4);
  L.o_stats = take(16);
  L.o_pb = take((size_t)L.r_pad * L.d_pad * L.elem);
  L.o_pb_lo = L.fmt == 2 ? take((size_t)L.r_pad * L.d_pad * L.elem) : 0;
  L.o_pn = take((size_t)L.r_pad * NORM_ROW);
  L.o_cn = take((size_t)L.r_pad * 4);
  L.o_cnrm = take((size_t)L.r_pad * 4);
  L.o_cid = take((size_t)L.r_pad * 4);
  L.bytes = off;
  return L;
}

size_t tc_cand_bytes(int nc, int d, int mode) { return cand_layout(nc, d, mode).bytes; }

cudaError_t tc_cand_prepare(TcCand *C, void *mem, int nc, int d, int mode, const float *Xc,
                            const float *Xc2, long long nrows_c, const int *cidx, int *status,
                            cudaStream_t st) {
  using namespace tc;
  const CandLayout L = cand_layout(nc, d, mode);
  char *base = static_cast<char *>(mem);
  C->fmt = L.fmt; C->elem = L.elem; C->d = d; C->d_pad = L.d_pad; C->nc = nc; C->r_pad = L.r_pad;
  C->mu = reinterpret_cast<float *>(base + L.o_mu);
  C->mu2 = reinterpret_cast<double *>(base + L.o_mu2);
  C->stats = reinterpret_cast<unsigned *>(base + L.o_stats);
  C->pb = base + L.o_pb;
  C->pb_lo = L.fmt == 2 ? base + L.o_pb_lo : nullptr;
  C->pn = base + L.o_pn;
  C->cn = reinterpret_cast<float *>(base + L.o_cn);
  C->cnrm = reinterpret_cast<float *>(base + L.o_cnrm);
  C->cid = reinterpret_cast<uint32_t *>(base + L.o_cid);
  C->Xc = Xc; C->Xc2 = Xc2; C->nrows_c = nrows_c; C->cidx = cidx;
  C->efmt = -1; C->epb = nullptr; C->epb_lo = nullptr; C->epn = nullptr;
  cudaError_t e = cudaMemsetAsync(C->stats, 0, 16, st);
  if (e != cudaSuccess) return e;
  const int nsample = std::min(nc, 4096);
  {
    double *part = reinterpret_cast<double *>(base + L.o_cpart);
    int *part_n = reinterpret_cast<int *>(base + L.o_cpart + (size_t)CENTER_SLICES * d * 8);
    tc_center<<<dim3((d + 31) / 32, CENTER_SLICES), 1024, 0, st>>>(Xc, d, nrows_c, cidx, nc,
                                                                    nsample, part, part_n);
    tc_center_fin<<<1, 256, 0, st>>>(part, part_n, d, C->mu, C->mu2);
  }
  tc_pack<<<tc_pack_grid(L.r_pad), 256, 0, st>>>(L.fmt, Xc, Xc2, d, L.d_pad, nrows_c, cidx, nc,
                                            L.r_pad, C->mu, C->mu2, 1, C->pb, C->pb_lo, C->cn,
                                            C->cnrm, C->cid, C->stats, status, nullptr, nullptr,
                                            nullptr, 0, C->pn);
  return cudaGetLastError();
}

static TcPlan tc_plan_base(int nq, int nc, int d, int k, int mode, int sms, bool with_cand,
                          int max_splits) {
  using namespace tc;
  TcPlan P{};
  P.ok = false;
  P.sms = sms;
  P.max_splits = max_splits;
  P.fmt = tc_format_of_mode(mode);
  const int elem = P.fmt == 0 ? 4 : 2;
  const int celems = CHUNK_BYTES / elem;
  P.elem = elem;
  P.d_pad = ((d + celems - 1) / celems) * celems;
  P.nkc = P.d_pad / celems;
  P.a_terms = P.b_terms = P.fmt == 2 ? 2 : 1;
  P.kp = 32;
  while (P.kp < k) P.kp <<= 1;
  if (k > 256) return P;
  // candidate tile width and pipeline depth that fit in shared memory
  const uint32_t smem_max = 227 * 1024;
  int best_N = 0, best_NST = 0;
  const int Ns[2] = {256, 128};
  for (int ni = 0; ni < 2 && !best_N; ni++) {
    const int N = Ns[ni];
    if (P.fmt == 0 && N == 256 && P.nkc > 4) continue;  // keep the TF32 A tile room
    for (int NST = 6; NST >= 2; NST--) {
      SmemLayout L = tc_smem_layout(P.nkc, P.a_terms, P.b_terms, N, NST, NPART * tc_heap_k(k));
      if (L.total <= smem_max) { best_N = N; best_NST = NST; break; }
    }
  }
  if (!best_N) return P;
  P.N = best_N;
  P.NST = best_NST;
  P.qtiles = (nq + TC_M - 1) / TC_M;
  P.r_pad = ((nc + 255) / 256) * 256;
  P.rtiles = P.r_pad / P.N;
  P.q_pad = P.qtiles * TC_M;
  // splits: balance waves (one CTA per SM)
  const int smax = std::min(P.rtiles, max_splits > 0 ? max_splits : 16);
  int best_s = 1;
  double best = 1e300;
  for (int s = 1; s <= smax; s++) {
    const long long items = (long long)P.qtiles * s;
    // each split pays a start-up burst before the shared threshold tightens
    const double cost = (double)((items + sms - 1) / sms) / s * (1.0 + 0.03 * s);
    if (cost < best - 1e-12) { best = cost; best_s = s; }
  }
  P.S = best_s;
  P.tiles_per_split = (P.rtiles + P.S - 1) / P.S;
  P.hk = tc_heap_k(k);
  P.smem = tc_smem_layout(P.nkc, P.a_terms, P.b_terms, P.N, P.NST, NPART * P.hk).total;
  // the norm column where its areas fit beside the same tiles: in split BF16, and in BF16 from
  // two K chunks (measured: config 2 split BF16 -4% in tc_knn, BF16 at d = 256 -1.6%, but
  // BF16 at d = 64 +5%)
  {
    const uint32_t sf =
        tc_smem_layout(P.nkc, P.a_terms, P.b_terms, P.N, P.NST, NPART * P.hk, true).total;
    const bool wanted = P.fmt == 2 || (P.fmt == 1 && P.nkc >= 2);
    P.smem_fold = wanted && sf <= smem_max ? sf : 0u;
    if (const char *v = getenv("GSKNN_TC_FOLD"))
      if (atoi(v) == 0) P.smem_fold = 0u;
  }
  P.logcap = std::max(8 * P.kp, 1024);
  // workspace: [prepared candidates | query side]
  P.cand_bytes = with_cand ? al256(tc_cand_bytes(nc, d, mode)) : 0;
  size_t off = P.cand_bytes;
  auto take = [&](size_t b) { size_t o = off; off = al256(off + b); return o; };
  P.o_pa = take((size_t)P.q_pad * P.d_pad * elem);
  P.o_pa_lo = P.fmt == 2 ? take((size_t)P.q_pad * P.d_pad * elem) : 0;
  P.o_qn = take((size_t)P.q_pad * 4);
  P.o_qnrm = take((size_t)P.q_pad * 4);
  // NPART logs per (query, split): one per epilogue warp of a lane quarter
  P.o_log = take((size_t)NPART * P.S * nq * P.logcap * 8);
  P.o_logcnt = take((size_t)NPART * P.S * nq * 4);
  P.o_proot = take((size_t)NPART * P.S * nq * 4);
  P.o_margin = take((size_t)nq * 4);
  P.o_fbl = take((size_t)nq * 4);
  P.o_fbc = take(16);
  P.bytes = off;
  // error-bound coefficients
  const double D = (double)P.d_pad;
  double inp, accum, u;
  if (P.fmt == 2) {
    u = 1.0 / 256.0;
    inp = 3.2 * u * u;
    accum = 3.0 * D * std::ldexp(1.0, -23);
  } else {
    u = P.fmt == 0 ? std::ldexp(1.0, -11) : std::ldexp(1.0, -8);
    inp = 2.0 * u + u * u;
    accum = D * std::ldexp(1.0, -23) * (1 + u) * (1 + u);
  }
  P.coefA = (float)(1.25 * 2.0 * (inp + accum + std::ldexp(1.0, -22)));
  P.coefB = (float)(1.25 * 3.0 * std::ldexp(1.0, -24) + 1e-12);
  P.coefC = 0.0f;
  // With the norm column the accumulation also adds the three parts of -cn/2 (exact in the
  // input format): n = (products) + 3 terms accumulate, charged as truncation on the sum of
  // their magnitudes, |<q~, c~>| (1 + u)^2 + CN / 2; in v = -2w that is twice as much. The final
  // d' = v + qn' rounds once, inside the coefB term.
  {
    const double n = (P.fmt == 2 ? 3.0 * D : D) + 3.0;
    const double accf = n * std::ldexp(1.0, -23);
    P.coefA_fold = (float)(1.25 * 2.0 * (inp + accf * (1 + u) * (1 + u) + std::ldexp(1.0, -22)));
    P.coefC_fold = (float)(1.25 * (accf + std::ldexp(1.0, -24)) + 1e-12);
  }
  P.ok = true;
  return P;
}

// panels in one format: the data panel(s), then the norm panel
static size_t panel_bytes(int r_pad, int d_pad, int fmt) {
  const size_t one = al256((size_t)r_pad * d_pad * (fmt == 0 ? 4 : 2));
  return (fmt == 2 ? 2 * one : one) + al256((size_t)r_pad * tc::NORM_ROW);
}

size_t tc_cand_panel_bytes(int nc, int d, int mode) {
  const CandLayout L = cand_layout(nc, d, mode);
  return panel_bytes(L.r_pad, L.d_pad, L.fmt);
}

// Split BF16 has the narrowest band; a query whose BF16 or TF32 log overflowed runs again in it
// (or, from BF16, in TF32 where the split tiles do not fit).
int tc_escalation_mode(int nq, int nc, int d, int k, int mode, int sms) {
  const int fmt = tc_format_of_mode(mode);
  if (fmt == 2) return 0;
  if (tc_plan_base(nq, nc, d, k, GSKNN_TC_BF16X3, sms, false, 0).ok) return GSKNN_TC_BF16X3;
  if (fmt == 1 && tc_plan_base(nq, nc, d, k, GSKNN_TC_TF32, sms, false, 0).ok)
    return GSKNN_TC_TF32;
  return 0;
}

TcPlan tc_plan(int nq, int nc, int d, int k, int mode, int sms, bool with_cand,
               int max_splits) {
  TcPlan P = tc_plan_base(nq, nc, d, k, mode, sms, with_cand, max_splits);
  if (!P.ok) return P;
  P.esc_mode = tc_escalation_mode(nq, nc, d, k, mode, sms);
  if (P.esc_mode) {
    const TcPlan EP = tc_plan_base(nq, nc, d, k, P.esc_mode, sms, false, max_splits);
    P.o_esc = al256(P.bytes);
    P.esc_bytes = EP.bytes;
    size_t off = al256(P.o_esc + EP.bytes);
    if (with_cand) {  // per-call candidates: their escalation panels live in the workspace
      P.o_ecand = off;
      P.ecand_bytes = panel_bytes(EP.r_pad, EP.d_pad, EP.fmt);
      off = al256(off + P.ecand_bytes);
    }
    P.bytes = off;
  }
  return P;
}

cudaError_t tc_run(const TcPlan &P, int nq, int nc, int d, int k, const float *Xq,
                   const float *Xq2, long long nrows_q, const int *qidx, const float *Xc,
                   const float *Xc2, long long nrows_c, const int *cidx, float *D, int *I,
                   int ldD, void *ws, int *status, float *dbg, long long dbg_ld,
                   unsigned long long *counters, cudaStream_t st, TraceHook hook,
                   void *hook_ctx) {
  if (P.cand_bytes == 0) return cudaErrorInvalidValue;
  // centre, mu.mu and the candidate pack share the tracer's packing bracket
  if (hook) hook(hook_ctx, "tc_pack", true, st, 0);
  TcCand C{};
  const int mode = P.fmt == 1 ? GSKNN_TC_BF16 : P.fmt == 2 ? GSKNN_TC_BF16X3 : GSKNN_TC_TF32;
  cudaError_t e = tc_cand_prepare(&C, ws, nc, d, mode, Xc, Xc2, nrows_c, cidx, status, st);
  if (hook) hook(hook_ctx, "tc_pack", false, st, 3);
  if (e != cudaSuccess) return e;
  return tc_run_prepared(P, C, nq, d, k, Xq, Xq2, nrows_q, qidx, D, I, ldD, ws, status, dbg,
                         dbg_ld, counters, st, hook, hook_ctx);
}

// One approximate pass + re-rank: pack the queries (all of them, or on an escalation pass the
// `dQ` queries listed in `rowmap`), tc_knn in the plan's format, tc_rerank. Queries whose log
// overflowed are appended (as heap rows) to the plan's fallback list, whose count sits at
// base + P.o_fbc.
static cudaError_t tc_pass(const TcPlan &P, const TcCand &C, void *cand_pb, void *cand_pb_lo,
                           void *cand_pn, int nq, int d, int k, const float *Xq, const float *Xq2,
                           long long nrows_q, const int *qidx, const int *dQ, const int *rowmap,
                           float *D, int *I, int ldD, char *base, int *status, float *dbg,
                           long long dbg_ld, unsigned long long *counters, cudaStream_t st,
                           TraceHook hook, void *hook_ctx, bool escalation) {
  using namespace tc;
  void *pa = base + P.o_pa;
  void *pa_lo = P.fmt == 2 ? base + P.o_pa_lo : nullptr;
  float *qn = reinterpret_cast<float *>(base + P.o_qn);
  float *qnrm = reinterpret_cast<float *>(base + P.o_qnrm);
  int *fbc = reinterpret_cast<int *>(base + P.o_fbc);
  cudaError_t e = cudaMemsetAsync(fbc, 0, 16, st);
  if (e == cudaSuccess)
    e = cudaMemsetAsync(base + P.o_proot, 0xFF, (size_t)NPART * P.S * nq * 4, st);
  if (e != cudaSuccess) return e;
  // tracer brackets; `nk` = kernels of this file launched inside the bracket
  auto mark = [&](const char *name, bool begin, int nk = 0) {
    if (hook) hook(hook_ctx, name, begin, st, nk);
  };
  const char *n_pack = escalation ? "tc_escalate" : "tc_pack";
  const char *n_knn = escalation ? "tc_escalate" : "tc_knn";
  const char *n_rr = escalation ? "tc_escalate" : "tc_rerank";
  mark(n_pack, true);
  tc_pack<<<tc_pack_grid(P.q_pad), 256, 0, st>>>(P.fmt, Xq, Xq2, d, P.d_pad, nrows_q, qidx, nq,
                                            P.q_pad, C.mu, C.mu2, 0, pa, pa_lo, qn, qnrm,
                                            nullptr, C.stats, status, dQ, rowmap, nullptr);
  e = cudaGetLastError();
  mark(n_pack, false, 1);  // query pack
  if (e != cudaSuccess) return e;

  CUtensorMap mA, mAlo, mB, mBlo;
  e = make_panel_map(&mA, pa, P.elem, P.d_pad, P.q_pad, TC_M);
  if (e == cudaSuccess) e = make_panel_map(&mB, cand_pb, P.elem, P.d_pad, P.r_pad, P.N);
  if (e != cudaSuccess) return e;
  mAlo = mA;
  mBlo = mB;
  if (P.fmt == 2) {
    e = make_panel_map(&mAlo, pa_lo, P.elem, P.d_pad, P.q_pad, TC_M);
    if (e == cudaSuccess) e = make_panel_map(&mBlo, cand_pb_lo, P.elem, P.d_pad, P.r_pad, P.N);
    if (e != cudaSuccess) return e;
  }
  TcParams tp{};
  tp.Q = nq; tp.k = k; tp.nkc = P.nkc; tp.ntiles_r = P.rtiles;
  tp.N = P.N; tp.NST = P.NST; tp.logcap = P.logcap;
  tp.a_terms = P.a_terms; tp.b_terms = P.b_terms; tp.fmt = P.fmt;
  tp.idesc = idesc_f32acc(P.fmt == 0 ? 2u : 1u, TC_M, P.N);
  tp.cn = C.cn; tp.cid = C.cid; tp.qn = qn; tp.qnrm = qnrm; tp.stats = C.stats;
  tp.Din = D; tp.ldD = ldD;
  tp.log = reinterpret_cast<uint2 *>(base + P.o_log);
  tp.logcnt = reinterpret_cast<int *>(base + P.o_logcnt);
  tp.proot = reinterpret_cast<unsigned *>(base + P.o_proot);
  tp.hk = P.hk;
  tp.W = tc_window(P.S);
  tp.S = P.S;
  tp.margin = reinterpret_cast<float *>(base + P.o_margin);
  tp.status = status;
  tp.dbg = dbg;
  tp.dbg_ld = dbg_ld;
  tp.dbg_ncols = C.nc;
  tp.counters = counters;
  tp.dQ = dQ;
  tp.rowmap = rowmap;
  tp.no_compact = P.esc_mode != 0;
  dim3 grid(P.qtiles, P.S);
  mark(n_knn, true);
  e = launch_tc_knn(P, cand_pn, P.r_pad, grid, mA, mAlo, mB, mBlo, tp, st);
  mark(n_knn, false, 1);
  if (e != cudaSuccess) return e;

  RerankParams rp{};
  rp.Q = nq; rp.k = k; rp.S = NPART * P.S; rp.logcap = P.logcap; rp.d = d;
  rp.log = tp.log; rp.logcnt = tp.logcnt; rp.margin = tp.margin;
  rp.proot = tp.proot;
  rp.Xq = Xq; rp.Xq2 = Xq2; rp.Xc = C.Xc; rp.Xc2 = C.Xc2; rp.qidx = qidx; rp.cid = C.cid;
  rp.D = D; rp.I = I; rp.ldD = ldD;
  rp.fallback_list = reinterpret_cast<int *>(base + P.o_fbl);
  rp.fallback_count = fbc;
  rp.counters = counters;
  rp.dQ = dQ;
  rp.rowmap = rowmap;
  const int rb = (nq + 7) / 8;
  // one BF16 MMA per product leaves the widest band: hold it back behind the core entries
  // (k <= 64: larger lists would spill the held variant's registers)
  const bool hold = P.fmt == 1 && P.kp <= 64;
  mark(n_rr, true);
  switch (P.kp) {
    case 32: hold ? tc_rerank_hold<1><<<rb, 256, 0, st>>>(rp)
                  : tc_rerank<1><<<rb, 256, 0, st>>>(rp); break;
    case 64: hold ? tc_rerank_hold<2><<<rb, 256, 0, st>>>(rp)
                  : tc_rerank<2><<<rb, 256, 0, st>>>(rp); break;
    case 128: tc_rerank<4><<<rb, 256, 0, st>>>(rp); break;
    case 256: tc_rerank<8><<<rb, 256, 0, st>>>(rp); break;
    default: return cudaErrorInvalidValue;
  }
  e = cudaGetLastError();
  mark(n_rr, false, 1);
  return e;
}

// Exact FP64 brute force for the queries (heap rows) listed at base + P.o_fbl.
static cudaError_t tc_brute(const TcPlan &P, const TcCand &C, int d, int k, const float *Xq,
                            const float *Xq2, const int *qidx, float *D, int *I, int ldD,
                            char *base, cudaStream_t st, TraceHook hook, void *hook_ctx) {
  using namespace tc;
  FallbackParams fp{};
  fp.k = k; fp.d = d; fp.nc = C.nc; fp.Xq = Xq; fp.Xq2 = Xq2; fp.Xc = C.Xc; fp.Xc2 = C.Xc2;
  fp.qidx = qidx; fp.cidx = C.cidx; fp.nrows_c = C.nrows_c; fp.D = D; fp.I = I; fp.ldD = ldD;
  fp.list = reinterpret_cast<const int *>(base + P.o_fbl);
  fp.count = reinterpret_cast<const int *>(base + P.o_fbc);
  if (hook) hook(hook_ctx, "tc_fallback", true, st, 0);
  switch (P.kp) {
    case 32: tc_fallback<1><<<148, 256, 0, st>>>(fp); break;
    case 64: tc_fallback<2><<<148, 256, 0, st>>>(fp); break;
    case 128: tc_fallback<4><<<148, 256, 0, st>>>(fp); break;
    case 256: tc_fallback<8><<<148, 256, 0, st>>>(fp); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (hook) hook(hook_ctx, "tc_fallback", false, st, 1);
  return e;
}

cudaError_t tc_run_prepared(const TcPlan &P, const TcCand &C, int nq, int d, int k,
                            const float *Xq, const float *Xq2, long long nrows_q,
                            const int *qidx, float *D, int *I, int ldD, void *ws, int *status,
                            float *dbg, long long dbg_ld, unsigned long long *counters,
                            cudaStream_t st, TraceHook hook, void *hook_ctx) {
  using namespace tc;
  if (C.fmt != P.fmt || C.d_pad != P.d_pad || C.r_pad != P.r_pad) return cudaErrorInvalidValue;
  char *base = static_cast<char *>(ws);
  cudaError_t e = tc_pass(P, C, C.pb, C.pb_lo, C.pn, nq, d, k, Xq, Xq2, nrows_q, qidx, nullptr,
                          nullptr, D, I, ldD, base, status, dbg, dbg_ld, counters, st, hook,
                          hook_ctx, false);
  if (e != cudaSuccess) return e;
  // Escalation: the queries whose log overflowed run again in the narrower format against the
  // same candidates (their panels in that format: prepared with the candidates, or packed here
  // only when some query overflowed), as a pass over the list of overflowed heap rows whose
  // length stays on the device. What overflows there too goes to the FP64 brute force.
  const TcPlan EP = P.esc_mode ? tc_plan_base(nq, C.nc, d, k, P.esc_mode, P.sms, false,
                                              P.max_splits)
                               : TcPlan{};
  void *epb = nullptr, *epb_lo = nullptr, *epn = nullptr;
  if (EP.ok && C.efmt == EP.fmt) {
    epb = C.epb;
    epb_lo = C.epb_lo;
    epn = C.epn;
  } else if (EP.ok && P.ecand_bytes) {
    // the layout of panel_bytes: data panel(s), then the norm panel
    const size_t one = al256((size_t)EP.r_pad * EP.d_pad * EP.elem);
    epb = base + P.o_ecand;
    epb_lo = EP.fmt == 2 ? base + P.o_ecand + one : nullptr;
    epn = base + P.o_ecand + (EP.fmt == 2 ? 2 * one : one);
    if (hook) hook(hook_ctx, "tc_escalate", true, st, 0);
    tc_pack<<<tc_pack_grid(C.r_pad), 256, 0, st>>>(EP.fmt, C.Xc, C.Xc2, d, EP.d_pad, C.nrows_c,
                                              C.cidx, C.nc, C.r_pad, C.mu, C.mu2, 1, epb,
                                              epb_lo, nullptr, nullptr, nullptr, nullptr,
                                              status, nullptr, nullptr,
                                              reinterpret_cast<int *>(base + P.o_fbc), 0, epn);
    e = cudaGetLastError();
    if (hook) hook(hook_ctx, "tc_escalate", false, st, 1);
    if (e != cudaSuccess) return e;
  }
  if (!epb) return tc_brute(P, C, d, k, Xq, Xq2, qidx, D, I, ldD, base, st, hook, hook_ctx);
  TcCand C2 = C;
  C2.fmt = EP.fmt;
  C2.elem = EP.elem;
  C2.d_pad = EP.d_pad;
  C2.pb = epb;
  C2.pb_lo = epb_lo;
  C2.pn = epn;
  char *ebase = base + P.o_esc;
  e = tc_pass(EP, C2, epb, epb_lo, epn, nq, d, k, Xq, Xq2, nrows_q, qidx,
              reinterpret_cast<const int *>(base + P.o_fbc),
              reinterpret_cast<const int *>(base + P.o_fbl), D, I, ldD, ebase, status, nullptr,
              0, nullptr, st, hook, hook_ctx, true);
  if (e != cudaSuccess) return e;
  return tc_brute(EP, C2, d, k, Xq, Xq2, qidx, D, I, ldD, ebase, st, hook, hook_ctx);
}

// Escalation panels of a prepared candidate set (kept with it, e.g. a serving engine's
// resident set): the same rows in `mode`'s format, sharing shift, norms, bounds and ids.
cudaError_t tc_cand_prepare_escalation(TcCand *C, void *mem, int mode, int *status,
                                       cudaStream_t st) {
  using namespace tc;
  const CandLayout L = cand_layout(C->nc, C->d, mode);
  if (L.r_pad != C->r_pad) return cudaErrorInvalidValue;
  char *b = static_cast<char *>(mem);
  const size_t one = al256((size_t)L.r_pad * L.d_pad * L.elem);
  C->efmt = L.fmt;
  C->epb = b;
  C->epb_lo = L.fmt == 2 ? b + one : nullptr;
  C->epn = b + (L.fmt == 2 ? 2 * one : one);
  tc_pack<<<tc_pack_grid(C->r_pad), 256, 0, st>>>(L.fmt, C->Xc, C->Xc2, C->d, L.d_pad,
                                             C->nrows_c, C->cidx, C->nc, C->r_pad, C->mu, C->mu2, 1,
                                             C->epb, C->epb_lo, nullptr, nullptr, nullptr,
                                             nullptr, status, nullptr, nullptr, nullptr, 0,
                                             C->epn);
  return cudaGetLastError();
}

// ------------------------------------------------------------------------------------------
// batching form: leaf panels
// ------------------------------------------------------------------------------------------
namespace tc {
__global__ void iota_kernel(int *a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    a[i] = (int)i;
}
}  // namespace tc

int tc_leaf_tile(int d, int k, int sms) {
  const TcPlan P = tc_plan_base(256, 256, d, k, GSKNN_TC_BF16X3, sms, false, 1);
  return P.ok ? P.N : 0;
}

TcLeafPlan tc_leaf_plan(long long npts, int rows_cap, int d, int k, int sms) {
  using namespace tc;
  TcLeafPlan L{};
  L.ok = false;
  // the tile plan: split BF16, one split, candidate tiles of N (256 where it fits)
  TcPlan P = tc_plan_base(256, 256, d, k, GSKNN_TC_BF16X3, sms, false, 1);
  if (!P.ok || npts <= 0 || rows_cap <= 0 || rows_cap % TC_M != 0) return L;
  L.rows_cap = rows_cap;
  // per-query area for rows_cap rows, one split; smaller logs than the per-call path (a leaf
  // offers at most a few thousand candidates; a full log overflows to the leaf brute force)
  P.logcap = std::max(2 * P.kp, 256);
  P.S = 1;
  P.qtiles = L.rows_cap / TC_M;
  P.q_pad = L.rows_cap;
  size_t off = 0;
  auto take = [&](size_t b) { size_t o = off; off = al256(off + b); return o; };
  const size_t R = (size_t)L.rows_cap;
  L.o_mu = take((size_t)d * 4);
  L.o_mu2 = take(8);
  L.o_cpart = take((size_t)CENTER_SLICES * d * 8 + CENTER_SLICES * 4);
  L.o_stats = take(16);
  L.o_pb = take(R * P.d_pad * 2);
  L.o_pb_lo = take(R * P.d_pad * 2);
  L.o_pn = take(R * NORM_ROW);
  L.o_cn = take(R * 4);
  L.o_cnrm = take(R * 4);
  L.o_cid = take(R * 4);
  L.o_iota = take((size_t)npts * 4);
  P.o_pa = L.o_pb;  // the query panel is the candidate panel
  P.o_pa_lo = L.o_pb_lo;
  P.o_qn = L.o_cn;
  P.o_qnrm = L.o_cnrm;
  P.o_log = take((size_t)NPART * R * P.logcap * 8);
  P.o_logcnt = take((size_t)NPART * R * 4);
  P.o_proot = take((size_t)NPART * R * 4);
  P.o_margin = take(R * 4);
  P.o_fbl = take(R * 4);
  P.o_fbc = take(16);
  P.esc_mode = 0;
  P.bytes = off;
  L.bytes = off;
  L.P = P;
  L.ok = true;
  return L;
}

int tc_leaf_tile(const TcLeafPlan &L) { return L.P.N; }

cudaError_t tc_leaf_pass(const TcLeafPlan &L, void *ws, const float *X, const float *X2,
                         long long npts, int d, int k, const int *pidx, int rows,
                         const int4 *qtab, int nqt, const int2 *rtab, float *D, int *I,
                         int ldD, int *status, cudaStream_t st, bool setup,
                         unsigned long long *counters) {
  using namespace tc;
  const TcPlan &P = L.P;
  if (!L.ok || rows > L.rows_cap || rows % P.N != 0 || k > 256) return cudaErrorInvalidValue;
  if (nqt == 0) return cudaSuccess;
  char *base = static_cast<char *>(ws);
  float *mu = reinterpret_cast<float *>(base + L.o_mu);
  double *mu2 = reinterpret_cast<double *>(base + L.o_mu2);
  unsigned *stats = reinterpret_cast<unsigned *>(base + L.o_stats);
  void *pb = base + L.o_pb, *pb_lo = base + L.o_pb_lo, *pn = base + L.o_pn;
  float *cn = reinterpret_cast<float *>(base + L.o_cn);
  float *cnrm = reinterpret_cast<float *>(base + L.o_cnrm);
  uint32_t *cid = reinterpret_cast<uint32_t *>(base + L.o_cid);
  int *iota = reinterpret_cast<int *>(base + L.o_iota);
  int *fbc = reinterpret_cast<int *>(base + P.o_fbc);
  cudaError_t e = cudaMemsetAsync(stats, 0, 16, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(fbc, 0, 16, st);
  if (e == cudaSuccess) e = cudaMemsetAsync(base + P.o_proot, 0xFF, (size_t)NPART * rows * 4, st);
  if (e != cudaSuccess) return e;
  if (setup) {
    // once per workspace: the row index map, and the shift (mean of a strided sample of the
    // first panel's rows, padding skipped), which serves every later tree of the same table
    iota_kernel<<<296, 256, 0, st>>>(iota, npts);
    double *part = reinterpret_cast<double *>(base + L.o_cpart);
    int *part_n = reinterpret_cast<int *>(base + L.o_cpart + (size_t)CENTER_SLICES * d * 8);
    tc_center<<<dim3((d + 31) / 32, CENTER_SLICES), 1024, 0, st>>>(
        X, d, npts, pidx, rows, std::min(rows, 4096), part, part_n);
    tc_center_fin<<<1, 256, 0, st>>>(part, part_n, d, mu, mu2);
  }
  tc_pack<<<tc_pack_grid(rows), 256, 0, st>>>(2, X, X2, d, P.d_pad, npts, pidx, rows, rows, mu, mu2,
                                         1, pb, pb_lo, cn, cnrm, cid, stats, status, nullptr,
                                         nullptr, nullptr, 1, pn);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  CUtensorMap mA, mAlo, mB, mBlo;
  e = make_panel_map(&mA, pb, P.elem, P.d_pad, rows, TC_M);
  if (e == cudaSuccess) e = make_panel_map(&mAlo, pb_lo, P.elem, P.d_pad, rows, TC_M);
  if (e == cudaSuccess) e = make_panel_map(&mB, pb, P.elem, P.d_pad, rows, P.N);
  if (e == cudaSuccess) e = make_panel_map(&mBlo, pb_lo, P.elem, P.d_pad, rows, P.N);
  if (e != cudaSuccess) return e;
  TcParams tp{};
  tp.Q = rows; tp.k = k; tp.nkc = P.nkc; tp.ntiles_r = rows / P.N;
  tp.N = P.N; tp.NST = P.NST; tp.logcap = P.logcap;
  tp.a_terms = P.a_terms; tp.b_terms = P.b_terms; tp.fmt = P.fmt;
  tp.idesc = idesc_f32acc(1u, TC_M, P.N);
  tp.cn = cn; tp.cid = cid; tp.qn = cn; tp.qnrm = cnrm; tp.stats = stats;
  tp.Din = D; tp.ldD = ldD;
  tp.log = reinterpret_cast<uint2 *>(base + P.o_log);
  tp.logcnt = reinterpret_cast<int *>(base + P.o_logcnt);
  tp.proot = reinterpret_cast<unsigned *>(base + P.o_proot);
  tp.hk = P.hk;
  tp.W = tc_window(P.S);
  tp.S = P.S;
  tp.margin = reinterpret_cast<float *>(base + P.o_margin);
  tp.status = status;
  tp.rowmap = pidx;
  tp.qtab = qtab;
  tp.counters = counters;
  e = launch_tc_knn(P, pn, rows, nqt, mA, mAlo, mB, mBlo, tp, st);
  if (e != cudaSuccess) return e;
  RerankParams rp{};
  rp.Q = rows; rp.k = k; rp.S = NPART; rp.logcap = P.logcap; rp.d = d;
  rp.log = tp.log; rp.logcnt = tp.logcnt; rp.margin = tp.margin;
  rp.proot = tp.proot;
  rp.Xq = X; rp.Xq2 = X2; rp.Xc = X; rp.Xc2 = X2; rp.qidx = iota; rp.cid = cid;
  rp.D = D; rp.I = I; rp.ldD = ldD;
  rp.fallback_list = reinterpret_cast<int *>(base + P.o_fbl);
  rp.fallback_count = fbc;
  rp.rowmap = pidx;
  rp.dedup = 1;
  rp.counters = counters;
  LeafFallbackParams fp{};
  fp.k = k; fp.d = d; fp.N = P.N; fp.X = X; fp.X2 = X2; fp.rowmap = pidx; fp.ids = cid;
  fp.rtab = rtab; fp.D = D; fp.I = I; fp.ldD = ldD; fp.list = rp.fallback_list;
  fp.count = fbc;
  const int rb = (rows + 7) / 8;
  switch (P.kp) {
    case 32:
      tc_rerank_leaf<1><<<rb, 256, 0, st>>>(rp);
      tc_fallback_leaf<1><<<148, 256, 0, st>>>(fp);
      break;
    case 64:
      tc_rerank_leaf<2><<<rb, 256, 0, st>>>(rp);
      tc_fallback_leaf<2><<<148, 256, 0, st>>>(fp);
      break;
    case 128:
      tc_rerank_leaf<4><<<rb, 256, 0, st>>>(rp);
      tc_fallback_leaf<4><<<148, 256, 0, st>>>(fp);
      break;
    case 256:
      tc_rerank_leaf<8><<<rb, 256, 0, st>>>(rp);
      tc_fallback_leaf<8><<<148, 256, 0, st>>>(fp);
      break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace gsknn
