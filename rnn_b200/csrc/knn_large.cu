// knn_large.cu -- the explicit-distance path: a distance block in HBM followed by a per-row
// selection. It serves
//   * dgssq2nrm (frame/gsknn.c:481-594): the distance block itself, -2<a,b> + |a|^2 + |b|^2,
//     no clamp, C[j*ldc + i];
//   * dgsknn_var3 (frame/gsknn.c:597-659): k > KNN_VAR_THRES with 4-ary heaps and a 3-slot
//     header (kernels/x86_64/sandybridge/gsknn_heapselect_int_d4.c): while the row is not full
//     every candidate enters; once full the k smallest stay;
//   * the reference-algorithm entry points sgsknn_ref / dgsknn_ref (frame/gsknn_ref.c), which
//     run this unfused path, and every call whose k is beyond the fused kernels' lists.
//
// dist_block: 64 x 64 tiles of (query, candidate) over the k-major panels of pack_panels, a
// 4 x 4 register block per thread on the FP32/FP64 pipes.
// select_rows: one CTA per heap row; the exact k-th smallest (distance, id) key of the row's
// candidates and incoming entries by an MSB-first radix select (8-bit digits), the keys below it
// gathered and bitonic-sorted in shared memory, written back in descending order (a valid
// binary heap, and a valid 4-ary heap forest over the filled region).
#include "gsknn.h"
#include "knn_common.cuh"
#include "knn_internal.h"

#include <algorithm>

namespace gsknn {

constexpr int LB_T = 64;   // tile edge (queries and candidates)
constexpr int LB_DK = 16;  // dimension chunk of the panels
constexpr int SEL_THREADS = 512;

// ------------------------------------------------------------------------------------------
// distance block
// ------------------------------------------------------------------------------------------
// METRIC 0: squared 2-norm -2<a,b> + |b|^2 + |a|^2 (clamped at 0 when `clamp`); METRIC 1: the
// 1-norm, sum over p in dimension order of |a_p - b_p|.
template <typename T, int METRIC>
__global__ void __launch_bounds__(256) dist_block(const T *__restrict__ Ap, const T *__restrict__ Bp,
                                                  const T *__restrict__ qn,
                                                  const T *__restrict__ cn, int nkc, int Q, int R,
                                                  int q0, T *__restrict__ C, long long ldc,
                                                  int clamp) {
  __shared__ __align__(16) T sA[LB_DK][LB_T];
  __shared__ __align__(16) T sB[LB_DK][LB_T];
  const int ct = blockIdx.x, qt = blockIdx.y;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  T acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int j = 0; j < 4; j++) acc[i][j] = T(0);
  for (int kc = 0; kc < nkc; kc++) {
    const T *ga = Ap + ((size_t)(qt * nkc + kc) * LB_DK) * LB_T;
    const T *gb = Bp + ((size_t)(ct * nkc + kc) * LB_DK) * LB_T;
    for (int e = threadIdx.x; e < LB_DK * LB_T; e += 256) {
      (&sA[0][0])[e] = ga[e];
      (&sB[0][0])[e] = gb[e];
    }
    __syncthreads();
#pragma unroll
    for (int p = 0; p < LB_DK; p++) {
      T a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; i++) a[i] = sA[p][ty * 4 + i];
#pragma unroll
      for (int j = 0; j < 4; j++) b[j] = sB[p][tx * 4 + j];
#pragma unroll
      for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
          if constexpr (METRIC == 1) acc[i][j] += abs_diff(a[i], b[j]);
          else acc[i][j] = fma(a[i], b[j], acc[i][j]);
        }
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < 4; i++) {
    const int q = qt * LB_T + ty * 4 + i;
    if (q >= Q) continue;
#pragma unroll
    for (int j = 0; j < 4; j++) {
      const int c = ct * LB_T + tx * 4 + j;
      if (c >= R) continue;
      T v = acc[i][j];
      if constexpr (METRIC == 0) {
        v = fma(T(-2), v, cn[c]) + qn[q];
        if (clamp && v < T(0)) v = T(0);
      }
      C[(size_t)(q - q0) * ldc + c] = v;
    }
  }
}

// ------------------------------------------------------------------------------------------
// per-row selection
// ------------------------------------------------------------------------------------------
// Order-preserving unsigned images of the distance (negative values and NaN included; NaN
// sorts last).
__device__ __forceinline__ unsigned long long ord_bits(double x) {
  if (x != x) return ~0ull;
  const unsigned long long b = (unsigned long long)__double_as_longlong(x);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ unsigned long long ord_bits(float x) {
  if (x != x) return 0xFFFFFFFFull;
  const unsigned b = __float_as_uint(x);
  return (unsigned long long)((b >> 31) ? ~b : (b | 0x80000000u));
}

template <typename T> struct KeyDigits;
template <> struct KeyDigits<double> { static constexpr int DIST = 8; };  // 8-bit digits
template <> struct KeyDigits<float> { static constexpr int DIST = 4; };

// digit `d` (0 = most significant) of the key (dist image, id)
template <typename T>
__device__ __forceinline__ unsigned key_digit(unsigned long long dimg, uint32_t id, int dgt) {
  constexpr int DD = KeyDigits<T>::DIST;
  if (dgt < DD) return (unsigned)(dimg >> (8 * (DD - 1 - dgt))) & 0xFFu;
  return (id >> (8 * (3 - (dgt - DD)))) & 0xFFu;
}

template <typename T>
struct SelArgs {
  const T *C;             // distance block rows (row r = heap row j0 + r), candidates by column
  long long ldc;
  const uint32_t *cid;    // candidate ids by column (NO_ID for padding)
  int m;                  // candidates
  int j0;                 // first heap row of the block
  T *D;                   // heap storage
  int *I;
  int ldD;
  int k;
  int four_ary;           // 1: header layout (D/I offset 3, filled count in I[1])
};

template <typename T>
__global__ void __launch_bounds__(SEL_THREADS) select_rows(SelArgs<T> a) {
  extern __shared__ __align__(16) unsigned char sm[];
  __shared__ unsigned hist[256];
  __shared__ unsigned s_digit[16];
  __shared__ int s_rem, s_nless, s_neq;
  const int r = blockIdx.x;
  const int j = a.j0 + r;
  const int tid = threadIdx.x;
  const T *crow = a.C + (size_t)r * a.ldc;
  T *Drow = a.D + (size_t)j * a.ldD;
  int *Irow = a.I + (size_t)j * a.ldD;
  const int off = a.four_ary ? KNN_HEAP_OFFSET : 0;
  const int k = a.k;
  // existing entries: the whole row (binary) or the filled tail [k - filled, k) (4-ary)
  int filled = k, e_begin = 0;
  if (a.four_ary) {
    filled = Irow[1];
    filled = filled < 0 ? 0 : (filled > k ? k : filled);
    e_begin = k - filled;
  }
  const int nE = k - e_begin;
  const int n_el = nE + a.m;
  const int kout = n_el < k ? n_el : k;
  // element e: e < nE -> existing entry e_begin + e; else candidate column e - nE
  auto fetch = [&](int e, T &dist, uint32_t &id) {
    if (e < nE) {
      dist = Drow[off + e_begin + e];
      id = (uint32_t)Irow[off + e_begin + e];
    } else {
      const int c = e - nE;
      dist = crow[c];
      id = a.cid[c];
    }
  };

  constexpr int NDIG = KeyDigits<T>::DIST + 4;
  // ---- radix select of the kout-th smallest key (skipped when everything is kept)
  if (tid == 0) s_rem = kout;
  if (kout < n_el) {
    for (int dgt = 0; dgt < NDIG; dgt++) {
      for (int b = tid; b < 256; b += SEL_THREADS) hist[b] = 0;
      __syncthreads();
      for (int e = tid; e < n_el; e += SEL_THREADS) {
        T dist;
        uint32_t id;
        fetch(e, dist, id);
        const unsigned long long im = ord_bits(dist);
        bool match = true;
        for (int q = 0; q < dgt; q++)
          if (key_digit<T>(im, id, q) != s_digit[q]) { match = false; break; }
        if (match) atomicAdd(&hist[key_digit<T>(im, id, dgt)], 1u);
      }
      __syncthreads();
      if (tid == 0) {
        unsigned cum = 0, rem = (unsigned)s_rem;
        int b = 0;
        for (; b < 256; b++) {
          if (cum + hist[b] >= rem) break;
          cum += hist[b];
        }
        s_digit[dgt] = (unsigned)b;
        s_rem = (int)(rem - cum);
      }
      __syncthreads();
    }
  }
  // ---- gather: keys below the k-th, then s_rem of the keys equal to it
  T *sd = reinterpret_cast<T *>(sm);
  int kp = 1;
  while (kp < kout) kp <<= 1;
  uint32_t *si = reinterpret_cast<uint32_t *>(sm + (size_t)kp * sizeof(T));
  if (tid == 0) { s_nless = 0; s_neq = 0; }
  __syncthreads();
  const int rem = s_rem;
  for (int e = tid; e < n_el; e += SEL_THREADS) {
    T dist;
    uint32_t id;
    fetch(e, dist, id);
    int cmp = -1;  // -1 below, 0 equal, 1 above the selected key
    if (kout < n_el) {
      const unsigned long long im = ord_bits(dist);
      cmp = 0;
      for (int q = 0; q < NDIG; q++) {
        const unsigned dg = key_digit<T>(im, id, q);
        if (dg != s_digit[q]) { cmp = dg < s_digit[q] ? -1 : 1; break; }
      }
    }
    int slot = -1;
    if (cmp < 0) {
      slot = atomicAdd(&s_nless, 1);
    } else if (cmp == 0) {
      const int t = atomicAdd(&s_neq, 1);
      if (t < rem) slot = kout - rem + t;
    }
    if (slot >= 0) {
      sd[slot] = dist;
      si[slot] = id;
    }
  }
  for (int e = kout + tid; e < kp; e += SEL_THREADS) {
    sd[e] = Num<T>::inf();
    si[e] = NO_ID;
  }
  __syncthreads();
  // ---- bitonic sort ascending by (dist image, id)
  for (int size = 2; size <= kp; size <<= 1) {
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      for (int t = tid; t < kp / 2; t += SEL_THREADS) {
        const int lo = 2 * t - (t & (stride - 1));
        const int hi = lo + stride;
        const bool asc = (lo & size) == 0;
        const unsigned long long ia = ord_bits(sd[lo]), ib = ord_bits(sd[hi]);
        const bool less_hi = ib < ia || (ib == ia && si[hi] < si[lo]);
        if (less_hi == asc) {
          const T td = sd[lo]; sd[lo] = sd[hi]; sd[hi] = td;
          const uint32_t ti = si[lo]; si[lo] = si[hi]; si[hi] = ti;
        }
      }
      __syncthreads();
    }
  }
  // ---- write back in descending order into the tail [k - kout, k) of the row
  for (int t = tid; t < kout; t += SEL_THREADS) {
    const int pos = off + (k - kout) + t;
    Drow[pos] = sd[kout - 1 - t];
    Irow[pos] = (int)si[kout - 1 - t];
  }
  if (a.four_ary && tid == 0) Irow[1] = kout;
}

// ------------------------------------------------------------------------------------------
// host side
// ------------------------------------------------------------------------------------------
size_t large_select_smem(int k, size_t elem) {
  int kp = 1;
  while (kp < k) kp <<= 1;
  return (size_t)kp * (elem + 4);
}

template <typename T>
LargePlan large_plan(int nq, int nc, int d, int k, size_t max_block_bytes) {
  LargePlan P{};
  P.nkc = (d + LB_DK - 1) / LB_DK;
  P.qtiles = (nq + LB_T - 1) / LB_T;
  P.rtiles = (nc + LB_T - 1) / LB_T;
  const size_t per_row = (size_t)nc * sizeof(T);
  long long rows = (long long)(max_block_bytes / std::max(per_row, (size_t)1));
  rows = std::max<long long>(LB_T, (rows / LB_T) * LB_T);
  P.chunk_rows = (int)std::min<long long>(rows, (long long)P.qtiles * LB_T);
  size_t off = 0;
  auto al = [](size_t x) { return (x + 255) & ~(size_t)255; };
  auto take = [&](size_t b) { size_t o = off; off = al(off + b); return o; };
  P.o_ap = take((size_t)P.qtiles * P.nkc * LB_DK * LB_T * sizeof(T));
  P.o_bp = take((size_t)P.rtiles * P.nkc * LB_DK * LB_T * sizeof(T));
  P.o_qn = take((size_t)P.qtiles * LB_T * sizeof(T));
  P.o_cn = take((size_t)P.rtiles * LB_T * sizeof(T));
  P.o_cid = take((size_t)P.rtiles * LB_T * 4);
  P.o_c = take((size_t)P.chunk_rows * nc * sizeof(T));
  P.bytes = off;
  P.sel_smem = large_select_smem(k, sizeof(T));
  return P;
}

template <typename T>
cudaError_t large_run(const LargePlan &P, int nq, int nc, int d, int k, const T *Xq,
                      const T *Xq2, long long nrows_q, const int *qidx, const T *Xc,
                      const T *Xc2, long long nrows_c, const int *cidx, T *D, int *I, int ldD,
                      int four_ary, void *ws, int *status, cudaStream_t st, int metric) {
  char *base = static_cast<char *>(ws);
  T *Ap = reinterpret_cast<T *>(base + P.o_ap);
  T *Bp = reinterpret_cast<T *>(base + P.o_bp);
  T *qn = reinterpret_cast<T *>(base + P.o_qn);
  T *cn = reinterpret_cast<T *>(base + P.o_cn);
  uint32_t *cid = reinterpret_cast<uint32_t *>(base + P.o_cid);
  T *C = reinterpret_cast<T *>(base + P.o_c);
  cudaError_t e = launch_pack<T>(Xq, metric == 1 ? nullptr : Xq2, d, nrows_q, qidx, nq, LB_T,
                                 LB_DK, P.nkc, Ap, qn, nullptr, status, st);
  if (e == cudaSuccess)
    e = launch_pack<T>(Xc, metric == 1 ? nullptr : Xc2, d, nrows_c, cidx, nc, LB_T, LB_DK,
                       P.nkc, Bp, cn, cid, status, st);
  if (e != cudaSuccess) return e;
  if (P.sel_smem > 48 * 1024) {
    e = cudaFuncSetAttribute(select_rows<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)P.sel_smem);
    if (e != cudaSuccess) return e;
  }
  for (int q0 = 0; q0 < nq; q0 += P.chunk_rows) {
    const int rows = std::min(P.chunk_rows, nq - q0);
    dim3 grid(P.rtiles, (rows + LB_T - 1) / LB_T);
    // the block covers query tiles [q0 / 64, ...): offset the query panel and norms
    const T *Aq = Ap + (size_t)(q0 / LB_T) * P.nkc * LB_DK * LB_T;
    if (metric == 1)
      dist_block<T, 1><<<grid, 256, 0, st>>>(Aq, Bp, qn + q0, cn, P.nkc, rows, nc, 0, C, nc, 1);
    else
      dist_block<T, 0><<<grid, 256, 0, st>>>(Aq, Bp, qn + q0, cn, P.nkc, rows, nc, 0, C, nc, 1);
    SelArgs<T> sa{};
    sa.C = C; sa.ldc = nc; sa.cid = cid; sa.m = nc; sa.j0 = q0; sa.D = D; sa.I = I;
    sa.ldD = ldD; sa.k = k; sa.four_ary = four_ary;
    select_rows<T><<<rows, SEL_THREADS, P.sel_smem, st>>>(sa);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

// Explicit distance block C[j*ldc + i] (j < nq rows of queries, i < nc candidates), no clamp.
template <typename T>
cudaError_t block_run(const LargePlan &P, int nq, int nc, int d, const T *Xq, const T *Xq2,
                      long long nrows_q, const int *qidx, const T *Xc, const T *Xc2,
                      long long nrows_c, const int *cidx, T *Cout, long long ldc, void *ws,
                      int *status, cudaStream_t st) {
  char *base = static_cast<char *>(ws);
  T *Ap = reinterpret_cast<T *>(base + P.o_ap);
  T *Bp = reinterpret_cast<T *>(base + P.o_bp);
  T *qn = reinterpret_cast<T *>(base + P.o_qn);
  T *cn = reinterpret_cast<T *>(base + P.o_cn);
  uint32_t *cid = reinterpret_cast<uint32_t *>(base + P.o_cid);
  cudaError_t e = launch_pack<T>(Xq, Xq2, d, nrows_q, qidx, nq, LB_T, LB_DK, P.nkc, Ap, qn,
                                 nullptr, status, st);
  if (e == cudaSuccess)
    e = launch_pack<T>(Xc, Xc2, d, nrows_c, cidx, nc, LB_T, LB_DK, P.nkc, Bp, cn, cid, status, st);
  if (e != cudaSuccess) return e;
  dim3 grid(P.rtiles, P.qtiles);
  dist_block<T, 0><<<grid, 256, 0, st>>>(Ap, Bp, qn, cn, P.nkc, nq, nc, 0, Cout, ldc, 0);
  return cudaGetLastError();
}

#define GSKNN_LARGE_INST(T)                                                                     \
  template LargePlan large_plan<T>(int, int, int, int, size_t);                                 \
  template cudaError_t large_run<T>(const LargePlan &, int, int, int, int, const T *, const T *, \
                                    long long, const int *, const T *, const T *, long long,    \
                                    const int *, T *, int *, int, int, void *, int *,            \
                                    cudaStream_t, int);                                         \
  template cudaError_t block_run<T>(const LargePlan &, int, int, int, const T *, const T *,     \
                                    long long, const int *, const T *, const T *, long long,    \
                                    const int *, T *, long long, void *, int *, cudaStream_t);
GSKNN_LARGE_INST(float)
GSKNN_LARGE_INST(double)
#undef GSKNN_LARGE_INST

}  // namespace gsknn
