// knn_simt_body.cuh -- the CUDA-core tile body shared by the per-call kernel (fused_knn_simt,
// one CTA per query tile and candidate split) and the persistent leaf kernel of the batching
// form (batch_knn_simt, one CTA looping over work items).
//
// One block = BQ query rows of a packed panel against a range of packed candidate tiles:
// cp.async ring of (A, B) panel chunks, TM x TN register blocks of dot products on the FP32 /
// FP64 pipes (the role of rnn_r_int_d8x4_row / knn_r_ref_s8x8_row), then per candidate tile
// squared distances, the k-th-distance prefilter (rnn_r_int_d8x4_row.c:424-494), per-query
// survivor buffers in shared memory and warp bitonic merges into each query's sorted list (the
// role of heapSelect_* / HeapAdjust_*, frame/gsknn_heap.c:52-162). The block ends by writing
// the first k entries of every query's list.
#pragma once

#include <type_traits>

#include "knn_common.cuh"
#include "knn_internal.h"

namespace gsknn {

template <typename T, int KP_, int GM, int GN, int WQ_, int WR_, int DK_, int NSTAGE_,
          int MINB_ = 1>
struct SimtCfg {
  using type = T;
  static constexpr int KP = KP_, DK = DK_, NSTAGE = NSTAGE_, WQ = WQ_, WR = WR_;
  static constexpr int MINB = MINB_;  // resident CTAs per SM the launch bounds ask for
  static constexpr int TM = 4 * GM, TN = 4 * GN;
  static constexpr int WTQ = 16 * GM, WTR = 32 * GN;  // warp tile: 4 x 8 lanes
  static constexpr int BQ = WQ * WTQ, BR = WR * WTR;
  static constexpr int NWARP = WQ * WR, NTHR = 32 * NWARP;
  static constexpr int E = KP / 32;
  static constexpr int CAP = 32;  // per-query candidate buffer
  // shared memory carve-up (bytes)
  static constexpr size_t STAGE = (size_t)DK * (BQ + BR) * sizeof(T);
  static constexpr size_t OFF_LD = NSTAGE * STAGE;
  static constexpr size_t OFF_LI = OFF_LD + (size_t)BQ * KP * sizeof(T);
  static constexpr size_t OFF_BD = OFF_LI + (size_t)BQ * KP * 4;
  static constexpr size_t OFF_BI = OFF_BD + (size_t)BQ * CAP * sizeof(T);
  static constexpr size_t OFF_QN = OFF_BI + (size_t)BQ * CAP * 4;
  static constexpr size_t OFF_TH = OFF_QN + (size_t)BQ * sizeof(T);
  static constexpr size_t OFF_CNT = OFF_TH + (size_t)BQ * sizeof(T);
  static constexpr size_t SMEM = OFF_CNT + (size_t)BQ * 4;
  static_assert(TM * TN <= 64, "pending mask is 64 bits");
};

template <typename T>
__device__ __forceinline__ void load4(T (&v)[4], const T *p);
template <>
__device__ __forceinline__ void load4<float>(float (&v)[4], const float *p) {
  float4 t = *reinterpret_cast<const float4 *>(p);
  v[0] = t.x; v[1] = t.y; v[2] = t.z; v[3] = t.w;
}
template <>
__device__ __forceinline__ void load4<double>(double (&v)[4], const double *p) {
  double2 a = reinterpret_cast<const double2 *>(p)[0];
  double2 b = reinterpret_cast<const double2 *>(p)[1];
  v[0] = a.x; v[1] = a.y; v[2] = b.x; v[3] = b.y;
}

// Merge every non-empty per-query buffer into its sorted list; lower the thresholds.
template <class C>
__device__ __forceinline__ void merge_buffers(unsigned char *smem, int k, int warp, int lane) {
  using T = typename C::type;
  T *Ld = reinterpret_cast<T *>(smem + C::OFF_LD);
  uint32_t *Li = reinterpret_cast<uint32_t *>(smem + C::OFF_LI);
  T *Bd = reinterpret_cast<T *>(smem + C::OFF_BD);
  uint32_t *Bi = reinterpret_cast<uint32_t *>(smem + C::OFF_BI);
  T *thr = reinterpret_cast<T *>(smem + C::OFF_TH);
  int *cnt = reinterpret_cast<int *>(smem + C::OFF_CNT);
  for (int q = warp; q < C::BQ; q += C::NWARP) {
    int c = cnt[q];
    if (c == 0) continue;
    c = c < C::CAP ? c : C::CAP;
    T bd = lane < c ? Bd[q * C::CAP + lane] : Num<T>::inf();
    uint32_t bi = lane < c ? Bi[q * C::CAP + lane] : NO_ID;
    T b1[1] = {bd};
    uint32_t i1[1] = {bi};
    warp_sort<T, 1>(b1, i1, lane);
    T ld[C::E];
    uint32_t li[C::E];
#pragma unroll
    for (int e = 0; e < C::E; e++) {
      ld[e] = Ld[q * C::KP + e * 32 + lane];
      li[e] = Li[q * C::KP + e * 32 + lane];
    }
    warp_merge_32<T, C::E>(ld, li, b1[0], i1[0], lane);
#pragma unroll
    for (int e = 0; e < C::E; e++) {
      Ld[q * C::KP + e * 32 + lane] = ld[e];
      Li[q * C::KP + e * 32 + lane] = li[e];
    }
    // k-th smallest distance: element k-1
    T kth = ld[0];
#pragma unroll
    for (int e = 0; e < C::E; e++)
      if (e == (k - 1) / 32) kth = ld[e];
    kth = __shfl_sync(FULL_MASK, kth, (k - 1) & 31);
    if (lane == 0) {
      if (kth < thr[q]) thr[q] = kth;
      cnt[q] = 0;
    }
  }
}

// One block of work: a query tile against candidate tiles [t_begin, t_end).
template <typename T>
struct SimtBlock {
  const T *Apan;          // the query tile's panels [nkc][DK][BQ]
  const T *Bpack;         // candidate panels [tile][nkc][DK][BR]
  const T *qn;            // norms of the tile's query rows [BQ] (NaN for padding)
  const T *cn;            // candidate norms by packed candidate position (NaN for padding)
  const uint32_t *cid;    // candidate ids by packed candidate position
  int nkc, k, t_begin, t_end;
  int nrows;              // rows [0, nrows) of the tile may be queries
  const uint32_t *rowid;  // heap row of each query row [BQ] (NO_ID: padding); null: row0 + r
  long long row0;
  const T *Din;           // incoming heap rows (initial threshold), may be null
  int ldD;
  T *outD;                // sorted lists: k entries at row (out0 + heap row)
  uint32_t *outI;
  long long out0;
};

// Distance of the tile body. L2: squared 2-norm from the dot product and the norms (the
// reference's rnn_r_int_d8x4_row.c). L1: the sum of |a_p - b_p| over p in dimension order, as
// the reference's rnn_r_1norm_int_d8x4_row.c accumulates it; the packed candidate norm is used
// only as the padding flag (0 for a real candidate, NaN past the end).
constexpr int METRIC_L2 = 0;
constexpr int METRIC_L1 = 1;

template <class C, int METRIC = METRIC_L2>
__device__ __forceinline__ void simt_block(unsigned char *smem, const SimtBlock<typename C::type> &a) {
  using T = typename C::type;
  T *Ld = reinterpret_cast<T *>(smem + C::OFF_LD);
  uint32_t *Li = reinterpret_cast<uint32_t *>(smem + C::OFF_LI);
  T *Bd = reinterpret_cast<T *>(smem + C::OFF_BD);
  uint32_t *Bi = reinterpret_cast<uint32_t *>(smem + C::OFF_BI);
  T *qn_s = reinterpret_cast<T *>(smem + C::OFF_QN);
  T *thr = reinterpret_cast<T *>(smem + C::OFF_TH);
  int *cnt = reinterpret_cast<int *>(smem + C::OFF_CNT);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wq = warp / C::WR, wr = warp % C::WR;
  const int lq = lane >> 3, lr = lane & 7;
  const int k = a.k;
  const int t_begin = a.t_begin;
  const int ntile = a.t_end > t_begin ? a.t_end - t_begin : 0;
  const int total = ntile * a.nkc;
  auto heap_row = [&](int q) -> long long {
    if (q >= a.nrows) return -1;
    if (!a.rowid) return a.row0 + q;
    const uint32_t r = a.rowid[q];
    return r == NO_ID ? -1 : (long long)r;
  };

  // ---- init lists, buffers, thresholds
  for (int e = tid; e < C::BQ * C::KP; e += C::NTHR) {
    Ld[e] = Num<T>::inf();
    Li[e] = NO_ID;
  }
  for (int q = tid; q < C::BQ; q += C::NTHR) {
    const long long hr = heap_row(q);
    cnt[q] = 0;
    T t = Num<T>::inf();
    if (hr < 0) {
      t = -Num<T>::inf();
    } else if (a.Din) {
      // the incoming heap already holds k entries, so nothing above its largest can enter
      T mx = -Num<T>::inf();
      const T *row = a.Din + (size_t)hr * a.ldD;
      for (int j = 0; j < k; j++) {
        T v = row[j];
        if (v > mx) mx = v;
      }
      if (mx > -Num<T>::inf()) t = mx;
    }
    thr[q] = t;
    qn_s[q] = a.qn[q];
  }

  // ---- producer: cp.async of one (candidate tile, dim chunk) pair of panels into a slot
  auto issue = [&](int c, int slot) {
    const int tile = t_begin + c / a.nkc, kc = c % a.nkc;
    T *sA = reinterpret_cast<T *>(smem + slot * C::STAGE);
    T *sB = sA + C::DK * C::BQ;
    const T *gA = a.Apan + (size_t)kc * C::DK * C::BQ;
    const T *gB = a.Bpack + ((size_t)tile * a.nkc + kc) * C::DK * C::BR;
    constexpr int VA = C::DK * C::BQ * (int)sizeof(T) / 16;
    constexpr int VB = C::DK * C::BR * (int)sizeof(T) / 16;
    for (int v = tid; v < VA; v += C::NTHR)
      cp_async16(reinterpret_cast<char *>(sA) + 16 * v, reinterpret_cast<const char *>(gA) + 16 * v);
    for (int v = tid; v < VB; v += C::NTHR)
      cp_async16(reinterpret_cast<char *>(sB) + 16 * v, reinterpret_cast<const char *>(gB) + 16 * v);
  };

#pragma unroll
  for (int c = 0; c < C::NSTAGE - 1; c++) {
    if (c < total) issue(c, c);
    cp_async_commit();
  }
  __syncthreads();  // lists/thresholds initialised

  T acc[C::TM][C::TN];
#pragma unroll
  for (int i = 0; i < C::TM; i++)
#pragma unroll
    for (int j = 0; j < C::TN; j++) acc[i][j] = T(0);

  const int arow = wq * C::WTQ + lq * 4;  // + g*16 + t
  const int bcol = wr * C::WTR + lr * 4;  // + h*32 + u

  for (int c = 0; c < total; c++) {
    cp_async_wait<C::NSTAGE - 2>();
    __syncthreads();
    {
      const int cn = c + C::NSTAGE - 1;
      if (cn < total) issue(cn, cn % C::NSTAGE);
      cp_async_commit();
    }
    const T *sA = reinterpret_cast<const T *>(smem + (c % C::NSTAGE) * C::STAGE);
    const T *sB = sA + C::DK * C::BQ;
#pragma unroll 4
    for (int kk = 0; kk < C::DK; kk++) {
      T av[C::TM], bv[C::TN];
#pragma unroll
      for (int g = 0; g < C::TM / 4; g++) {
        T t4[4];
        load4<T>(t4, sA + kk * C::BQ + arow + g * 16);
#pragma unroll
        for (int u = 0; u < 4; u++) av[g * 4 + u] = t4[u];
      }
#pragma unroll
      for (int h = 0; h < C::TN / 4; h++) {
        T t4[4];
        load4<T>(t4, sB + kk * C::BR + bcol + h * 32);
#pragma unroll
        for (int u = 0; u < 4; u++) bv[h * 4 + u] = t4[u];
      }
#pragma unroll
      for (int i = 0; i < C::TM; i++) {
        if constexpr (METRIC == METRIC_L2 && std::is_same<T, float>::value) {
          // two candidates per instruction (packed FP32 FMA, rounded as fmaf)
#pragma unroll
          for (int j = 0; j < C::TN; j += 2)
            fma_pair(acc[i][j], acc[i][j + 1], bv[j], bv[j + 1], av[i], acc[i][j],
                     acc[i][j + 1]);
        } else {
#pragma unroll
          for (int j = 0; j < C::TN; j++) {
            if constexpr (METRIC == METRIC_L1) acc[i][j] += abs_diff(av[i], bv[j]);
            else acc[i][j] = fma(av[i], bv[j], acc[i][j]);
          }
        }
      }
    }

    if (c % a.nkc != a.nkc - 1) continue;

    // ---- end of a candidate tile: distances, filter, buffered selection
    const int tile = t_begin + c / a.nkc;
    const size_t cbase = (size_t)tile * C::BR;
    T thr_r[C::TM], qn_r[C::TM], cn_r[C::TN];
#pragma unroll
    for (int i = 0; i < C::TM; i++) {
      const int q = arow + (i / 4) * 16 + (i & 3);
      thr_r[i] = thr[q];
      qn_r[i] = qn_s[q];
    }
#pragma unroll
    for (int j = 0; j < C::TN; j++) cn_r[j] = a.cn[cbase + bcol + (j / 4) * 32 + (j & 3)];
    unsigned long long pend = 0ull;
#pragma unroll
    for (int i = 0; i < C::TM; i++)
#pragma unroll
      for (int j = 0; j < C::TN; j++) {
        // L1: adding (cn - cn) keeps a real candidate's sum exactly and makes padding NaN
        const T dv = METRIC == METRIC_L1 ? acc[i][j] + (cn_r[j] - cn_r[j])
                                         : sq_dist(acc[i][j], cn_r[j], qn_r[i]);
        acc[i][j] = dv;
        if (dv <= thr_r[i]) pend |= 1ull << (i * C::TN + j);
      }
    while (true) {
      if (pend) {
#pragma unroll
        for (int i = 0; i < C::TM; i++)
#pragma unroll
          for (int j = 0; j < C::TN; j++) {
            const unsigned long long bit = 1ull << (i * C::TN + j);
            if (pend & bit) {
              const int q = arow + (i / 4) * 16 + (i & 3);
              const int pos = atomicAdd(&cnt[q], 1);
              if (pos < C::CAP) {
                Bd[q * C::CAP + pos] = acc[i][j];
                Bi[q * C::CAP + pos] = a.cid[cbase + bcol + (j / 4) * 32 + (j & 3)];
                pend &= ~bit;
              }
            }
          }
      }
      if (!__syncthreads_or(pend != 0ull)) break;
      merge_buffers<C>(smem, k, warp, lane);
      __syncthreads();
#pragma unroll
      for (int i = 0; i < C::TM; i++) {
        const int q = arow + (i / 4) * 16 + (i & 3);
        thr_r[i] = thr[q];
      }
#pragma unroll
      for (int i = 0; i < C::TM; i++)
#pragma unroll
        for (int j = 0; j < C::TN; j++)
          if (!(acc[i][j] <= thr_r[i])) pend &= ~(1ull << (i * C::TN + j));
    }
#pragma unroll
    for (int i = 0; i < C::TM; i++)
#pragma unroll
      for (int j = 0; j < C::TN; j++) acc[i][j] = T(0);
  }
  cp_async_wait<0>();
  __syncthreads();
  merge_buffers<C>(smem, k, warp, lane);
  __syncthreads();

  // ---- write the sorted list (first k entries) of every query row
  for (int e = tid; e < C::BQ * k; e += C::NTHR) {
    const int q = e / k, t = e % k;
    const long long hr = heap_row(q);
    if (hr >= 0) {
      const size_t o = (size_t)(a.out0 + hr) * k + t;
      a.outD[o] = Ld[q * C::KP + t];
      a.outI[o] = Li[q * C::KP + t];
    }
  }
}

}  // namespace gsknn
