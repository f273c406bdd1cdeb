// knn_simt.cu -- packing, the fused CUDA-core distance + k-selection kernel, and the heap
// write-back kernel.
//
// Pipeline of one call (query = heap row = C-API beta side, candidate = C-API alpha side):
//   1. pack_panels: gather the query rows (beta) and candidate rows (alpha) of the point tables
//      into k-major panels, the B200 analogue of packA_kcxmc / packB_kcxnc
//      (frame/gsknn.c:62-185): tile t, dimension chunk c is one contiguous DK x BT block, padded
//      with zeros in d and with invalid (NaN-norm) points past the end. Norms and candidate ids
//      are gathered alongside (frame/gsknn.c:959-964, 981-986).
//   2. fused_knn_simt: one CTA owns BQ queries and streams a range of candidate tiles through a
//      cp.async ring; each thread accumulates a TM x TN block of dot products on the FP32/FP64
//      pipes (the role of rnn_r_int_d8x4_row / knn_r_ref_s8x8_row), then turns them into squared
//      distances, filters them against each query's current k-th distance (the prefilter of
//      rnn_r_int_d8x4_row.c:424-494) and appends survivors to a per-query shared-memory buffer.
//      Full buffers are merged into each query's sorted list with warp bitonic networks (the role
//      of heapSelect_d / HeapAdjust_d, frame/gsknn_heap.c:52-162). The m x n distance matrix never
//      leaves the SM.
//   3. finalize_heap: merges the per-split sorted lists with the caller's incoming heap row and
//      writes the k smallest back in place in descending order, which is a valid binary max-heap
//      with the k-th distance at the root (the in-place merge contract of dgsknn/sgsknn).
#include "knn_common.cuh"
#include "knn_internal.h"

#include <algorithm>

namespace gsknn {

// ------------------------------------------------------------------------------------------
// 1. Packing
// ------------------------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) pack_panels(
    const T *__restrict__ X, const T *__restrict__ X2, int d, long long nrows,
    const int *__restrict__ idx, int count, int BT, int DK, int nkc, T *__restrict__ P,
    T *__restrict__ norms, uint32_t *__restrict__ ids, int *__restrict__ status) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T *s = reinterpret_cast<T *>(smem_raw);  // [DK][BT + 1]
  const int tile = blockIdx.x / nkc;
  const int kc = blockIdx.x % nkc;
  const int tid = threadIdx.x;
  for (int e = tid; e < BT * DK; e += blockDim.x) {
    const int r = e / DK, p = e % DK;
    const int gr = tile * BT + r, gp = kc * DK + p;
    T v = T(0);
    if (gr < count && gp < d) {
      const long long row = idx[gr];
      if (row >= 0 && row < nrows) v = X[row * d + gp];
    }
    s[p * (BT + 1) + r] = v;
  }
  __syncthreads();
  T *dst = P + ((size_t)(tile * nkc + kc) * DK) * BT;
  for (int e = tid; e < BT * DK; e += blockDim.x) {
    const int p = e / BT, r = e % BT;
    dst[(size_t)p * BT + r] = s[p * (BT + 1) + r];
  }
  if (kc == 0) {
    for (int r = tid; r < BT; r += blockDim.x) {
      const int gr = tile * BT + r;
      T nv = Num<T>::nan();
      uint32_t id = NO_ID;
      if (gr < count) {
        const long long row = idx[gr];
        if (row >= 0 && row < nrows) {
          nv = X2[row];
          id = (uint32_t)row;
        } else {
          atomicExch(status, GSKNN_ERR_INDEX);
        }
      }
      norms[gr] = nv;
      if (ids) ids[gr] = id;
    }
  }
}

// ------------------------------------------------------------------------------------------
// 2. Fused distance + selection on the CUDA cores
// ------------------------------------------------------------------------------------------
template <typename T, int KP_, int GM, int GN, int WQ_, int WR_, int DK_, int NSTAGE_>
struct SimtCfg {
  using type = T;
  static constexpr int KP = KP_, DK = DK_, NSTAGE = NSTAGE_, WQ = WQ_, WR = WR_;
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

template <class C>
__global__ void __launch_bounds__(C::NTHR) fused_knn_simt(SimtArgs<typename C::type> a) {
  using T = typename C::type;
  extern __shared__ __align__(128) unsigned char smem[];
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
  const int qt = blockIdx.x, split = blockIdx.y;
  const int q0 = qt * C::BQ;
  const int k = a.k;

  // candidate tile range of this split
  const int t_begin = split * a.tiles_per_split;
  int t_end = t_begin + a.tiles_per_split;
  if (t_end > a.ntiles_r) t_end = a.ntiles_r;
  const int ntile = t_end > t_begin ? t_end - t_begin : 0;
  const int total = ntile * a.nkc;

  // ---- init lists, buffers, thresholds
  for (int e = tid; e < C::BQ * C::KP; e += C::NTHR) {
    Ld[e] = Num<T>::inf();
    Li[e] = NO_ID;
  }
  for (int q = tid; q < C::BQ; q += C::NTHR) {
    const int gq = q0 + q;
    cnt[q] = 0;
    T t = Num<T>::inf();
    if (gq >= a.Q) {
      t = -Num<T>::inf();
    } else if (a.Din) {
      // the incoming heap already holds k entries, so nothing above its largest can enter
      T mx = -Num<T>::inf();
      const T *row = a.Din + (size_t)gq * a.ldD;
      for (int j = 0; j < k; j++) {
        T v = row[j];
        if (v > mx) mx = v;
      }
      if (mx > -Num<T>::inf()) t = mx;
    }
    thr[q] = t;
    qn_s[q] = a.qn[q0 + q];
  }

  // ---- producer: cp.async of one (candidate tile, dim chunk) pair of panels into a slot
  const T *Apan = a.Apack + (size_t)qt * a.nkc * C::DK * C::BQ;
  auto issue = [&](int c, int slot) {
    const int tile = t_begin + c / a.nkc, kc = c % a.nkc;
    T *sA = reinterpret_cast<T *>(smem + slot * C::STAGE);
    T *sB = sA + C::DK * C::BQ;
    const T *gA = Apan + (size_t)kc * C::DK * C::BQ;
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
      for (int i = 0; i < C::TM; i++)
#pragma unroll
        for (int j = 0; j < C::TN; j++) acc[i][j] = fma(av[i], bv[j], acc[i][j]);
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
        const T dv = sq_dist(acc[i][j], cn_r[j], qn_r[i]);
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

  // ---- write this split's sorted list (first k entries) for every valid query
  for (int e = tid; e < C::BQ * k; e += C::NTHR) {
    const int q = e / k, t = e % k;
    const int gq = q0 + q;
    if (gq < a.Q) {
      const size_t o = ((size_t)split * a.Q + gq) * k + t;
      a.partD[o] = Ld[q * C::KP + t];
      a.partI[o] = Li[q * C::KP + t];
    }
  }
}

// ------------------------------------------------------------------------------------------
// 3. Merge split lists with the incoming heap; write a descending (max-heap) row.
// ------------------------------------------------------------------------------------------
template <typename T, int E>
__global__ void __launch_bounds__(256) finalize_heap(FinalizeArgs<T> a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int q = blockIdx.x * 8 + warp;
  if (q >= a.Q) return;
  const int k = a.k;
  T ld[E];
  uint32_t li[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (a.Din && t < k) {
      ld[e] = a.Din[(size_t)q * a.ldD + t];
      li[e] = (uint32_t)a.Iin[(size_t)q * a.ldD + t];
    } else {
      ld[e] = Num<T>::inf();
      li[e] = NO_ID;
    }
  }
  warp_sort<T, E>(ld, li, lane);
  for (int s = 0; s < a.S; s++) {
    T bd[E];
    uint32_t bi[E];
    const size_t base = ((size_t)s * a.Q + q) * k;
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int t = e * 32 + lane;
      bd[e] = t < k ? a.partD[base + t] : Num<T>::inf();
      bi[e] = t < k ? a.partI[base + t] : NO_ID;
    }
    warp_merge_lists<T, E>(ld, li, bd, bi, lane);
  }
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int t = e * 32 + lane;
    if (t < k) {
      a.Dout[(size_t)q * a.ldD + (k - 1 - t)] = ld[e];
      a.Iout[(size_t)q * a.ldD + (k - 1 - t)] = (int)li[e];
    }
  }
}

// ------------------------------------------------------------------------------------------
// Host-side launchers
// ------------------------------------------------------------------------------------------
template <typename T>
cudaError_t launch_pack(const T *X, const T *X2, int d, long long nrows, const int *idx,
                        int count, int BT, int DK, int nkc, T *P, T *norms, uint32_t *ids,
                        int *status, cudaStream_t st) {
  const int ntiles = (count + BT - 1) / BT;
  if (ntiles == 0) return cudaSuccess;
  const size_t sm = (size_t)DK * (BT + 1) * sizeof(T);
  pack_panels<T><<<ntiles * nkc, 256, sm, st>>>(X, X2, d, nrows, idx, count, BT, DK, nkc, P,
                                                norms, ids, status);
  return cudaGetLastError();
}

template <class C>
static cudaError_t run_simt(const SimtArgs<typename C::type> &a, int qtiles, int S,
                            cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(fused_knn_simt<C>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid(qtiles, S);
  fused_knn_simt<C><<<grid, C::NTHR, C::SMEM, st>>>(a);
  return cudaGetLastError();
}

// Tile configurations per (precision, list size). Float: 8x8 per thread, 128 queries x 128
// candidates per CTA (64 queries for the larger lists); double: 4x8 per thread.
template <typename T, int KP> struct SimtPick;
template <> struct SimtPick<float, 32> { using C = SimtCfg<float, 32, 2, 2, 4, 2, 16, 3>; };
template <> struct SimtPick<float, 64> { using C = SimtCfg<float, 64, 2, 2, 4, 2, 16, 3>; };
template <> struct SimtPick<float, 128> { using C = SimtCfg<float, 128, 2, 2, 2, 4, 16, 3>; };
template <> struct SimtPick<float, 256> { using C = SimtCfg<float, 256, 2, 2, 2, 4, 16, 3>; };
template <> struct SimtPick<double, 32> { using C = SimtCfg<double, 32, 1, 2, 4, 2, 16, 3>; };
template <> struct SimtPick<double, 64> { using C = SimtCfg<double, 64, 1, 2, 4, 2, 16, 3>; };
template <> struct SimtPick<double, 128> { using C = SimtCfg<double, 128, 1, 2, 4, 2, 8, 3>; };
template <> struct SimtPick<double, 256> { using C = SimtCfg<double, 256, 1, 2, 2, 4, 8, 3>; };

template <typename T>
SimtGeom simt_geometry(int k) {
  SimtGeom g{};
  int kp = 32;
  while (kp < k) kp <<= 1;
  g.kp = kp;
#define GSKNN_GEOM(KPV)                                   \
  if (kp == KPV) {                                        \
    using C = typename SimtPick<T, KPV>::C;               \
    g.bq = C::BQ; g.br = C::BR; g.dk = C::DK;             \
    g.smem = C::SMEM; g.nthr = C::NTHR;                   \
    return g;                                             \
  }
  GSKNN_GEOM(32) GSKNN_GEOM(64) GSKNN_GEOM(128) GSKNN_GEOM(256)
#undef GSKNN_GEOM
  g.kp = 0;
  return g;
}

template <typename T>
cudaError_t launch_simt(const SimtArgs<T> &a, int kp, int qtiles, int S, cudaStream_t st) {
  switch (kp) {
    case 32: return run_simt<typename SimtPick<T, 32>::C>(a, qtiles, S, st);
    case 64: return run_simt<typename SimtPick<T, 64>::C>(a, qtiles, S, st);
    case 128: return run_simt<typename SimtPick<T, 128>::C>(a, qtiles, S, st);
    case 256: return run_simt<typename SimtPick<T, 256>::C>(a, qtiles, S, st);
  }
  return cudaErrorInvalidValue;
}

template <typename T>
cudaError_t launch_finalize(const FinalizeArgs<T> &a, int kp, cudaStream_t st) {
  const int blocks = (a.Q + 7) / 8;
  if (blocks == 0) return cudaSuccess;
  switch (kp) {
    case 32: finalize_heap<T, 1><<<blocks, 256, 0, st>>>(a); break;
    case 64: finalize_heap<T, 2><<<blocks, 256, 0, st>>>(a); break;
    case 128: finalize_heap<T, 4><<<blocks, 256, 0, st>>>(a); break;
    case 256: finalize_heap<T, 8><<<blocks, 256, 0, st>>>(a); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

#define GSKNN_INST(T)                                                                       \
  template cudaError_t launch_pack<T>(const T *, const T *, int, long long, const int *, int, \
                                      int, int, int, T *, T *, uint32_t *, int *,           \
                                      cudaStream_t);                                        \
  template SimtGeom simt_geometry<T>(int);                                                  \
  template cudaError_t launch_simt<T>(const SimtArgs<T> &, int, int, int, cudaStream_t);    \
  template cudaError_t launch_finalize<T>(const FinalizeArgs<T> &, int, cudaStream_t);
GSKNN_INST(float)
GSKNN_INST(double)
#undef GSKNN_INST

}  // namespace gsknn
