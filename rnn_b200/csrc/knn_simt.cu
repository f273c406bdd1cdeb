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
#include "knn_simt_body.cuh"

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
          nv = X2 ? X2[row] : T(0);
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
// 2. Fused distance + selection on the CUDA cores: one CTA per (query tile, candidate split);
//    the tile body is simt_block (knn_simt_body.cuh)
// ------------------------------------------------------------------------------------------
template <class C, int METRIC>
__global__ void __launch_bounds__(C::NTHR, C::MINB) fused_knn_simt(SimtArgs<typename C::type> a) {
  using T = typename C::type;
  extern __shared__ __align__(128) unsigned char smem[];
  const int qt = blockIdx.x, split = blockIdx.y;
  const int q0 = qt * C::BQ;
  SimtBlock<T> b;
  b.Apan = a.Apack + (size_t)qt * a.nkc * C::DK * C::BQ;
  b.Bpack = a.Bpack;
  b.qn = a.qn + q0;
  b.cn = a.cn;
  b.cid = a.cid;
  b.nkc = a.nkc;
  b.k = a.k;
  b.t_begin = split * a.tiles_per_split;
  b.t_end = b.t_begin + a.tiles_per_split;
  if (b.t_end > a.ntiles_r) b.t_end = a.ntiles_r;
  b.nrows = a.Q - q0 < C::BQ ? a.Q - q0 : C::BQ;
  b.rowid = nullptr;
  b.row0 = q0;
  b.Din = a.Din;
  b.ldD = a.ldD;
  b.outD = a.partD;
  b.outI = a.partI;
  b.out0 = (long long)split * a.Q;
  simt_block<C, METRIC>(smem, b);
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

template <class C, int METRIC>
static cudaError_t run_simt_metric(const SimtArgs<typename C::type> &a, int qtiles, int S,
                                   cudaStream_t st) {
  cudaError_t e = cudaFuncSetAttribute(fused_knn_simt<C, METRIC>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, (int)C::SMEM);
  if (e != cudaSuccess) return e;
  dim3 grid(qtiles, S);
  fused_knn_simt<C, METRIC><<<grid, C::NTHR, C::SMEM, st>>>(a);
  return cudaGetLastError();
}

template <class C>
static cudaError_t run_simt(const SimtArgs<typename C::type> &a, int qtiles, int S,
                            cudaStream_t st) {
  return a.metric == METRIC_L1 ? run_simt_metric<C, METRIC_L1>(a, qtiles, S, st)
                               : run_simt_metric<C, METRIC_L2>(a, qtiles, S, st);
}

// Tile configurations per (precision, list size). Float: 8x8 per thread, 128 queries x 128
// candidates per CTA (64 queries for the larger lists); double: 4x8 per thread.
template <typename T, int KP> struct SimtPick;
template <> struct SimtPick<float, 32> { using C = SimtCfg<float, 32, 2, 2, 4, 2, 16, 2, 2>; };
template <> struct SimtPick<float, 64> { using C = SimtCfg<float, 64, 2, 2, 4, 2, 16, 3>; };
template <> struct SimtPick<float, 128> { using C = SimtCfg<float, 128, 2, 2, 2, 4, 16, 3>; };
template <> struct SimtPick<float, 256> { using C = SimtCfg<float, 256, 2, 2, 2, 4, 16, 3>; };
template <> struct SimtPick<double, 32> { using C = SimtCfg<double, 32, 1, 2, 4, 2, 16, 2, 2>; };
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
    g.smem = C::SMEM; g.nthr = C::NTHR; g.minb = C::MINB; \
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
