// knn_common.cuh -- device helpers shared by the fused kNN kernels.
//
// Selection keys are (distance, index) pairs ordered lexicographically with the index compared
// as unsigned: among equal distances the lower point id wins and the -1 sentinel (0xFFFFFFFF)
// loses to every real point. This is the deterministic tie rule of the library; the reference
// heaps (frame/gsknn_heap.c:104-162) give exact ties to the later candidate instead, so results
// agree with the reference as index sets modulo exact ties at the k-th boundary.
//
// Sorted lists live across the 32 lanes of a warp: a list of N = 32*E keys is held as E
// registers per lane, element i at (register i/32, lane i%32). Bitonic networks use register
// swaps for strides >= 32 and warp shuffles below.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace gsknn {

constexpr unsigned FULL_MASK = 0xffffffffu;
constexpr uint32_t NO_ID = 0xffffffffu;  // the -1 sentinel of the reference heaps

template <typename T> struct Num;
template <> struct Num<float> {
  __host__ __device__ static constexpr float inf() { return __builtin_huge_valf(); }
  __host__ __device__ static float nan() { return __builtin_nanf(""); }
};
template <> struct Num<double> {
  __host__ __device__ static constexpr double inf() { return __builtin_huge_val(); }
  __host__ __device__ static double nan() { return __builtin_nan(""); }
};

template <typename T>
__device__ __forceinline__ bool key_less(T da, uint32_t ia, T db, uint32_t ib) {
  return da < db || (da == db && ia < ib);
}

// Squared distance from the accumulated dot product: (-2<q,c> + |c|^2) + |q|^2, clamped at 0
// as the reference's AVX double micro-kernel does (rnn_r_int_d8x4_row.c:373-382). A NaN (an
// invalid padding candidate carries a NaN norm) stays NaN and never passes a `<=` filter.
__device__ __forceinline__ float sq_dist(float dot, float cn, float qn) {
  float v = fmaf(-2.0f, dot, cn) + qn;
  return v < 0.0f ? 0.0f : v;
}
__device__ __forceinline__ double sq_dist(double dot, double cn, double qn) {
  double v = fma(-2.0, dot, cn) + qn;
  return v < 0.0 ? 0.0 : v;
}

// Packed FP32 pair FMA of sm_100: (d0, d1) = (a0 * m + c0, a1 * m + c1), each lane rounded to
// nearest exactly as fmaf, in one instruction.
__device__ __forceinline__ void fma_pair(float &d0, float &d1, float a0, float a1, float m,
                                         float c0, float c1) {
  asm("{\n\t.reg .b64 ra, rm, rc, rd;\n\t"
      "mov.b64 ra, {%2, %3};\n\t"
      "mov.b64 rm, {%4, %4};\n\t"
      "mov.b64 rc, {%5, %6};\n\t"
      "fma.rn.f32x2 rd, ra, rm, rc;\n\t"
      "mov.b64 {%0, %1}, rd;\n\t}\n"
      : "=f"(d0), "=f"(d1)
      : "f"(a0), "f"(a1), "f"(m), "f"(c0), "f"(c1));
}

// |a - b| of the 1-norm distance (the reference's AVX kernel masks the sign bit of a - b)
__device__ __forceinline__ float abs_diff(float a, float b) { return fabsf(a - b); }
__device__ __forceinline__ double abs_diff(double a, double b) { return fabs(a - b); }

template <typename T>
__device__ __forceinline__ void swap_key(T &da, uint32_t &ia, T &db, uint32_t &ib) {
  T td = da; da = db; db = td;
  uint32_t ti = ia; ia = ib; ib = ti;
}

// Compare-exchange of two register-held elements at indices i0 < i1.
template <typename T>
__device__ __forceinline__ void cx_reg(T &d0, uint32_t &i0, T &d1, uint32_t &i1, bool asc) {
  bool sw = asc ? key_less(d1, i1, d0, i0) : key_less(d0, i0, d1, i1);
  if (sw) swap_key(d0, i0, d1, i1);
}

// Compare-exchange with the partner lane (lane ^ stride) for one register.
template <typename T>
__device__ __forceinline__ void cx_shfl(T &d, uint32_t &id, int stride, bool asc, int lane) {
  T od = __shfl_xor_sync(FULL_MASK, d, stride);
  uint32_t oi = __shfl_xor_sync(FULL_MASK, id, stride);
  bool lower = (lane & stride) == 0;
  bool take;
  if (lower == asc) take = key_less(od, oi, d, id);  // keep the smaller
  else take = key_less(d, id, od, oi);               // keep the larger
  if (take) { d = od; id = oi; }
}

// Full bitonic sort, ascending, of N = 32*E keys held by the warp.
template <typename T, int E>
__device__ __forceinline__ void warp_sort(T (&d)[E], uint32_t (&id)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
    for (int stride = size >> 1; stride > 0; stride >>= 1) {
      if (stride >= 32) {
        const int es = stride >> 5;
#pragma unroll
        for (int e = 0; e < E; e++) {
          if ((e & es) == 0) {
            const bool asc = (((e << 5) & size) == 0);
            cx_reg(d[e], id[e], d[e | es], id[e | es], asc);
          }
        }
      } else {
#pragma unroll
        for (int e = 0; e < E; e++) {
          const bool asc = ((((e << 5) + lane) & size) == 0);
          cx_shfl(d[e], id[e], stride, asc, lane);
        }
      }
    }
  }
}

// Bitonic merge of a bitonic sequence of N = 32*E keys into ascending order.
template <typename T, int E>
__device__ __forceinline__ void warp_bitonic_merge(T (&d)[E], uint32_t (&id)[E], int lane) {
  constexpr int N = 32 * E;
#pragma unroll
  for (int stride = N >> 1; stride > 0; stride >>= 1) {
    if (stride >= 32) {
      const int es = stride >> 5;
#pragma unroll
      for (int e = 0; e < E; e++)
        if ((e & es) == 0) cx_reg(d[e], id[e], d[e | es], id[e | es], true);
    } else {
#pragma unroll
      for (int e = 0; e < E; e++) cx_shfl(d[e], id[e], stride, true, lane);
    }
  }
}

// L <- the N smallest of (L U B), both ascending lists of N = 32*E keys, result ascending.
template <typename T, int E>
__device__ __forceinline__ void warp_merge_lists(T (&ld)[E], uint32_t (&li)[E],
                                                 const T (&bd)[E], const uint32_t (&bi)[E],
                                                 int lane) {
#pragma unroll
  for (int e = 0; e < E; e++) {
    // partner of index i = e*32+lane is N-1-i = (E-1-e)*32 + (31-lane)
    T od = __shfl_sync(FULL_MASK, bd[E - 1 - e], 31 - lane);
    uint32_t oi = __shfl_sync(FULL_MASK, bi[E - 1 - e], 31 - lane);
    if (key_less(od, oi, ld[e], li[e])) { ld[e] = od; li[e] = oi; }
  }
  warp_bitonic_merge<T, E>(ld, li, lane);
}

// L <- the N smallest of (L U B) where B is one ascending register of 32 keys.
template <typename T, int E>
__device__ __forceinline__ void warp_merge_32(T (&ld)[E], uint32_t (&li)[E], T bd, uint32_t bi,
                                              int lane) {
  T od = __shfl_sync(FULL_MASK, bd, 31 - lane);
  uint32_t oi = __shfl_sync(FULL_MASK, bi, 31 - lane);
  if (key_less(od, oi, ld[E - 1], li[E - 1])) { ld[E - 1] = od; li[E - 1] = oi; }
  warp_bitonic_merge<T, E>(ld, li, lane);
}

// ----------------------------------------------------------------------------------------
// cp.async (16-byte global -> shared copies, Ampere-style groups; no waits that can hang).
// ----------------------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(smem_u32(smem)), "l"(gmem)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

}  // namespace gsknn
