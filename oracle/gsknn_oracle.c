/*
 * gsknn_oracle.c -- CPU restatement of the GSKNN reference algorithm.
 *
 * TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA library in rnn_b200/. It is
 * loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline leg, never by
 * the product. Built with -ffp-contract=off semantics (no fused multiply-add) so that the
 * restated reference routines reproduce the reference's rounding bit for bit; this is
 * checked against outputs of the reference library itself (tests/golden/).
 *
 * Citations are paths inside the reference project (ChenhanYu/rnn).
 */
#include "gsknn_oracle.h"

#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int g_threads = 0;

void oracle_set_threads(int nthreads) { g_threads = nthreads; }

static int nthreads_for(long work) {
  int t = g_threads;
#ifdef _OPENMP
  if (t <= 0) t = omp_get_max_threads();
#else
  t = 1;
#endif
  if (work < 4096) t = 1;
  return t < 1 ? 1 : t;
}

/* ------------------------------------------------------------------------------------------
 * Binary max-heap (frame/gsknn_heap.c:52-96 sift-down, 104-162 select).
 * A candidate replaces the root when x <= root (ties go to the later candidate).
 * ---------------------------------------------------------------------------------------- */
#define DEFINE_SIFT(NAME, T)                                         \
  static void NAME(T *D, int s, int n, int *I) {                     \
    while (2 * s + 1 < n) {                                          \
      int j = 2 * s + 1;                                             \
      if (j + 1 < n && D[j] < D[j + 1]) j++;                         \
      if (D[s] < D[j]) {                                             \
        T td = D[s]; D[s] = D[j]; D[j] = td;                         \
        int ti = I[s]; I[s] = I[j]; I[j] = ti;                       \
        s = j;                                                       \
      } else {                                                       \
        break;                                                       \
      }                                                              \
    }                                                                \
  }
DEFINE_SIFT(sift_down_d, double)
DEFINE_SIFT(sift_down_s, float)

void oracle_heap_select_d(int m, int k, const double *x, const int *alpha, double *D, int *I) {
  for (int i = 0; i < m; i++) {
    if (x[i] > D[0]) continue;
    D[0] = x[i];
    I[0] = alpha[i];
    sift_down_d(D, 0, k, I);
  }
}

void oracle_heap_select_s(int m, int k, const float *x, const int *alpha, float *D, int *I) {
  for (int i = 0; i < m; i++) {
    if (x[i] > D[0]) continue;
    D[0] = x[i];
    I[0] = alpha[i];
    sift_down_s(D, 0, k, I);
  }
}

/* ------------------------------------------------------------------------------------------
 * dgsknn_ref / sgsknn_ref (frame/gsknn_ref.c:63-162; arithmetic of dgsknn_ref_impl.h:19-81
 * and sgsknn_ref_impl.h:19-81 without BLAS): Cs = sum_p a_p*b_p accumulated in p order in the
 * working precision, Cs *= -2, Cs += XA2[alpha[i]], Cs += XB2[beta[j]], then heapSelect per
 * query row j on D[j*k], I[j*k]. One row of Cs at a time instead of the full m x n matrix.
 * ---------------------------------------------------------------------------------------- */
void oracle_dgsknn_ref(int m, int n, int d, int k,
                       const double *XA, const double *XA2, const int *alpha,
                       const double *XB, const double *XB2, const int *beta,
                       double *D, int *I) {
  if (m == 0 || n == 0 || d == 0 || k == 0) return;
  int nt = nthreads_for((long)m * n * d);
#pragma omp parallel num_threads(nt)
  {
    double *row = (double *)malloc(sizeof(double) * (size_t)m);
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < n; j++) {
      const double *b = XB + (size_t)beta[j] * d;
      for (int i = 0; i < m; i++) {
        const double *a = XA + (size_t)alpha[i] * d;
        double c = 0.0;
        for (int p = 0; p < d; p++) c += a[p] * b[p];
        c *= -2.0;
        c += XA2[alpha[i]];
        c += XB2[beta[j]];
        row[i] = c;
      }
      oracle_heap_select_d(m, k, row, alpha, D + (size_t)j * k, I + (size_t)j * k);
    }
    free(row);
  }
}

void oracle_sgsknn_ref(int m, int n, int d, int k,
                       const float *XA, const float *XA2, const int *alpha,
                       const float *XB, const float *XB2, const int *beta,
                       float *D, int *I) {
  if (m == 0 || n == 0 || d == 0 || k == 0) return;
  int nt = nthreads_for((long)m * n * d);
#pragma omp parallel num_threads(nt)
  {
    float *row = (float *)malloc(sizeof(float) * (size_t)m);
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < n; j++) {
      const float *b = XB + (size_t)beta[j] * d;
      for (int i = 0; i < m; i++) {
        const float *a = XA + (size_t)alpha[i] * d;
        float c = 0.0f;
        for (int p = 0; p < d; p++) c += a[p] * b[p];
        c = (float)((double)c * -2.0);
        c += XA2[alpha[i]];
        c += XB2[beta[j]];
        row[i] = c;
      }
      oracle_heap_select_s(m, k, row, alpha, D + (size_t)j * k, I + (size_t)j * k);
    }
    free(row);
  }
}

/* ------------------------------------------------------------------------------------------
 * dgssq2nrm (frame/gsknn.c:481-594 driving sq2nrm_asm_d8x4.c): the dot product is summed in
 * p order inside each KC = 256 slab (gsknn_config.h: DKNN_KC), slab sums are added in slab
 * order, then -2 * c + aa + bb on the last slab. No clamp.
 * ---------------------------------------------------------------------------------------- */
static double slab_dot(const double *a, const double *b, int d) {
  double total = 0.0;
  for (int pc = 0; pc < d; pc += 256) {
    int pe = pc + 256 < d ? pc + 256 : d;
    double s = 0.0;
    for (int p = pc; p < pe; p++) s += a[p] * b[p];
    total = (pc == 0) ? s : s + total;
  }
  return total;
}

void oracle_dgssq2nrm(int m, int n, int d,
                      const double *XA, const double *XA2, const int *amap,
                      const double *XB, const double *XB2, const int *bmap,
                      double *C, int ldc) {
  if (m == 0 || n == 0 || d == 0) return;
  int nt = nthreads_for((long)m * n * d);
#pragma omp parallel for num_threads(nt) schedule(dynamic, 4)
  for (int j = 0; j < n; j++) {
    const double *b = XB + (size_t)bmap[j] * d;
    for (int i = 0; i < m; i++) {
      const double *a = XA + (size_t)amap[i] * d;
      double c = slab_dot(a, b, d);
      c = -2.0 * c;
      c = c + XA2[amap[i]];
      c = c + XB2[bmap[j]];
      C[(size_t)j * ldc + i] = c;
    }
  }
}

/* ------------------------------------------------------------------------------------------
 * 4-ary heap with a 3-slot header (gsknn_heapselect_int_d4.c:6-93). Children of s are
 * 4s+1..4s+4; the largest child is the first maximal one. Fill phase: while I[1] < I[0] the
 * key is written at position I[0]-1-I[1] and sifted down, unconditionally. Replace phase: a key
 * replaces the root only when strictly smaller.
 * ---------------------------------------------------------------------------------------- */
#define HO 3 /* KNN_HEAP_OFFSET, include/gsknn.h:47 */
static void sift_down4(double *D, int s, int k, int *I) {
  while (4 * s + 1 < k) {
    int j = 4 * s + 1;
    int last = 4 * s + 4 < k - 1 ? 4 * s + 4 : k - 1;
    for (int p = 4 * s + 2; p <= last; p++)
      if (D[p + HO] > D[j + HO]) j = p;
    if (D[s + HO] < D[j + HO]) {
      double td = D[s + HO]; D[s + HO] = D[j + HO]; D[j + HO] = td;
      int ti = I[s + HO]; I[s + HO] = I[j + HO]; I[j + HO] = ti;
      s = j;
    } else {
      break;
    }
  }
}

void oracle_heapselect_d4(int m, int k, const double *key, const int *val, double *D, int *I) {
  for (int i = 0; i < m; i++) {
    if (I[1] < I[0]) {
      int p = I[0] - 1 - I[1];
      D[p + HO] = key[i];
      I[p + HO] = val[i];
      if (p * 4 < k - 1) sift_down4(D, p, k, I);
      I[1] = I[1] + 1;
    } else if (key[i] < D[HO]) {
      D[HO] = key[i];
      I[HO] = val[i];
      sift_down4(D, 0, k, I);
    }
  }
}

void oracle_dgsknn_var3(int m, int n, int d, int k,
                        const double *XA, const double *XA2, const int *alpha,
                        const double *XB, const double *XB2, const int *beta,
                        double *D, int *I, int ldk) {
  if (m == 0 || n == 0 || d == 0) return;
  int nt = nthreads_for((long)m * n * d);
#pragma omp parallel num_threads(nt)
  {
    double *row = (double *)malloc(sizeof(double) * (size_t)m);
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < n; j++) {
      const double *b = XB + (size_t)beta[j] * d;
      for (int i = 0; i < m; i++) {
        double c = slab_dot(XA + (size_t)alpha[i] * d, b, d);
        c = -2.0 * c;
        c = c + XA2[alpha[i]];
        c = c + XB2[beta[j]];
        row[i] = c;
      }
      oracle_heapselect_d4(m, k, row, alpha, D + (size_t)j * ldk, I + (size_t)j * ldk);
    }
    free(row);
  }
}

/* ------------------------------------------------------------------------------------------
 * Tie-resolved exact selection: (distance, index as unsigned) lexicographic order.
 * ---------------------------------------------------------------------------------------- */
typedef struct { double d; uint32_t i; } entry_t;

static int entry_less(entry_t a, entry_t b) {
  if (a.d < b.d) return 1;
  if (a.d > b.d) return 0;
  return a.i < b.i;
}

/* Max-heap of the k best entries seen so far under entry_less. */
static void ent_sift(entry_t *h, int s, int n) {
  while (2 * s + 1 < n) {
    int j = 2 * s + 1;
    if (j + 1 < n && entry_less(h[j], h[j + 1])) j++;
    if (entry_less(h[s], h[j])) {
      entry_t t = h[s]; h[s] = h[j]; h[j] = t;
      s = j;
    } else {
      break;
    }
  }
}

static void ent_push_bounded(entry_t *h, int *cnt, int k, entry_t e) {
  if (*cnt < k) {
    /* sift up */
    int s = (*cnt)++;
    h[s] = e;
    while (s > 0) {
      int p = (s - 1) / 2;
      if (entry_less(h[p], h[s])) {
        entry_t t = h[p]; h[p] = h[s]; h[s] = t;
        s = p;
      } else {
        break;
      }
    }
  } else if (entry_less(e, h[0])) {
    h[0] = e;
    ent_sift(h, 0, k);
  }
}

static int ent_cmp(const void *pa, const void *pb) {
  entry_t a = *(const entry_t *)pa, b = *(const entry_t *)pb;
  if (entry_less(a, b)) return -1;
  if (entry_less(b, a)) return 1;
  return 0;
}

static void finish_row(entry_t *h, int cnt, int k, double *Dout, int *Iout) {
  qsort(h, (size_t)cnt, sizeof(entry_t), ent_cmp);
  for (int t = 0; t < k; t++) {
    if (t < cnt) {
      Dout[t] = h[t].d;
      Iout[t] = (int)h[t].i;
    } else {
      Dout[t] = INFINITY;
      Iout[t] = -1;
    }
  }
}

#define DEFINE_EXACT(NAME, T)                                                               \
  void NAME(int m, int n, int d, int k, const T *XA, const T *XA2, const int *alpha,        \
            const T *XB, const T *XB2, const int *beta, const T *Din, const int *Iin,       \
            int ldin, int clamp, double *Dout, int *Iout) {                                 \
    if (n == 0 || k == 0) return;                                                           \
    int nt = nthreads_for((long)m * n * (d > 0 ? d : 1));                                   \
    _Pragma("omp parallel num_threads(nt)") {                                               \
      entry_t *h = (entry_t *)malloc(sizeof(entry_t) * (size_t)k);                          \
      _Pragma("omp for schedule(dynamic, 4)") for (int j = 0; j < n; j++) {                 \
        int cnt = 0;                                                                        \
        const T *b = XB + (size_t)beta[j] * d;                                              \
        double bb = 0.0;                                                                    \
        if (XB2) {                                                                          \
          bb = (double)XB2[beta[j]];                                                        \
        } else {                                                                            \
          for (int p = 0; p < d; p++) bb += (double)b[p] * (double)b[p];                    \
        }                                                                                   \
        if (Din) {                                                                          \
          for (int t = 0; t < k; t++) {                                                     \
            entry_t e = {(double)Din[(size_t)j * ldin + t],                                 \
                         (uint32_t)Iin[(size_t)j * ldin + t]};                              \
            ent_push_bounded(h, &cnt, k, e);                                                \
          }                                                                                 \
        }                                                                                   \
        for (int i = 0; i < m; i++) {                                                       \
          const T *a = XA + (size_t)alpha[i] * d;                                           \
          double dot = 0.0, aa = 0.0;                                                       \
          for (int p = 0; p < d; p++) dot += (double)a[p] * (double)b[p];                   \
          if (XA2) {                                                                        \
            aa = (double)XA2[alpha[i]];                                                     \
          } else {                                                                          \
            for (int p = 0; p < d; p++) aa += (double)a[p] * (double)a[p];                  \
          }                                                                                 \
          double c = -2.0 * dot + aa + bb;                                                  \
          if (clamp && !(c >= 0.0)) c = c < 0.0 ? 0.0 : c;                                  \
          if (c != c) c = INFINITY;                                                         \
          entry_t e = {c, (uint32_t)alpha[i]};                                              \
          ent_push_bounded(h, &cnt, k, e);                                                  \
        }                                                                                   \
        finish_row(h, cnt, k, Dout + (size_t)j * k, Iout + (size_t)j * k);                  \
      }                                                                                     \
      free(h);                                                                              \
    }                                                                                       \
  }
DEFINE_EXACT(oracle_knn_exact_d, double)
DEFINE_EXACT(oracle_knn_exact_s, float)

/* ------------------------------------------------------------------------------------------
 * 1-norm kNN (kernels/x86_64/sandybridge/rnn_r_1norm_int_d8x4_row.c: per (query, candidate) the
 * sum over p, in dimension order, of |a_p - b_p| in the working precision, then max(0, .), then
 * the heap select): the same sum here, in T, merged with Din/Iin, tie-resolved like
 * oracle_knn_exact_*, rows ascending.
 * ---------------------------------------------------------------------------------------- */
#define DEFINE_EXACT_L1(NAME, T, ABS)                                                       \
  void NAME(int m, int n, int d, int k, const T *XA, const int *alpha, const T *XB,         \
            const int *beta, const T *Din, const int *Iin, int ldin, double *Dout,          \
            int *Iout) {                                                                    \
    if (n == 0 || k == 0) return;                                                           \
    int nt = nthreads_for((long)m * n * (d > 0 ? d : 1));                                   \
    _Pragma("omp parallel num_threads(nt)") {                                               \
      entry_t *h = (entry_t *)malloc(sizeof(entry_t) * (size_t)k);                          \
      _Pragma("omp for schedule(dynamic, 4)") for (int j = 0; j < n; j++) {                 \
        int cnt = 0;                                                                        \
        const T *b = XB + (size_t)beta[j] * d;                                              \
        if (Din) {                                                                          \
          for (int t = 0; t < k; t++) {                                                     \
            entry_t e = {(double)Din[(size_t)j * ldin + t],                                 \
                         (uint32_t)Iin[(size_t)j * ldin + t]};                              \
            ent_push_bounded(h, &cnt, k, e);                                                \
          }                                                                                 \
        }                                                                                   \
        for (int i = 0; i < m; i++) {                                                       \
          const T *a = XA + (size_t)alpha[i] * d;                                           \
          T acc = (T)0;                                                                     \
          for (int p = 0; p < d; p++) acc += ABS(a[p] - b[p]);                              \
          double c = (double)acc;                                                           \
          if (c != c) c = INFINITY;                                                         \
          entry_t e = {c, (uint32_t)alpha[i]};                                              \
          ent_push_bounded(h, &cnt, k, e);                                                  \
        }                                                                                   \
        finish_row(h, cnt, k, Dout + (size_t)j * k, Iout + (size_t)j * k);                  \
      }                                                                                     \
      free(h);                                                                              \
    }                                                                                       \
  }
DEFINE_EXACT_L1(oracle_knn_exact_l1_d, double, fabs)
DEFINE_EXACT_L1(oracle_knn_exact_l1_s, float, fabsf)

void oracle_select_rows_d(int m, int n, int k, const double *C, int ldc, const int *alpha,
                          const double *Din, const int *Iin, int ldin,
                          double *Dout, int *Iout) {
  if (n == 0 || k == 0) return;
  int nt = nthreads_for((long)m * n);
#pragma omp parallel num_threads(nt)
  {
    entry_t *h = (entry_t *)malloc(sizeof(entry_t) * (size_t)k);
#pragma omp for schedule(dynamic, 4)
    for (int j = 0; j < n; j++) {
      int cnt = 0;
      if (Din) {
        for (int t = 0; t < k; t++) {
          entry_t e = {Din[(size_t)j * ldin + t], (uint32_t)Iin[(size_t)j * ldin + t]};
          ent_push_bounded(h, &cnt, k, e);
        }
      }
      for (int i = 0; i < m; i++) {
        double c = C[(size_t)j * ldc + i];
        if (c != c) c = INFINITY;
        entry_t e = {c, (uint32_t)alpha[i]};
        ent_push_bounded(h, &cnt, k, e);
      }
      finish_row(h, cnt, k, Dout + (size_t)j * k, Iout + (size_t)j * k);
    }
    free(h);
  }
}

/* ------------------------------------------------------------------------------------------
 * Batching form: union of leaf-mates per point, de-duplicated, exact FP64 selection.
 * ---------------------------------------------------------------------------------------- */
void oracle_allnn_leaves_s(int N, int d, int k, const float *X, const float *X2, int nleaves,
                           const int *ptr, const int *pts, const float *Din, const int *Iin,
                           int ldin, double *Dout, int *Iout) {
  if (N <= 0 || k <= 0) return;
  /* leaves of every point (CSR inversion) */
  int *cnt = (int *)calloc((size_t)N + 1, sizeof(int));
  for (int l = 0; l < nleaves; l++)
    for (int t = ptr[l]; t < ptr[l + 1]; t++) cnt[pts[t] + 1]++;
  for (int p = 0; p < N; p++) cnt[p + 1] += cnt[p];
  int *fill = (int *)malloc(sizeof(int) * (size_t)N);
  memcpy(fill, cnt, sizeof(int) * (size_t)N);
  int *mine = (int *)malloc(sizeof(int) * (size_t)(cnt[N] > 0 ? cnt[N] : 1));
  for (int l = 0; l < nleaves; l++)
    for (int t = ptr[l]; t < ptr[l + 1]; t++) mine[fill[pts[t]]++] = l;
  int nt = nthreads_for((long)N * 256 * d);
#pragma omp parallel num_threads(nt)
  {
    entry_t *h = (entry_t *)malloc(sizeof(entry_t) * (size_t)k);
    int *seen = (int *)malloc(sizeof(int) * (size_t)N);
    for (int i = 0; i < N; i++) seen[i] = -1;
#pragma omp for schedule(dynamic, 16)
    for (int p = 0; p < N; p++) {
      int c = 0;
      const float *b = X + (size_t)p * d;
      const double bb = (double)X2[p];
      for (int u = cnt[p]; u < cnt[p + 1]; u++) {
        const int l = mine[u];
        for (int t = ptr[l]; t < ptr[l + 1]; t++) {
          const int q = pts[t];
          if (seen[q] == p) continue;
          seen[q] = p;
          const float *a = X + (size_t)q * d;
          double dot = 0.0;
          for (int j = 0; j < d; j++) dot += (double)a[j] * (double)b[j];
          double v = -2.0 * dot + (double)X2[q] + bb;
          if (!(v >= 0.0)) v = v < 0.0 ? 0.0 : v;
          if (v != v) v = INFINITY;
          entry_t e = {v, (uint32_t)q};
          ent_push_bounded(h, &c, k, e);
        }
      }
      if (Din) {
        for (int t = 0; t < k; t++) {
          const int q = Iin[(size_t)p * ldin + t];
          if (q >= 0 && q < N && seen[q] == p) continue; /* already taken from a leaf */
          if (q >= 0 && q < N) seen[q] = p;
          entry_t e = {(double)Din[(size_t)p * ldin + t], (uint32_t)q};
          ent_push_bounded(h, &c, k, e);
        }
      }
      finish_row(h, c, k, Dout + (size_t)p * k, Iout + (size_t)p * k);
    }
    free(seen);
    free(h);
  }
  free(mine);
  free(fill);
  free(cnt);
}

/* ------------------------------------------------------------------------------------------
 * Heap validity.
 * ---------------------------------------------------------------------------------------- */
int oracle_is_maxheap_d(int n, int k, int ld, const double *D) {
  for (int j = 0; j < n; j++) {
    const double *r = D + (size_t)j * ld;
    for (int s = 1; s < k; s++)
      if (r[(s - 1) / 2] < r[s]) return 0;
  }
  return 1;
}

int oracle_is_maxheap_s(int n, int k, int ld, const float *D) {
  for (int j = 0; j < n; j++) {
    const float *r = D + (size_t)j * ld;
    for (int s = 1; s < k; s++)
      if (r[(s - 1) / 2] < r[s]) return 0;
  }
  return 1;
}

/* 4-ary heap with header: only the filled region [k - I[1], k) is checked; it is a forest of
 * 4-ary subtrees whose parents are all inside the region. */
int oracle_is_maxheap4_d(int n, int k, int ld, const double *D, const int *I) {
  for (int j = 0; j < n; j++) {
    const double *r = D + (size_t)j * ld;
    const int *ri = I + (size_t)j * ld;
    if (ri[0] != k || ri[2] != ld) return 0;
    int filled = ri[1];
    if (filled < 0 || filled > k) return 0;
    for (int s = k - filled; s < k; s++) {
      if (s == 0) continue;
      int p = (s - 1) / 4;
      if (p >= k - filled && r[HO + p] < r[HO + s]) return 0;
    }
  }
  return 1;
}

/* ------------------------------------------------------------------------------------------
 * Heap rows to ascending lists by repeated pops (frame/old/dgsrnn_directKQuery.cpp:112-124):
 * pass j sifts the root down over the first k - j entries, emits the root at position
 * k - j - 1 and moves the last live entry to the root. The row (stride ld) is consumed; the
 * list goes to Dout / Iout (n x k, ids widened to 64 bits as the reference's std::pair).
 * ---------------------------------------------------------------------------------------- */
#define DEFINE_POP_ROWS(NAME, T, SIFT)                                                      \
  void NAME(int n, int k, int ld, T *D, int *I, T *Dout, long long *Iout) {                 \
    for (int i = 0; i < n; i++) {                                                           \
      T *d = D + (size_t)i * ld;                                                            \
      int *id = I + (size_t)i * ld;                                                         \
      for (int j = 0; j < k; j++) {                                                         \
        SIFT(d, 0, k - j, id);                                                              \
        Dout[(size_t)i * k + k - j - 1] = d[0];                                             \
        Iout[(size_t)i * k + k - j - 1] = (long long)id[0];                                 \
        d[0] = d[k - j - 1];                                                                \
        id[0] = id[k - j - 1];                                                              \
      }                                                                                     \
    }                                                                                       \
  }
DEFINE_POP_ROWS(oracle_heap_pop_rows_d, double, sift_down_d)
DEFINE_POP_ROWS(oracle_heap_pop_rows_s, float, sift_down_s)
