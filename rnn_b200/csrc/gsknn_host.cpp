// gsknn_host.cpp -- host-side utilities of the GSKNN C ABI: heap_t construction, the scalar
// heap-select helpers and the small sort/swap routines the reference exports
// (frame/gsknn_heap.c, frame/gsknn_util.c). None of these is on the GPU path: the CUDA
// pipeline keeps its own lists on chip and only reads and writes the heap rows.
#include "gsknn.h"

#include <stdlib.h>

// Binary max-heap sift-down over n entries from position s (frame/gsknn_heap.c:52-96).
template <typename T>
static void sift_down(T *D, int s, int n, int *I) {
  while (2 * s + 1 < n) {
    int j = 2 * s + 1;
    if (j + 1 < n && D[j] < D[j + 1]) j++;
    if (!(D[s] < D[j])) break;
    T td = D[s]; D[s] = D[j]; D[j] = td;
    int ti = I[s]; I[s] = I[j]; I[j] = ti;
    s = j;
  }
}

extern "C" {

void swap_float(float *x, int i, int j) {
  float t = x[i]; x[i] = x[j]; x[j] = t;
}
void swap_double(double *x, int i, int j) {
  double t = x[i]; x[i] = x[j]; x[j] = t;
}
void swap_int(int *x, int i, int j) {
  int t = x[i]; x[i] = x[j]; x[j] = t;
}

// Ascending sort of (D, I) pairs by D (frame/gsknn_util.c:77-112). Kept as a stable
// exchange sort so equal keys keep their order, as the reference's does.
void bubbleSort_s(int n, float *D, int *I) {
  for (int i = 0; i < n - 1; i++)
    for (int j = 0; j < n - 1 - i; j++)
      if (D[j] > D[j + 1]) { swap_float(D, j, j + 1); swap_int(I, j, j + 1); }
}
void bubbleSort_d(int n, double *D, int *I) {
  for (int i = 0; i < n - 1; i++)
    for (int j = 0; j < n - 1 - i; j++)
      if (D[j] > D[j + 1]) { swap_double(D, j, j + 1); swap_int(I, j, j + 1); }
}

// 32-byte aligned host allocation of m*n elements of `size` bytes (frame/gsknn_util.c:119-133).
// Returns NULL on failure instead of exiting the process.
double *gsknn_malloc_aligned(int m, int n, int size) {
  void *p = nullptr;
  size_t bytes = (size_t)m * (size_t)n * (size_t)size;
  if (bytes == 0) bytes = 32;
  if (posix_memalign(&p, 32, bytes) != 0) return nullptr;
  return static_cast<double *>(p);
}

// Replace the root whenever x <= root (frame/gsknn_heap.c:104-162).
void heapSelect_s(int m, int r, float *x, int *alpha, float *D, int *I) {
  for (int i = 0; i < m; i++) {
    if (x[i] > D[0]) continue;
    D[0] = x[i];
    I[0] = alpha[i];
    sift_down(D, 0, r, I);
  }
}
void heapSelect_d(int m, int r, double *x, int *alpha, double *D, int *I) {
  for (int i = 0; i < m; i++) {
    if (x[i] > D[0]) continue;
    D[0] = x[i];
    I[0] = alpha[i];
    sift_down(D, 0, r, I);
  }
}

// 4-ary heap with the 3-slot header (layout of frame/gsknn_heap.c:257-307; select rule of
// kernels/x86_64/sandybridge/gsknn_heapselect_int_d4.c:58-93): fill unconditionally while
// I[1] < I[0], then replace the root when strictly smaller.
static void sift_down4(double *D, int s, int k, int *I) {
  const int H = KNN_HEAP_OFFSET;
  while (4 * s + 1 < k) {
    int j = 4 * s + 1;
    const int last = 4 * s + 4 < k - 1 ? 4 * s + 4 : k - 1;
    for (int p = 4 * s + 2; p <= last; p++)
      if (D[p + H] > D[j + H]) j = p;
    if (!(D[s + H] < D[j + H])) break;
    double td = D[s + H]; D[s + H] = D[j + H]; D[j + H] = td;
    int ti = I[s + H]; I[s + H] = I[j + H]; I[j + H] = ti;
    s = j;
  }
}
void heapSelect_dheap(int m, int k, double *key, int *val, double *D, int *I) {
  const int H = KNN_HEAP_OFFSET;
  for (int i = 0; i < m; i++) {
    if (I[1] < I[0]) {
      const int p = I[0] - 1 - I[1];
      D[p + H] = key[i];
      I[p + H] = val[i];
      if (p * 4 < k - 1) sift_down4(D, p, k, I);
      I[1] = I[1] + 1;
    } else if (key[i] < D[H]) {
      D[H] = key[i];
      I[H] = val[i];
      sift_down4(D, 0, k, I);
    }
  }
}

// heap_t wrappers around caller storage (frame/gsknn_heap.c:169-207): binary layout, ldk = k.
heap_t *heapAttach_s(int m, int k, float *D, int *I) {
  heap_t *h = static_cast<heap_t *>(calloc(1, sizeof(heap_t)));
  if (!h) return nullptr;
  h->m = m; h->k = k; h->d = 2; h->ro_s = 0.0f; h->ldk = k;
  h->D_s = D; h->I = I; h->type = KNN_2NORM; h->prec = KNN_SINGLE;
  return h;
}
heap_t *heapAttach_d(int m, int k, double *D, int *I) {
  heap_t *h = static_cast<heap_t *>(calloc(1, sizeof(heap_t)));
  if (!h) return nullptr;
  h->m = m; h->k = k; h->d = 2; h->ro = 0.0; h->ldk = k;
  h->D = D; h->I = I; h->type = KNN_2NORM; h->prec = KNN_DOUBLE;
  return h;
}

// Owning heaps (frame/gsknn_heap.c:215-319): rows of k sentinels (ro, -1). Double heaps with
// k > KNN_VAR_THRES use the 4-ary layout with ldk = ((k + 2) / 4 + 1) * 4 and the header
// D = [ro, 0, 0], I = [k, 0, ldk].
heap_t *heapCreate_s(int m, int k, float ro) {
  heap_t *h = static_cast<heap_t *>(calloc(1, sizeof(heap_t)));
  if (!h) return nullptr;
  h->m = m; h->k = k; h->d = 2; h->ro_s = ro; h->ldk = k;
  h->type = KNN_2NORM; h->prec = KNN_SINGLE;
  h->D_s = static_cast<float *>(malloc(sizeof(float) * (size_t)k * m + 4));
  h->I = static_cast<int *>(malloc(sizeof(int) * (size_t)k * m + 4));
  if (!h->D_s || !h->I) { free(h->D_s); free(h->I); free(h); return nullptr; }
  for (size_t i = 0; i < (size_t)m * k; i++) { h->D_s[i] = ro; h->I[i] = -1; }
  return h;
}

heap_t *heapCreate_d(int m, int k, double ro) {
  heap_t *h = static_cast<heap_t *>(calloc(1, sizeof(heap_t)));
  if (!h) return nullptr;
  int ldk;
  if (k > KNN_VAR_THRES) {
    ldk = ((k + KNN_HEAP_OFFSET - 1) / 4 + 1) * 4;
    h->d = 4;
  } else {
    ldk = k;
    h->d = 2;
  }
  h->m = m; h->k = k; h->ro = ro; h->ldk = ldk;
  h->type = KNN_2NORM; h->prec = KNN_DOUBLE;
  h->D = gsknn_malloc_aligned(ldk, m, sizeof(double));
  h->I = reinterpret_cast<int *>(gsknn_malloc_aligned(ldk, m, sizeof(int)));
  if (!h->D || !h->I) { free(h->D); free(h->I); free(h); return nullptr; }
  for (int i = 0; i < m; i++) {
    double *Dr = h->D + (size_t)i * ldk;
    int *Ir = h->I + (size_t)i * ldk;
    int o = 0;
    if (k > KNN_VAR_THRES) {
      Dr[0] = ro; Dr[1] = 0.0; Dr[2] = 0.0;
      Ir[0] = k; Ir[1] = 0; Ir[2] = ldk;
      o = KNN_HEAP_OFFSET;
    }
    for (int j = 0; j < k; j++) { Dr[o + j] = ro; Ir[o + j] = -1; }
  }
  return h;
}

void heapFree_s(heap_t *heap) {
  if (!heap) return;
  free(heap->D_s);
  free(heap->I);
  free(heap);
}
void heapFree_d(heap_t *heap) {
  if (!heap) return;
  free(heap->D);
  free(heap->I);
  free(heap);
}

}  // extern "C"
