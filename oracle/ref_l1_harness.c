/*
 * ref_l1_harness.c -- TEST INFRASTRUCTURE ONLY: drives the reference's own 1-norm micro-kernel
 * (kernels/x86_64/sandybridge/rnn_r_1norm_int_d8x4_row.c, compiled from the reference sources
 * into oracle/_ref/libgsknn_ref.so by oracle/Makefile) over every 8-query x 4-candidate block of
 * a small problem, so that the 1-norm restatement in gsknn_oracle.c can be pinned to the
 * reference's outputs (tests/golden/make_golden.py). The reference's dispatch never selects
 * this kernel (frame/gsknn.c uses micro_d[0], the 2-norm kernel), so it is called directly,
 * with its operands packed the way its loads expect them:
 *   a[p * 8 + i]  query i of the block, dimension p  (8 rows, zero padded);
 *   b[p * 4 + j]  candidate j of the block             (4 columns, zero padded);
 *   aux->D / aux->I / aux->ldr  the block's heap rows, aux->m / aux->n the valid rows / columns,
 *   bmap[j]  the candidate ids given to heapSelect_d (frame/gsknn_heap.c:139-162).
 * The kernel reads up to two dimensions past the end of a and b while prefetching, so both
 * buffers carry 16 zero doubles of slack.
 */
#include <stdlib.h>
#include <string.h>

#include <gsknn.h> /* the reference header (aux_t) */

void rnn_r_1norm_int_d8x4_row(int k, int r, double *aa, double *a, double *bb, double *b,
                              double *c, aux_t *aux, int *bmap);

/* Queries XQ (m x d) against candidates XC (n x d) into the heaps D / I (m rows of r, stride
 * r), which the caller initialises (the reference's heapCreate_d: DBL_MAX and -1). */
int ref_l1_knn(int m, int n, int d, int r, const double *XQ, const double *XC, double *D,
               int *I) {
  double *a = (double *)aligned_alloc(32, sizeof(double) * ((size_t)8 * d + 16));
  double *b = (double *)aligned_alloc(32, sizeof(double) * ((size_t)4 * d + 16));
  double *c = (double *)aligned_alloc(32, sizeof(double) * 32);
  int bmap[4];
  if (!a || !b || !c) {
    free(a);
    free(b);
    free(c);
    return 1;
  }
  memset(a, 0, sizeof(double) * ((size_t)8 * d + 16));
  memset(b, 0, sizeof(double) * ((size_t)4 * d + 16));
  memset(c, 0, sizeof(double) * 32);
  for (int i0 = 0; i0 < m; i0 += 8) {
    const int mr = m - i0 < 8 ? m - i0 : 8;
    for (int p = 0; p < d; p++)
      for (int i = 0; i < 8; i++) a[p * 8 + i] = i < mr ? XQ[(size_t)(i0 + i) * d + p] : 0.0;
    for (int j0 = 0; j0 < n; j0 += 4) {
      const int nr = n - j0 < 4 ? n - j0 : 4;
      for (int p = 0; p < d; p++)
        for (int j = 0; j < 4; j++) b[p * 4 + j] = j < nr ? XC[(size_t)(j0 + j) * d + p] : 0.0;
      for (int j = 0; j < 4; j++) bmap[j] = j0 + j;
      aux_t aux;
      memset(&aux, 0, sizeof(aux));
      aux.b_next = b;
      aux.D = D + (size_t)i0 * r;
      aux.I = I + (size_t)i0 * r;
      aux.ldr = r;
      aux.pc = 0;
      aux.m = mr;
      aux.n = nr;
      rnn_r_1norm_int_d8x4_row(d, r, NULL, a, NULL, b, c, &aux, bmap);
    }
  }
  free(a);
  free(b);
  free(c);
  return 0;
}
