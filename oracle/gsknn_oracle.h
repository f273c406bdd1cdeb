/*
 * gsknn_oracle.h -- CPU restatement of the GSKNN reference algorithm.
 *
 * TEST INFRASTRUCTURE ONLY. This file and liboracle.so are the parity checker for the CUDA
 * library in rnn_b200/. Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg
 * may load it. The product library never links, loads or calls it.
 *
 * Notation (same as the reference C API): m = number of candidate points (alpha, the "A"
 * side of dgsknn), n = number of query points (beta, heap rows), d = dimension, k = number
 * of neighbours. Point tables are row-major N x d; norms are indexed by global point id.
 *
 * Parity pinning: every function here is checked bit-for-bit against outputs of the reference
 * library compiled from its own sources (oracle/_ref, fixtures in tests/golden/).
 */
#ifndef GSKNN_ORACLE_H
#define GSKNN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Binary max-heap replace-root-if-(x <= root) selection (frame/gsknn_heap.c:52-162). */
void oracle_heap_select_d(int m, int k, const double *x, const int *alpha, double *D, int *I);
void oracle_heap_select_s(int m, int k, const float *x, const int *alpha, float *D, int *I);

/* The reference oracle dgsknn_ref / sgsknn_ref (frame/gsknn_ref.c:63-162 with
 * frame/dgsknn_ref_impl.h and frame/sgsknn_ref_impl.h): gather, naive dot product in the
 * reference's summation order, times -2, plus both norms, heap select per query row.
 * Runs row by row (no m x n matrix); rows are independent so this is exact. */
void oracle_dgsknn_ref(int m, int n, int d, int k,
                       const double *XA, const double *XA2, const int *alpha,
                       const double *XB, const double *XB2, const int *beta,
                       double *D, int *I);
void oracle_sgsknn_ref(int m, int n, int d, int k,
                       const float *XA, const float *XA2, const int *alpha,
                       const float *XB, const float *XB2, const int *beta,
                       float *D, int *I);

/* Full squared-distance block of dgssq2nrm (frame/gsknn.c:481-594, sq2nrm_asm_d8x4.c):
 * C[j*ldc + i] = -2 <XA[amap[i]], XB[bmap[j]]> + XA2[amap[i]] + XB2[bmap[j]]. No clamp. */
void oracle_dgssq2nrm(int m, int n, int d,
                      const double *XA, const double *XA2, const int *amap,
                      const double *XB, const double *XB2, const int *bmap,
                      double *C, int ldc);

/* 4-ary heap with the 3-slot header used by dgsknn when k > 512
 * (kernels/x86_64/sandybridge/gsknn_heapselect_int_d4.c:6-93; layout from
 * frame/gsknn_heap.c:257-307): D = [ro,0,0 | heap], I = [k, filled, ldk | heap]. */
void oracle_heapselect_d4(int m, int k, const double *key, const int *val, double *D, int *I);

/* dgsknn_var3 (frame/gsknn.c:597-659): full distances, then the 4-ary select per query row.
 * D/I are heap_t rows of leading dimension ldk (with the 3-slot header). */
void oracle_dgsknn_var3(int m, int n, int d, int k,
                        const double *XA, const double *XA2, const int *alpha,
                        const double *XB, const double *XB2, const int *beta,
                        double *D, int *I, int ldk);

/* Tie-resolved oracle used for exact index-set parity: for every query row j, the k smallest
 * entries of (incoming row D/I) U (all candidates), ordered by (distance, index as unsigned),
 * i.e. among equal distances the lower index wins and the -1 sentinel loses. Distances are
 * computed in FP64 from the (float or double) inputs: -2<a,b> + |a|^2 + |b|^2, optionally
 * clamped at zero (the CUDA kernels clamp, as the reference's AVX double micro-kernel does,
 * rnn_r_int_d8x4_row.c:373-382). Output rows are sorted ascending (Dout/Iout are n x k).
 * The norms may be NULL, in which case they are recomputed in FP64 from the table. */
void oracle_knn_exact_d(int m, int n, int d, int k,
                        const double *XA, const double *XA2, const int *alpha,
                        const double *XB, const double *XB2, const int *beta,
                        const double *Din, const int *Iin, int ldin,
                        int clamp, double *Dout, int *Iout);
void oracle_knn_exact_s(int m, int n, int d, int k,
                        const float *XA, const float *XA2, const int *alpha,
                        const float *XB, const float *XB2, const int *beta,
                        const float *Din, const int *Iin, int ldin,
                        int clamp, double *Dout, int *Iout);

/* The same selection rule applied to an explicit FP64 distance row set: rows j of C
 * (C[j*ldc + i], i < m) with ids alpha[i]. Used for the batching and serving forms. */
void oracle_select_rows_d(int m, int n, int k, const double *C, int ldc, const int *alpha,
                          const double *Din, const int *Iin, int ldin,
                          double *Dout, int *Iout);

/* Batching form (no reference function; restates what the reference's tree drivers obtain by
 * calling sgsknn once per leaf with alpha = beta = the leaf, frame/gsknn.c:1106-1135, plus the
 * removal of neighbours found twice): for every point p < N, the k nearest (FP64 distances of
 * the float inputs as in oracle_knn_exact_s, clamped, lower id first on ties) among the union
 * of p's leaf-mates over all leaves listed (leaf l = pts[ptr[l] .. ptr[l+1])) and its incoming
 * heap row Din/Iin (ids found in a leaf take the leaf's distance). Output sorted ascending. */
void oracle_allnn_leaves_s(int N, int d, int k, const float *X, const float *X2, int nleaves,
                           const int *ptr, const int *pts, const float *Din, const int *Iin,
                           int ldin, double *Dout, int *Iout);

/* Heap checks: 1 if every row is a valid binary (or 4-ary with header) max-heap. */
int oracle_is_maxheap_d(int n, int k, int ld, const double *D);
int oracle_is_maxheap_s(int n, int k, int ld, const float *D);
int oracle_is_maxheap4_d(int n, int k, int ld, const double *D, const int *I);

/* 1-norm kNN (rnn_r_1norm_int_d8x4_row.c): candidates alpha of XA against queries beta of XB,
 * in-order sums of |a_p - b_p| in the input precision, merged with Din/Iin (may be NULL),
 * (distance, unsigned id) order, rows ascending. */
void oracle_knn_exact_l1_d(int m, int n, int d, int k, const double *XA, const int *alpha,
                           const double *XB, const int *beta, const double *Din, const int *Iin,
                           int ldin, double *Dout, int *Iout);
void oracle_knn_exact_l1_s(int m, int n, int d, int k, const float *XA, const int *alpha,
                           const float *XB, const int *beta, const float *Din, const int *Iin,
                           int ldin, double *Dout, int *Iout);

/* Pops of max-heap rows into ascending lists (frame/old/dgsrnn_directKQuery.cpp:112-124). */
void oracle_heap_pop_rows_d(int n, int k, int ld, double *D, int *I, double *Dout,
                            long long *Iout);
void oracle_heap_pop_rows_s(int n, int k, int ld, float *D, int *I, float *Dout,
                            long long *Iout);

/* Number of OpenMP threads the oracle uses (0 = runtime default). */
void oracle_set_threads(int nthreads);

#ifdef __cplusplus
}
#endif
#endif
