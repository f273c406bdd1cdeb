/*
 * gsknn.h -- public C ABI of the B200 GSKNN library (libgsknn.so).
 *
 * Drop-in for the GSKNN C API (ChenhanYu/rnn, include/gsknn.h): every prototype, constant and
 * struct layout of the reference header is kept, with the same argument meaning, so a program
 * or binding built against the reference links against this library unchanged. Behind it the
 * fused distance + k-selection work runs as CUDA kernels on one B200 (sm_100a).
 *
 * Argument convention of the reference (frame/gsknn.c:1106-1184):
 *   dgsknn/sgsknn(m, n, k, r, XA, XA2, alpha, XB, XB2, beta, heap)
 *     m  = number of candidate points alpha[0..m) of table XA (norms XA2)
 *     n  = number of query points beta[0..n) of table XB (norms XB2) = heap rows
 *     k  = dimension d, r = number of neighbours
 *   *_var1(m, n, k, r, XA, XA2, amap, XB, XB2, bmap, D, I) have the roles swapped:
 *     m/XA/amap are the queries (heap rows), n/XB/bmap the candidates, D/I are m x r.
 * Tables are row-major (row i of table X is X[i*d .. i*d+d)); norms are squared 2-norms indexed
 * by global point id; D/I rows are max-heaps updated in place, so repeated calls merge.
 *
 * All pointers of the reference API are host pointers; each call copies what it needs to the
 * GPU and back, and returns when D/I are updated. Extensions (prefixed gsknn_) take device
 * pointers and a CUDA stream for resident data.
 *
 * Behavioural notes against the reference:
 *   - ties at the k-th distance go to the lower point id (the reference keeps the later
 *     candidate), so results equal the reference's as index sets modulo exact ties;
 *   - squared distances are clamped at 0 in both precisions (the reference clamps in its
 *     double micro-kernel only, kernels/x86_64/sandybridge/rnn_r_int_d8x4_row.c:373-382);
 *   - errors never exit() the process: the call returns with D/I untouched and the status is
 *     available from gsknn_last_error().
 */
#ifndef GSKNN_B200_H
#define GSKNN_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#include <math.h>
#include <stddef.h>

/* include/gsknn.h:46-47 of the reference */
#define KNN_VAR_THRES 512
#define KNN_HEAP_OFFSET 3

typedef unsigned long long dim_t;

/* include/gsknn.h:51-59 */
typedef enum { KNN_2NORM, KNN_1NORM } knn_type;
typedef enum { KNN_DOUBLE, KNN_SINGLE } knn_prec;

/* include/gsknn.h:61-73: micro-kernel side channel. Kept for layout compatibility only; the
 * CUDA kernels take their parameters by value and never read it. */
struct aux_s {
  double *b_next;
  float *b_next_s;
  int *I;
  double *D;
  float *D_s;
  int ldr;
  char *flag;
  int pc;
  int m;
  int n;
};
typedef struct aux_s aux_t;

/* include/gsknn.h:75-88: a set of m neighbour lists of k entries, row stride ldk.
 * `type` (KNN_2NORM from heapCreate_* / heapAttach_*) selects the distance of sgsknn / dgsknn /
 * dgsknn_var3 calls on the heap: set it to KNN_1NORM for the 1-norm (see gsknn_s_device_metric).
 * d = 2 for binary heaps; d = 4 for the 4-ary heaps with a 3-slot header that heapCreate_d
 * builds when k > KNN_VAR_THRES (D = [ro,0,0 | heap], I = [k, filled, ldk | heap]). */
struct heap_s {
  int m;
  int k;
  int ldk;
  int d;
  double ro;
  double *D;
  float ro_s;
  float *D_s;
  int *I;
  knn_type type;
  knn_prec prec;
};
typedef struct heap_s heap_t;

/* ---- fused kNN: replaces frame/gsknn.c:1106-1135 (sgsknn) and 1138-1184 (dgsknn) ---- */
void sgsknn(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
            float *XB2, int *beta, heap_t *heap);
void dgsknn(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
            double *XB2, int *beta, heap_t *heap);

/* ---- replaces frame/gsknn.c:665-880 (sgsknn_var1) and 883-1103 (dgsknn_var1); the entry
 *      points python/gsknn.py:79-92 and 169-182 bind ---- */
void sgsknn_var1(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                 float *XB2, int *beta, float *D, int *I);
void dgsknn_var1(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
                 double *XB2, int *beta, double *D, int *I);

/* ---- replaces frame/gsknn.c:597-659: large-k double path over heap_t storage (4-ary heaps
 *      with header when heap->d == 4, binary heaps otherwise) ---- */
void dgsknn_var3(int m, int n, int k, int r, double *XA, double *XA2, int *amap, double *XB,
                 double *XB2, int *bmap, heap_t *heap);

/* ---- replaces frame/gsknn.c:481-594: C[j*ldc + i] = |XA[amap[i]] - XB[bmap[j]]|^2 computed
 *      as -2<a,b> + XA2[amap[i]] + XB2[bmap[j]] (no clamp), i < m, j < n ---- */
void dgssq2nrm(int m, int n, int k, double *XA, double *XA2, int *amap, double *XB,
               double *XB2, int *bmap, double *C, int ldc);

/* ---- host utilities: replace frame/gsknn_util.c:53-133 and frame/gsknn_heap.c:52-337 ---- */
double *gsknn_malloc_aligned(int m, int n, int size);
heap_t *heapCreate_s(int m, int k, float ro);
heap_t *heapCreate_d(int m, int k, double ro);
void heapFree_s(heap_t *heap);
void heapFree_d(heap_t *heap);
heap_t *heapAttach_s(int m, int k, float *D, int *I);
heap_t *heapAttach_d(int m, int k, double *D, int *I);
void heapSelect_s(int m, int r, float *x, int *alpha, float *D, int *I);
void heapSelect_d(int m, int r, double *x, int *alpha, double *D, int *I);
/* Declared by the reference (include/gsknn.h:236-243) without a definition; here it is the
 * 4-ary header-heap select that dgsknn_var3 performs per row. */
void heapSelect_dheap(int m, int k, double *key, int *val, double *D, int *I);
void swap_float(float *x, int i, int j);
void swap_double(double *x, int i, int j);
void swap_int(int *I, int i, int j);
void bubbleSort_s(int n, float *D, int *I);
void bubbleSort_d(int n, double *D, int *I);

/* ---- reference-algorithm entry points: replace frame/gsknn_ref.c:63-162 (the
 *      python/gsknn.py:34 and 124 bindings). They run the unfused GPU path (explicit distance
 *      block, then per-row heap selection) with the reference oracle's D/I convention
 *      (n rows of r, m candidates on the XA/alpha side). ---- */
void sgsknn_ref(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                float *XB2, int *beta, float *D, int *I);
void dgsknn_ref(int m, int n, int k, int r, double *XA, double *XA2, int *alpha, double *XB,
                double *XB2, int *beta, double *D, int *I);

/* ---- replace frame/gsknn_ref_stl.cpp:81-147 (sgsknn_ref_stl) and 149-214 (dgsknn_ref_stl),
 *      declared by include/gsknn_ref_stl.hpp: the reference oracle with an STL heap. The same
 *      GPU path and D/I convention as *_ref; the rows come back as descending binary max-heaps
 *      (the STL heap keeps its own layout, and on exact ties the earlier candidate). ---- */
void sgsknn_ref_stl(int m, int n, int k, int r, float *XA, float *XA2, int *alpha, float *XB,
                    float *XB2, int *beta, float *D, int *I);
void dgsknn_ref_stl(int m, int n, int k, int r, double *XA, double *XA2, int *alpha,
                    double *XB, double *XB2, int *beta, double *D, int *I);

/* =====================================================================================
 * Extensions (no counterpart in the reference)
 * ===================================================================================== */

/* Status of the calling thread's last call: 0 = ok, 1 = early return (m, n, d or k was 0,
 * as frame/gsknn.c:910-913), >= 2 = error; the string says what failed. */
int gsknn_last_error(void);
const char *gsknn_last_error_string(void);

/* Arithmetic of the float path of sgsknn / sgsknn_var1 / gsknn_s_device:
 *   GSKNN_MODE_FP32 -- CUDA-core FP32 distances;
 *   GSKNN_MODE_TF32, GSKNN_MODE_BF16 -- tensor-core distances with an FP64 re-rank of every
 *     candidate within the rounding bound of the k-th distance (exact index sets);
 *   GSKNN_MODE_AUTO -- from d = 128, BF16 (queries whose re-rank band overflows its log run
 *     again in split BF16); below d = 128, split BF16 (the narrowest band; plain BF16 overflows
 *     there); TF32 where neither fits in shared memory; else FP32 (default). Each choice was
 *     measured fastest of the exact forms on the d = 64 and d = 256 workloads. */
#define GSKNN_MODE_AUTO 0
#define GSKNN_MODE_FP32 1
#define GSKNN_MODE_TF32 2
#define GSKNN_MODE_BF16 3
#define GSKNN_MODE_BF16X3 4 /* split BF16: hi*hi + hi*lo + lo*hi, near-FP32 distances */
int gsknn_set_mode(int mode);
int gsknn_get_mode(void);

/* The tensor-core form on device pointers (roles and heaps as gsknn_s_device) in a given mode,
 * which additionally writes the approximate distance of every (query j, candidate i) pair to
 * C[j*ldc + i] (when C is not NULL) and each query's re-rank band 2E to margin[j] (when not
 * NULL): every approximate distance lies within E of the exact FP64 distance. For tests and
 * for callers that want the low-precision distance block itself. */
int gsknn_tc_distances(int mode, int m, int n, int d, int k, const float *XA, const float *XA2,
                       long long nA, const int *alpha, const float *XB, const float *XB2,
                       long long nB, const int *beta, float *D, int *I, int ldD, float *C,
                       long long ldc, float *margin, void *stream);

/* Device-pointer entry points, asynchronous on `stream` (a cudaStream_t; NULL = the legacy
 * default stream). Roles as in dgsknn: m candidates alpha[] of table XA (nA rows), n queries
 * beta[] of table XB (nB rows); D/I are n rows of stride ldD holding binary max-heaps of k
 * entries, updated in place. Indices outside a table are reported as an error (not read).
 * Scratch memory is taken from a per-(device, stream) cache owned by the library.
 * Returns 0 when the work was enqueued; call gsknn_stream_status(stream) after the stream has
 * drained to learn whether device-side checks failed. */
int gsknn_s_device(int m, int n, int d, int k, const float *XA, const float *XA2, long long nA,
                   const int *alpha, const float *XB, const float *XB2, long long nB,
                   const int *beta, float *D, int *I, int ldD, void *stream);
int gsknn_d_device(int m, int n, int d, int k, const double *XA, const double *XA2,
                   long long nA, const int *alpha, const double *XB, const double *XB2,
                   long long nB, const int *beta, double *D, int *I, int ldD, void *stream);

/* gsknn_s_device / gsknn_d_device with a distance type: KNN_2NORM (the squared 2-norm, as
 * gsknn_*_device) or KNN_1NORM, the sum over dimensions of |a_p - b_p|. The 1-norm is the
 * reference's rnn_r_1norm_int_d8x4_row.c kernel (declared by its knn_type enum, include/gsknn.h
 * :51-55, but never selected by its dispatch). Here it runs on the CUDA cores with an in-order
 * sum in the input precision, so double results equal the reference kernel's bit for bit (ties
 * to the lower id). For KNN_1NORM the norm arrays are not read and may be NULL. The same metric
 * is selected for sgsknn / dgsknn / dgsknn_var3 by a heap_t whose `type` is KNN_1NORM. */
int gsknn_s_device_metric(int type, int m, int n, int d, int k, const float *XA,
                          const float *XA2, long long nA, const int *alpha, const float *XB,
                          const float *XB2, long long nB, const int *beta, float *D, int *I,
                          int ldD, void *stream);
int gsknn_d_device_metric(int type, int m, int n, int d, int k, const double *XA,
                          const double *XA2, long long nA, const int *alpha, const double *XB,
                          const double *XB2, long long nB, const int *beta, double *D, int *I,
                          int ldD, void *stream);

/* Synchronises `stream` and returns the device-side status of the last call enqueued on it. */
int gsknn_stream_status(void *stream);

/* gsknn_s_device in GSKNN_MODE_FP32 (the CUDA-core FP32 pipeline) without any memory
 * allocation. No counterpart in the reference.
 *
 * For callers that must not allocate GPU memory while they run: a host program that hands all
 * of the GPU's memory to its own fixed arena or caching pool up front (a surprise cudaMalloc then
 * fails or evicts its cache), a latency-bound serving loop that cannot absorb cudaMalloc's cost
 * or cudaFree's implicit device synchronisation in the middle of a request, and plugin hosts
 * that forbid plugins from allocating device memory. Everything gsknn_s_device keeps in its
 * per-stream cache
 * here lives in one fixed 64 MiB array compiled into the library (each GPU that loads the
 * library holds it until the process exits). The call itself allocates nothing; inputs and
 * outputs are the caller's device buffers, with the same meaning as for gsknn_s_device.
 *
 * Limits and rules:
 *   - the packed problem must fit the fixed scratch: about (m + n) * round_up(d, 16) * 4 bytes
 *     of panels plus n * k * 8 bytes of partial lists; larger problems are rejected with
 *     GSKNN_ERR_UNSUPPORTED and a message (nothing is launched), use gsknn_s_device for them;
 *   - k <= 256 (the fused kernel's list size); larger k is rejected with
 *     GSKNN_ERR_UNSUPPORTED (gsknn_s_device takes it through its explicit-distance path);
 *   - the first call on a device looks up the array's device address (cudaGetSymbolAddress)
 *     with that device current and keeps it for the life of the process; make that first
 *     call before any stream capture, and do not use the entry point across a device reset
 *     (cudaDeviceReset), after which the kept address no longer names the array;
 *   - every call on a device shares the one array and it keeps the last call's contents:
 *     calls whose work may overlap on the GPU (different streams without ordering) race and
 *     corrupt each other's results; serialise them, e.g. on one stream;
 *   - `status` (device pointer, may be NULL) is cleared and then receives GSKNN_ERR_INDEX if
 *     an alpha/beta entry lies outside its table; with NULL the check still guards the reads
 *     but the error is not observable. gsknn_stream_status() does not cover this entry point
 *     (it reports the per-stream word of the caching entry points): pass `status` to see
 *     index errors.
 * Returns 0 when the work was enqueued on `stream`. */
int gsknn_s_device_noalloc(int m, int n, int d, int k, const float *XA, const float *XA2,
                           long long nA, const int *alpha, const float *XB, const float *XB2,
                           long long nB, const int *beta, float *D, int *I, int ldD, int *status,
                           void *stream);

/* Launch tracing: while enabled, every kernel the library launches is bracketed by CUDA events
 * on its stream. gsknn_trace_read() waits for the recorded launches, writes a JSON object
 * {"kernel": {"launches": n, "ms": total}, ...} into buf and clears the record; it returns the
 * number of launches read. */
void gsknn_trace_enable(int on);
int gsknn_trace_read(char *buf, int len);

/* Frees the library's cached device scratch memory of the current device. */
void gsknn_release_workspace(void);

/* ---- Batching form: all-nearest-neighbour search over randomized-tree leaves ---------------
 * No counterpart in the reference, whose tree drivers (frame/old/dgsrnn_directKQuery.cpp and
 * the rnn tree code) call dgsknn once per leaf with alpha = beta = the leaf's point list.
 *
 * A job owns device buffers for N points (table X, norms X2: device pointers, float) and
 * updates the caller's device heap D / I (N rows, row stride ldD >= k, initialised by the
 * caller, e.g. +inf / -1). Each pass takes the leaves of up to `trees_per_pass` trees over the
 * same points as host CSR arrays: leaf l holds leaf_pts[leaf_ptr[l] .. leaf_ptr[l+1]) and
 * belongs to tree leaf_tree[l] (a point appears at most once per tree). For every leaf, every
 * point of the leaf gets the leaf's points as candidates (itself included, at distance 0);
 * the pass's lists are merged into the heap with duplicates removed, so the heap converges to
 * the k nearest among every leaf-mate seen in any pass. Arithmetic: FP32 on the CUDA cores as
 * in sgsknn (ties to the lower id); rows are written in descending order (valid max-heaps).
 *
 * One pass is one persistent launch over all leaves (work items dealt by an atomic counter,
 * longest first), packed and merged by two more kernels, captured once in a CUDA graph and
 * replayed for every pass on `stream`. `leaf_min` bounds the smallest leaf (it sizes the
 * buffers); `shape` picks the tile shape (0: 128-row tiles, 1 and 2: 64-row tiles on the CUDA
 * cores; 3: the tensor-core shape) or, with -1, lets the autotuner time every shape on the
 * first pass of each (d, k, mean leaf size) class and remember the fastest for the process.
 * The tensor-core shape runs the precision form per tree: the tree's leaves laid out in one
 * split-BF16 panel (each leaf padded to whole 256-point tiles), every query tile against its own
 * leaf's tiles, and the exact FP64 re-rank merging straight into the heap rows, entering no id
 * twice; its results are the exact FP64 neighbours (the CUDA-core shapes give FP32 ones). It is
 * not open to jobs whose rows stand for global ids (the streaming form). Passes are asynchronous: gsknn_batch_pass
 * returns once the pass is enqueued (it waits only for the previous pass's plan upload);
 * gsknn_batch_sync waits and reports index errors. */
typedef struct gsknn_batch_s gsknn_batch_t;
gsknn_batch_t *gsknn_batch_create(int N, int d, int k, const float *X, const float *X2,
                                  float *D, int *I, int ldD, int trees_per_pass, int leaf_min,
                                  int shape, void *stream);
int gsknn_batch_pass(gsknn_batch_t *job, const int *leaf_ptr, const int *leaf_pts,
                     const int *leaf_tree, int nleaves);
int gsknn_batch_sync(gsknn_batch_t *job);
/* Shape in use, its tile rows, persistent grid, tiles / work items / distance evaluations of
 * the last pass, and (when this job ran the autotuner) the trial time of each of the 4 shapes
 * in ms (-1: not tried; tune_ms holds 4 entries). Any pointer may be NULL. */
int gsknn_batch_info(const gsknn_batch_t *job, int *shape, int *tile_rows, int *grid,
                     int *tiles, int *items, double *evals, float *tune_ms);
void gsknn_batch_destroy(gsknn_batch_t *job);
/* Forgets every tile shape the autotuner has chosen in this process. */
void gsknn_batch_forget_tuning(void);

/* ---- Serving form: requests against a device-resident reference set -----------------------
 * No counterpart in the reference (a caller would run sgsknn once per request).
 *
 * gsknn_serve_create prepares the nref x d float reference set R (device pointer, with norms
 * R2) once: packed for the tensor cores (mode AUTO / TF32 / BF16 / BF16X3) and resident until
 * destroy. In BF16 or TF32 the set is also packed in split BF16, where queries whose re-rank
 * band overflows finish. AUTO prepares BF16 with those split panels, times one probe batch of
 * resident points (k = max_k) both in BF16 and in split BF16 alone, and serves in the faster
 * (TF32 where split tiles do not fit); gsknn_serve_mode reports the choice. Each request is m query rows
 * (host memory, copied at submit) and a k <= max_k; its result is the exact FP64 top-k of every
 * query against R (ties to the lower id), as a heap of m rows x k (descending rows) that stays
 * on the device until the request is released.
 *
 * A dispatcher thread admits queued requests in arrival order while their heaps (m*k*8 bytes)
 * fit `heap_budget` bytes of device memory, packs admitted requests into batches and runs each
 * batch on one of `slots` streams: requests that arrive while a batch is on the GPU start in
 * the next free slot (continuous batching). A batch holds at most a slice of rows (a multiple
 * of 128, at most max_batch_queries), by default sized to about 3 ms of tensor work against
 * this reference set. A request of more rows runs as pieces over several batches, so m is
 * limited only by the heap budget. Whole requests that fit are packed first, and the oldest
 * larger request gets at least half of every batch. A request's result does not depend on its
 * batch or its pieces. Released requests return their heap memory to the budget; requests that
 * are never released keep it, and later requests then wait. */
typedef struct gsknn_serve_s gsknn_serve_t;
gsknn_serve_t *gsknn_serve_create(const float *R, const float *R2, int nref, int d, int mode,
                                  int max_batch_queries, int max_k, size_t heap_budget,
                                  int slots);
/* Returns the request id (>= 0), or minus an error code. */
long long gsknn_serve_submit(gsknn_serve_t *eng, const float *Q, int m, int k);
/* 1 done, 0 pending, negative: unknown request or failed. */
int gsknn_serve_test(gsknn_serve_t *eng, long long id);
int gsknn_serve_wait(gsknn_serve_t *eng, long long id, double timeout_s);
/* Device pointers of a finished request's heap (m x k floats, m x k ints). */
int gsknn_serve_heap(gsknn_serve_t *eng, long long id, float **D, int **I);
/* Copies a finished request's heap to host memory. */
int gsknn_serve_fetch(gsknn_serve_t *eng, long long id, float *D, int *I);
/* Milliseconds from submit to launch and from submit to completion; batch number and rows. */
int gsknn_serve_stats(gsknn_serve_t *eng, long long id, double *queue_ms, double *total_ms,
                      int *batch, int *batch_rows);
int gsknn_serve_release(gsknn_serve_t *eng, long long id);
/* Sets the rows per batch (rounded up to a multiple of 128, at most max_batch_queries; rows <= 0
 * restores the default) and returns the value in effect; applies to batches formed afterwards. */
int gsknn_serve_set_slice(gsknn_serve_t *eng, int rows);
/* While paused (nonzero) the dispatcher starts no new batch; requests still queue. Running
 * batches finish. Resuming dispatches everything queued in arrival order. */
int gsknn_serve_pause(gsknn_serve_t *eng, int paused);
/* The arithmetic the engine serves in (GSKNN_MODE_TF32 / BF16 / BF16X3) and, after an AUTO
 * choice, the probe batch's milliseconds in BF16 and in split BF16 (0 when not probed). */
int gsknn_serve_mode(gsknn_serve_t *eng, double *probe_bf16_ms, double *probe_bf16x3_ms);
void gsknn_serve_destroy(gsknn_serve_t *eng);

/* ---- Streaming form: the batching form for point sets beyond HBM ---------------------------
 * The point table X / X2 (N x d float, squared norms) and the heap D / I (N rows of stride
 * ldD >= k, initialised by the caller) are HOST memory: pageable, pinned, or a table mapped from
 * disk (gsknn_table_open). Each pass takes leaves exactly as gsknn_batch_pass does. The leaves of
 * a tree partition the points, so every tree is cut into groups of whole leaves of at most
 * `group_points` points. Each group's rows and heap rows are gathered by host threads, copied
 * to a device staging table of `group_points` rows, run through the batching pipeline, and
 * copied back. The next group is gathered while the current one runs. Results equal a resident
 * gsknn_batch_* job's after the same passes. A leaf larger than group_points is rejected.
 * Device memory: about group_points * (d + 2k + 2) * 4 bytes plus the staging batch job.
 * Calls block until the heaps are updated. */
typedef struct gsknn_stream_s gsknn_stream_t;
gsknn_stream_t *gsknn_stream_create(int N, int d, int k, const float *X, const float *X2,
                                    float *D, int *I, int ldD, int group_points, int leaf_min,
                                    int shape);
int gsknn_stream_pass(gsknn_stream_t *job, const int *leaf_ptr, const int *leaf_pts,
                      const int *leaf_tree, int nleaves);
/* Groups, bytes copied each way and the host time of the last pass. */
int gsknn_stream_info(const gsknn_stream_t *job, int *groups, double *h2d_bytes,
                      double *d2h_bytes, double *pass_ms);
void gsknn_stream_destroy(gsknn_stream_t *job);

/* On-disk point table for the streaming form: a 64-byte header ("GSKNNTB1", version 1, d, N,
 * offsets), the N x d float32 rows, then their N float32 squared 2-norms, little-endian.
 * gsknn_table_write writes one (norms from X2, or accumulated in double when X2 is NULL);
 * gsknn_table_open maps one read-only (NULL and a status if the file is not a valid table);
 * the row and norm pointers stay valid until gsknn_table_close. */
typedef struct gsknn_table_s gsknn_table_t;
int gsknn_table_write(const char *path, const float *X, const float *X2, long long N, int d);
gsknn_table_t *gsknn_table_open(const char *path);
long long gsknn_table_rows(const gsknn_table_t *t);
int gsknn_table_dim(const gsknn_table_t *t);
const float *gsknn_table_points(const gsknn_table_t *t);
const float *gsknn_table_norms(const gsknn_table_t *t);
void gsknn_table_close(gsknn_table_t *t);

/* Randomized projection trees on the host (the caller side of the batching form): `ntrees`
 * trees over the N x d row-major float points X. Each tree first draws leaf sizes uniformly in
 * [leaf_min, leaf_max] (leaf_max >= 2 leaf_min) that sum to N, then splits every node along a
 * random Gaussian direction at the rank that separates its leaves into two halves of nearly
 * equal size. Output: leaf_ptr (capacity max_leaves + 1), leaf_pts (ntrees * N entries),
 * leaf_tree (capacity max_leaves), *nleaves. Trees are built in parallel (`threads`, 0 = all
 * cores); the result depends only on `seed`. Returns 0, or GSKNN_ERR_ARG / GSKNN_ERR_UNSUPPORTED
 * (capacity too small). */
int gsknn_rkdt_leaves(const float *X, int N, int d, int ntrees, int leaf_min, int leaf_max,
                      unsigned long long seed, int threads, int *leaf_ptr, int *leaf_pts,
                      int *leaf_tree, int max_leaves, int *nleaves);

/* ---- Sorted-output adapters: replace frame/old/dgsrnn_directKQuery.cpp:14-135
 *      (dgsrnn_directKQuery) and 141-222 (dgsrnn_directKQuery_var2) ----
 * The reference returns std::pair<double, long> lists; a C ABI cannot, so each list is two
 * row-major m x k arrays: dist (squared distances) and id (64-bit point ids, -1 = none).
 *
 * gsknn_direct_kquery_d/_s(ref, query, n, m, k, dim, dist, id): all m queries (rows of `query`,
 * m x dim) against all n references (rows of `ref`, n x dim), norms computed here; row i of the
 * result is query i's k nearest references in ascending (distance, id) order, as the
 * reference's heap pops produce (dgsrnn_directKQuery.cpp:112-124; exact ties ordered by id).
 * With n < k the last entries are (largest finite value, -1), the reference's initial heap
 * (dgsrnn_directKQuery.cpp:50-53). Arithmetic as dgsknn_var1 / sgsknn_var1.
 *
 * gsknn_direct_kquery_maps_d/_s(m, n, dim, k, query, XA2, amap, ref, XB2, bmap, dist, id): the
 * _var2 form: queries amap[0..m) of `query` with norms XA2, references bmap[0..n) of `ref` with
 * norms XB2; rows left in heap order (max-heaps, descending here), as the reference copies them.
 *
 * Both take host pointers, block until done and return 0, GSKNN_EARLY_RETURN (a size is 0) or
 * an error code (also in gsknn_last_error()). */
int gsknn_direct_kquery_d(const double *ref, const double *query, long n, long m, long k,
                          long dim, double *dist, long *id);
int gsknn_direct_kquery_s(const float *ref, const float *query, long n, long m, long k, long dim,
                          float *dist, long *id);
int gsknn_direct_kquery_maps_d(int m, int n, int dim, int k, const double *query,
                               const double *XA2, const int *amap, const double *ref,
                               const double *XB2, const int *bmap, double *dist, long *id);
int gsknn_direct_kquery_maps_s(int m, int n, int dim, int k, const float *query,
                               const float *XA2, const int *amap, const float *ref,
                               const float *XB2, const int *bmap, float *dist, long *id);

/* Device heap rows to ascending lists in place: each of the n rows (stride ldk >= k) of D / I
 * is sorted ascending by (distance, id), ids compared as unsigned so -1 entries come last among
 * equal distances. k <= 512. Asynchronous on `stream`; returns 0 when enqueued. The device form
 * of the heap pops of dgsrnn_directKQuery.cpp:112-124, for heaps that stay on the GPU. */
int gsknn_heap_sort_s_device(float *D, int *I, int n, int k, int ldk, void *stream);
int gsknn_heap_sort_d_device(double *D, int *I, int n, int k, int ldk, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* GSKNN_B200_H */
