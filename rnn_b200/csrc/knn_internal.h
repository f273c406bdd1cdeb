// knn_internal.h -- internal interfaces between the C-ABI layer and the CUDA kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

// Status codes (also reported through gsknn_last_error()).
#define GSKNN_OK 0
#define GSKNN_EARLY_RETURN 1     // m, n, d or k was 0: nothing to do (frame/gsknn.c:910-913)
#define GSKNN_ERR_ARG 2          // invalid argument
#define GSKNN_ERR_CUDA 3         // a CUDA runtime call failed
#define GSKNN_ERR_INDEX 4        // an alpha/beta entry lies outside the point table
#define GSKNN_ERR_UNSUPPORTED 5  // size outside what this library supports
#define GSKNN_ERR_NOMEM 6        // device memory exhausted
#define GSKNN_ERR_TIMEOUT 7      // a bounded device-side wait gave up

namespace gsknn {

// Sets the calling thread's status (read by gsknn_last_error / gsknn_last_error_string) and
// returns `code`; fmt == nullptr means "ok".
int set_status(int code, const char *fmt, ...);

struct SimtGeom {
  int kp;      // list length (power of two >= k, >= 32), 0 when k is unsupported
  int bq, br;  // queries / candidates per CTA tile
  int dk;      // dimension chunk
  size_t smem;
  int nthr;
  int minb;  // resident CTAs per SM the kernel is built for
};

template <typename T>
struct SimtArgs {
  const T *Apack;        // query panels [qtiles][nkc][DK][BQ]
  const T *Bpack;        // candidate panels [rtiles][nkc][DK][BR]
  const T *qn;           // packed query norms [qtiles*BQ]
  const T *cn;           // packed candidate norms [rtiles*BR] (NaN past the end)
  const uint32_t *cid;   // packed candidate ids [rtiles*BR]
  const T *Din;          // incoming heap (for the initial threshold), may be null
  int ldD;
  int Q, k, nkc;
  int ntiles_r, tiles_per_split;
  T *partD;              // [S][Q][k] sorted ascending
  uint32_t *partI;
  int metric;            // 0: squared 2-norm, 1: 1-norm
};

template <typename T>
struct FinalizeArgs {
  const T *Din;          // incoming heap rows (may alias Dout), may be null
  const int *Iin;
  int ldD;
  int Q, k, S;
  const T *partD;
  const uint32_t *partI;
  T *Dout;
  int *Iout;
};

template <typename T>
cudaError_t launch_pack(const T *X, const T *X2, int d, long long nrows, const int *idx,
                        int count, int BT, int DK, int nkc, T *P, T *norms, uint32_t *ids,
                        int *status, cudaStream_t st);
template <typename T>
SimtGeom simt_geometry(int k);
template <typename T>
cudaError_t launch_simt(const SimtArgs<T> &a, int kp, int qtiles, int S, cudaStream_t st);
template <typename T>
cudaError_t launch_finalize(const FinalizeArgs<T> &a, int kp, cudaStream_t st);

// ---- explicit distance block + per-row selection (large k, var3, dgssq2nrm, *_ref) ----------
struct LargePlan {
  int nkc, qtiles, rtiles, chunk_rows;
  size_t o_ap, o_bp, o_qn, o_cn, o_cid, o_c, bytes, sel_smem;
};
template <typename T>
LargePlan large_plan(int nq, int nc, int d, int k, size_t max_block_bytes);
size_t large_select_smem(int k, size_t elem);
template <typename T>
cudaError_t large_run(const LargePlan &P, int nq, int nc, int d, int k, const T *Xq,
                      const T *Xq2, long long nrows_q, const int *qidx, const T *Xc,
                      const T *Xc2, long long nrows_c, const int *cidx, T *D, int *I, int ldD,
                      int four_ary, void *ws, int *status, cudaStream_t st,
                      int metric = 0);  // metric 1: the 1-norm (norms unused)
template <typename T>
cudaError_t block_run(const LargePlan &P, int nq, int nc, int d, const T *Xq, const T *Xq2,
                      long long nrows_q, const int *qidx, const T *Xc, const T *Xc2,
                      long long nrows_c, const int *cidx, T *Cout, long long ldc, void *ws,
                      int *status, cudaStream_t st);

// ---- tensor-core (tcgen05) precision form, float inputs ------------------------------------
// Arithmetic formats of the approximate pass (the public GSKNN_MODE_* values map onto them).
#define GSKNN_TC_TF32 2
#define GSKNN_TC_BF16 3
#define GSKNN_TC_BF16X3 4

// Kernel-launch bracket used by the library's tracer (begin/end around a group of launches);
// `nkernels` (read at the end) counts the library's own kernels launched inside the bracket.
typedef void (*TraceHook)(void *ctx, const char *name, bool begin, cudaStream_t st,
                          int nkernels);

// Epilogue warps of the tensor-core kernel: TC_EPI_WARPS / 4 per TMEM lane quarter, each with its
// own band log per (query, split) and its own heap of ceil(k/2) entries per row (the partition
// bound).
constexpr int TC_EPI_WARPS = 8;
constexpr int TC_EPI_PARTS = TC_EPI_WARPS / 4;

// Batching form: the rows of a job's table (a gsknn_batch_t) stand for global points gid[row]
// (device array of the job's N rows); lists and heaps then carry global ids (knn_batch.cu).
void batch_set_global_ids(void *job, const uint32_t *gid);

struct TcPlan {
  bool ok;
  int fmt, elem, d_pad, nkc, a_terms, b_terms, kp;
  int N, NST, qtiles, rtiles, q_pad, r_pad, S, tiles_per_split, logcap;
  unsigned smem;
  float coefA, coefB;
  // norm column (the candidate norms enter through the MMA): shared memory of that form (0: it
  // does not fit), and its error-bound coefficients (coefB is shared; coefC multiplies CN)
  unsigned smem_fold;
  float coefA_fold, coefC_fold, coefC;
  // query-side workspace offsets (absolute within the workspace; they start after the
  // prepared-candidate area when the plan includes it)
  size_t o_pa, o_pa_lo, o_qn, o_qnrm, o_log, o_logcnt, o_proot, o_margin, o_fbl, o_fbc;
  int hk;  // partition bound: heap entries per row and epilogue part
  size_t cand_bytes;  // prepared-candidate area at the start of the workspace (0: separate)
  // Escalation: queries whose band log overflowed in this format run again in a narrower one
  // (esc_mode, 0 = none: they go straight to the FP64 brute force). Its query-side workspace
  // starts at o_esc; o_ecand holds its candidate panels when the prepared candidates carry
  // none (packed only when some query overflowed).
  int esc_mode;
  size_t o_esc, o_ecand, esc_bytes, ecand_bytes;
  int sms, max_splits;  // the plan's arguments, to re-derive the escalation pass's plan
  size_t bytes;       // whole workspace
};

// Candidates packed once in the MMA input format, with everything a query batch needs from
// them: shift mu, |mu|^2, bound statistics (max centred norm, max |effective norm|), packed
// panels [r_pad][d_pad] (r_pad a multiple of 256), effective norms, centred norm bounds, ids,
// and the caller's table for the FP64 re-rank. A resident reference set is prepared once and
// serves any number of query batches.
struct TcCand {
  int fmt, elem, d, d_pad, nc, r_pad;
  float *mu;
  double *mu2;
  unsigned *stats;
  void *pb, *pb_lo;
  void *pn;  // norm panel (the MMA's norm column), null when absent
  float *cn, *cnrm;
  uint32_t *cid;
  const float *Xc, *Xc2;
  long long nrows_c;
  const int *cidx;
  // optional panels of the same candidates in a second format (escalation pass; shift, norms,
  // bounds and ids are shared with the first): efmt is a format of tc_format_of_mode, -1 when
  // absent
  int efmt;
  void *epb, *epb_lo, *epn;
};

int tc_format_of_mode(int mode);
// The narrower format a tensor-core mode escalates overflowed queries to (0: none).
int tc_escalation_mode(int nq, int nc, int d, int k, int mode, int sms);
size_t tc_cand_bytes(int nc, int d, int mode);
// Bytes of candidate panels in `mode`'s format alone (the escalation panels of a prepared set).
size_t tc_cand_panel_bytes(int nc, int d, int mode);
// Packs the escalation panels of prepared candidates C in `mode`'s format into `mem`.
cudaError_t tc_cand_prepare_escalation(TcCand *C, void *mem, int mode, int *status,
                                       cudaStream_t st);
cudaError_t tc_cand_prepare(TcCand *C, void *mem, int nc, int d, int mode, const float *Xc,
                            const float *Xc2, long long nrows_c, const int *cidx, int *status,
                            cudaStream_t st);

// with_cand: the workspace starts with the prepared-candidate area (tc_run); otherwise the
// plan covers the query side only (tc_run_prepared with separately prepared candidates).
// max_splits caps the candidate splits per query tile (0: the default, 16).
TcPlan tc_plan(int nq, int nc, int d, int k, int mode, int sms, bool with_cand = true,
               int max_splits = 0);
cudaError_t tc_run(const TcPlan &P, int nq, int nc, int d, int k, const float *Xq,
                   const float *Xq2, long long nrows_q, const int *qidx, const float *Xc,
                   const float *Xc2, long long nrows_c, const int *cidx, float *D, int *I,
                   int ldD, void *ws, int *status, float *dbg, long long dbg_ld,
                   unsigned long long *counters, cudaStream_t st, TraceHook hook,
                   void *hook_ctx);
// Tensor-core form of the batching pass (all-NN within randomized-tree leaves): one tree's
// leaves laid out in a panel, each leaf padded to whole candidate tiles; every query tile runs
// against its own leaf's tiles only, and the exact re-rank merges into the heap rows in place,
// entering no id twice (a point reached again by another tree or pass).
struct TcLeafPlan {
  bool ok;
  TcPlan P;        // the split-BF16 tile plan (one split), per-query area for rows_cap rows
  int rows_cap;    // panel rows one tree may need
  size_t o_mu, o_mu2, o_cpart, o_stats, o_pb, o_pb_lo, o_pn, o_cn, o_cnrm, o_cid, o_iota, bytes;
};
// npts: points of the table; rows_cap: panel rows one tree may use (a multiple of 128).
TcLeafPlan tc_leaf_plan(long long npts, int rows_cap, int d, int k, int sms);
// Candidate tile width of the leaf panels: every leaf starts at a multiple of it (0: no plan).
int tc_leaf_tile(int d, int k, int sms);
// One tree: pidx (rows entries: point or -1), qtab (nqt entries), rtab (rows / 128 entries);
// `setup` on the first call after the workspace was allocated (row index map and shift).
cudaError_t tc_leaf_pass(const TcLeafPlan &L, void *ws, const float *X, const float *X2,
                         long long npts, int d, int k, const int *pidx, int rows,
                         const int4 *qtab, int nqt, const int2 *rtab, float *D, int *I,
                         int ldD, int *status, cudaStream_t st, bool setup,
                         unsigned long long *counters = nullptr);

cudaError_t tc_run_prepared(const TcPlan &P, const TcCand &C, int nq, int d, int k,
                            const float *Xq, const float *Xq2, long long nrows_q,
                            const int *qidx, float *D, int *I, int ldD, void *ws, int *status,
                            float *dbg, long long dbg_ld, unsigned long long *counters,
                            cudaStream_t st, TraceHook hook, void *hook_ctx);

}  // namespace gsknn
