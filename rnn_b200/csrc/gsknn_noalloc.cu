// gsknn_noalloc.cu -- gsknn_s_device_noalloc: the float fused-kNN device entry point with all of
// its scratch memory in one fixed array inside the library, for callers that cannot allocate
// GPU memory while they run (see include/gsknn.h for who they are).
//
// The pipeline is the same pack -> fused select -> finalize sequence as gsknn_s_device; only
// the place the intermediate buffers live differs. Those buffers (the packed query and
// candidate panels, their norms and ids, the per-split partial neighbour lists and one status
// word) are carved out of g_noalloc_scratch below instead of the library's per-stream cache.
#include "gsknn.h"
#include "knn_internal.h"

#include <algorithm>
#include <mutex>

namespace gsknn {
int set_status(int code, const char *fmt, ...);
}

namespace {

// Fixed scratch: 64 MiB per GPU that loads the library, held until the process exits.
constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
void *g_scratch_addr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on the current device. In host code the symbol itself
// is only a host-side handle, so the address is looked up once per device, with that device
// current, and cached.
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return gsknn::set_status(GSKNN_ERR_CUDA, "cudaGetDevice failed: %s", cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return gsknn::set_status(GSKNN_ERR_UNSUPPORTED, "device ordinal %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p)
      return gsknn::set_status(GSKNN_ERR_CUDA, "cudaGetSymbolAddress(scratch) failed: %s",
                               cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return GSKNN_OK;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
  size_t oA, oB, oQN, oCN, oCI, oPD, oPI, oST, total;
};

Layout layout_for(const gsknn::SimtGeom &g, int nq, int nc, int nkc, int k, int S) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) { size_t o = off; off = align256(off + bytes); return o; };
  const int qtiles = (nq + g.bq - 1) / g.bq, rtiles = (nc + g.br - 1) / g.br;
  L.oA = take((size_t)qtiles * nkc * g.dk * g.bq * sizeof(float));
  L.oB = take((size_t)rtiles * nkc * g.dk * g.br * sizeof(float));
  L.oQN = take((size_t)qtiles * g.bq * sizeof(float));
  L.oCN = take((size_t)rtiles * g.br * sizeof(float));
  L.oCI = take((size_t)rtiles * g.br * 4);
  L.oPD = take((size_t)S * nq * k * sizeof(float));
  L.oPI = take((size_t)S * nq * k * 4);
  L.oST = take(sizeof(int));
  L.total = off;
  return L;
}

}  // namespace

extern "C" int gsknn_s_device_noalloc(int m, int n, int d, int k, const float *XA,
                                      const float *XA2, long long nA, const int *alpha,
                                      const float *XB, const float *XB2, long long nB,
                                      const int *beta, float *D, int *I, int ldD,
                                      int *status, void *stream) {
  using namespace gsknn;
  cudaStream_t st = (cudaStream_t)stream;
  const int nq = n, nc = m;
  if (nq == 0 || nc == 0 || d == 0 || k == 0)
    return set_status(GSKNN_EARLY_RETURN, "early return: m, n, d or k is 0");
  if (nq < 0 || nc < 0 || d < 0 || k < 0 || ldD < k)
    return set_status(GSKNN_ERR_ARG, "invalid sizes (m=%d n=%d d=%d k=%d ldD=%d)", m, n, d, k,
                      ldD);
  if (!XA || !XA2 || !alpha || !XB || !XB2 || !beta || !D || !I)
    return set_status(GSKNN_ERR_ARG, "null pointer argument");
  const SimtGeom g = simt_geometry<float>(k);
  if (g.kp == 0)
    return set_status(GSKNN_ERR_UNSUPPORTED, "k=%d exceeds the fused kernel's list size", k);
  const int nkc = (d + g.dk - 1) / g.dk;
  const int qtiles = (nq + g.bq - 1) / g.bq, rtiles = (nc + g.br - 1) / g.br;

  // Same wave balancing as the caching entry point, then fewer splits if the partial lists
  // would not fit in the fixed scratch.
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int S = 1;
  double best = 1e300;
  for (int s = 1; s <= std::min(rtiles, 64); s++) {
    const long long items = (long long)qtiles * s;
    const double cost = (double)((items + sms - 1) / sms) / s * (1.0 + 0.004 * s);
    if (cost < best - 1e-12) { best = cost; S = s; }
  }
  Layout L = layout_for(g, nq, nc, nkc, k, S);
  while (L.total > kNoAllocScratchBytes && S > 1) L = layout_for(g, nq, nc, nkc, k, --S);
  if (L.total > kNoAllocScratchBytes)
    return set_status(GSKNN_ERR_UNSUPPORTED,
                      "problem needs %zu bytes of scratch, more than the %zu-byte fixed scratch "
                      "of gsknn_s_device_noalloc (m=%d n=%d d=%d k=%d); use gsknn_s_device",
                      L.total, kNoAllocScratchBytes, m, n, d, k);

  void *base_v = nullptr;
  int rc = scratch_address(&base_v);
  if (rc != GSKNN_OK) return rc;
  char *base = static_cast<char *>(base_v);
  int *stw = status ? status : reinterpret_cast<int *>(base + L.oST);
  cudaError_t e = cudaMemsetAsync(stw, 0, sizeof(int), st);  // the only word that must start at 0
  float *Apack = reinterpret_cast<float *>(base + L.oA);
  float *Bpack = reinterpret_cast<float *>(base + L.oB);
  float *qn = reinterpret_cast<float *>(base + L.oQN);
  float *cn = reinterpret_cast<float *>(base + L.oCN);
  uint32_t *cid = reinterpret_cast<uint32_t *>(base + L.oCI);
  float *partD = reinterpret_cast<float *>(base + L.oPD);
  uint32_t *partI = reinterpret_cast<uint32_t *>(base + L.oPI);
  if (e == cudaSuccess)
    e = launch_pack<float>(XB, XB2, d, nB, beta, nq, g.bq, g.dk, nkc, Apack, qn, nullptr, stw,
                           st);
  if (e == cudaSuccess)
    e = launch_pack<float>(XA, XA2, d, nA, alpha, nc, g.br, g.dk, nkc, Bpack, cn, cid, stw, st);
  if (e == cudaSuccess) {
    SimtArgs<float> sa{};
    sa.Apack = Apack; sa.Bpack = Bpack; sa.qn = qn; sa.cn = cn; sa.cid = cid;
    sa.Din = D; sa.ldD = ldD; sa.Q = nq; sa.k = k; sa.nkc = nkc;
    sa.ntiles_r = rtiles; sa.tiles_per_split = (rtiles + S - 1) / S;
    sa.partD = partD; sa.partI = partI;
    e = launch_simt<float>(sa, g.kp, qtiles, S, st);
  }
  if (e == cudaSuccess) {
    FinalizeArgs<float> fa{};
    fa.Din = D; fa.Iin = I; fa.ldD = ldD; fa.Q = nq; fa.k = k; fa.S = S;
    fa.partD = partD; fa.partI = partI; fa.Dout = D; fa.Iout = I;
    e = launch_finalize<float>(fa, g.kp, st);
  }
  if (e != cudaSuccess)
    return set_status(GSKNN_ERR_CUDA, "gsknn_s_device_noalloc: launch failed: %s",
                      cudaGetErrorString(e));
  return set_status(GSKNN_OK, nullptr);
}
