// gsknn_rkdt.cpp -- randomized projection trees on the host: the caller side of the batching
// form, which turns each tree's leaves into work for one persistent launch.
//
// The reference's tree drivers split point sets recursively and call dgsknn on every leaf
// (alpha = beta = leaf). Here a tree first draws its leaf sizes (uniform in [leaf_min,
// leaf_max], summing to N), then splits each node along a random Gaussian direction at the rank
// that gives its left child the first half of the node's leaves (by count), so leaves come out
// with exactly the drawn sizes and in depth-first order. Trees are independent (one seed each)
// and are built on parallel threads.
#include "gsknn.h"
#include "knn_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <thread>
#include <utility>
#include <vector>

namespace {

struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {  // splitmix64
    uint64_t z = (s += 0x9e3779b97f4a7c15ull);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
  double normal() {  // Box-Muller
    double u = uniform(), v = uniform();
    if (u < 1e-300) u = 1e-300;
    return std::sqrt(-2.0 * std::log(u)) * std::cos(6.283185307179586 * v);
  }
};

void draw_sizes(int N, int lmin, int lmax, Rng &r, std::vector<int> &sizes) {
  int rem = N;
  if (rem < lmin) {
    sizes.push_back(rem);
    return;
  }
  while (rem > 0) {
    if (rem <= lmax) {
      sizes.push_back(rem);
      break;
    }
    int s = lmin + (int)(r.next() % (uint64_t)(lmax - lmin + 1));
    if (rem - s < lmin) s = rem - lmin;  // leave a last leaf of at least lmin points
    sizes.push_back(s);
    rem -= s;
  }
}

struct TreeBuilder {
  const float *X;
  int d;
  Rng rng;
  const std::vector<int> &sizes;
  std::vector<long long> prefix;  // prefix[i] = sum of sizes[0..i)
  int *pts;                       // this tree's N point slots (leaf order on return)
  std::vector<std::pair<float, int>> buf;
  std::vector<float> dir;

  TreeBuilder(const float *X_, int d_, uint64_t seed, const std::vector<int> &sz, int *pts_)
      : X(X_), d(d_), rng(seed), sizes(sz), pts(pts_), dir(d_) {
    prefix.assign(sz.size() + 1, 0);
    for (size_t i = 0; i < sz.size(); i++) prefix[i + 1] = prefix[i] + sz[i];
  }

  // points pts[lo, hi) hold exactly leaves [a, b)
  void split(long long lo, long long hi, int a, int b) {
    if (b - a <= 1) return;
    const long long total = hi - lo;
    // leaf boundary m in (a, b) whose count to the left is closest to half of the node
    int m = a + 1;
    long long best = -1;
    for (int c = a + 1; c < b; c++) {
      const long long left = prefix[c] - prefix[a];
      const long long dev = std::llabs(2 * left - total);
      if (best < 0 || dev < best) {
        best = dev;
        m = c;
      }
    }
    const long long nleft = prefix[m] - prefix[a];
    for (int j = 0; j < d; j++) dir[j] = (float)rng.normal();
    buf.resize((size_t)total);
    for (long long i = 0; i < total; i++) {
      const int p = pts[lo + i];
      const float *x = X + (size_t)p * d;
      float s = 0.f;
      for (int j = 0; j < d; j++) s += x[j] * dir[j];
      buf[(size_t)i] = {s, p};
    }
    std::nth_element(buf.begin(), buf.begin() + nleft, buf.end());
    for (long long i = 0; i < total; i++) pts[lo + i] = buf[(size_t)i].second;
    split(lo, lo + nleft, a, m);
    split(lo + nleft, hi, m, b);
  }
};

}  // namespace

extern "C" int gsknn_rkdt_leaves(const float *X, int N, int d, int ntrees, int leaf_min,
                                 int leaf_max, unsigned long long seed, int threads,
                                 int *leaf_ptr, int *leaf_pts, int *leaf_tree, int max_leaves,
                                 int *nleaves) {
  if (!X || N <= 0 || d <= 0 || ntrees <= 0 || leaf_min <= 0 || leaf_max < 2 * leaf_min ||
      !leaf_ptr || !leaf_pts || !leaf_tree || !nleaves)
    return gsknn::set_status(GSKNN_ERR_ARG,
                             "gsknn_rkdt_leaves: invalid arguments (need leaf_max >= 2 leaf_min)");
  std::vector<std::vector<int>> sizes(ntrees);
  long long total_leaves = 0;
  for (int t = 0; t < ntrees; t++) {
    Rng r(seed * 0x2545F4914F6CDD1Dull + 0x1000 + (uint64_t)t);
    draw_sizes(N, leaf_min, leaf_max, r, sizes[t]);
    total_leaves += (long long)sizes[t].size();
  }
  if (total_leaves > max_leaves)
    return gsknn::set_status(GSKNN_ERR_UNSUPPORTED,
                             "gsknn_rkdt_leaves: %lld leaves exceed the capacity %d",
                             total_leaves, max_leaves);
  int nt = threads > 0 ? threads : (int)std::thread::hardware_concurrency();
  if (nt < 1) nt = 1;
  if (nt > ntrees) nt = ntrees;
  auto work = [&](int w) {
    for (int t = w; t < ntrees; t += nt) {
      int *pts = leaf_pts + (size_t)t * N;
      for (int i = 0; i < N; i++) pts[i] = i;
      TreeBuilder tb(X, d, seed * 0x9E3779B97F4A7C15ull + 0x77 + (uint64_t)t, sizes[t], pts);
      tb.split(0, N, 0, (int)sizes[t].size());
    }
  };
  std::vector<std::thread> pool;
  for (int w = 1; w < nt; w++) pool.emplace_back(work, w);
  work(0);
  for (auto &th : pool) th.join();
  int l = 0;
  for (int t = 0; t < ntrees; t++) {
    long long off = (long long)t * N;
    for (int s : sizes[t]) {
      leaf_ptr[l] = (int)off;
      leaf_tree[l] = t;
      off += s;
      l++;
    }
  }
  leaf_ptr[l] = (int)((long long)ntrees * N);
  *nleaves = l;
  return gsknn::set_status(GSKNN_OK, nullptr);
}
