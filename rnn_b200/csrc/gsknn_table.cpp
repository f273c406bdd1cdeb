// gsknn_table.cpp -- on-disk point table for the streaming form: a 64-byte header, the N x d
// float32 rows (row-major) and their N float32 squared 2-norms, little-endian. Tables are
// written once and memory-mapped read-only, so a streaming job gathers its groups' rows
// straight from the page cache.
//
//   offset  0  char[8]  magic "GSKNNTB1"
//           8  uint32   version (1)
//          12  uint32   d
//          16  uint64   N
//          24  uint64   byte offset of the rows (64)
//          32  uint64   byte offset of the norms (64 + N * d * 4)
//          40  uint64[3] zero
#include "gsknn.h"
#include "knn_internal.h"

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include <fcntl.h>
#include <sys/mman.h>
#include <sys/stat.h>
#include <unistd.h>

namespace {

struct TableHeader {
  char magic[8];
  uint32_t version, d;
  uint64_t N, rows_off, norms_off, reserved[3];
};
static_assert(sizeof(TableHeader) == 64, "header layout");

constexpr char kMagic[8] = {'G', 'S', 'K', 'N', 'N', 'T', 'B', '1'};

}  // namespace

struct gsknn_table_s {
  void *map;
  size_t bytes;
  long long N;
  int d;
  const float *X, *X2;
};

extern "C" {

int gsknn_table_write(const char *path, const float *X, const float *X2, long long N, int d) {
  using gsknn::set_status;
  if (!path || !X || N <= 0 || d <= 0)
    return set_status(GSKNN_ERR_ARG, "gsknn_table_write: invalid argument");
  std::FILE *f = std::fopen(path, "wb");
  if (!f) return set_status(GSKNN_ERR_ARG, "gsknn_table_write: cannot create %s", path);
  TableHeader h{};
  std::memcpy(h.magic, kMagic, 8);
  h.version = 1;
  h.d = (uint32_t)d;
  h.N = (uint64_t)N;
  h.rows_off = sizeof(TableHeader);
  h.norms_off = h.rows_off + (uint64_t)N * d * 4;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
            std::fwrite(X, sizeof(float) * (size_t)d, (size_t)N, f) == (size_t)N;
  // norms as given, or accumulated in double and rounded to float
  std::vector<float> buf;
  const long long chunk = 1 << 16;
  for (long long r0 = 0; ok && r0 < N; r0 += chunk) {
    const long long n = std::min(chunk, N - r0);
    buf.resize((size_t)n);
    for (long long i = 0; i < n; i++) {
      if (X2) {
        buf[(size_t)i] = X2[r0 + i];
      } else {
        double s = 0.0;
        const float *x = X + (size_t)(r0 + i) * d;
        for (int p = 0; p < d; p++) s += (double)x[p] * (double)x[p];
        buf[(size_t)i] = (float)s;
      }
    }
    ok = std::fwrite(buf.data(), sizeof(float), (size_t)n, f) == (size_t)n;
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) return set_status(GSKNN_ERR_ARG, "gsknn_table_write: writing %s failed", path);
  return set_status(GSKNN_OK, nullptr);
}

gsknn_table_t *gsknn_table_open(const char *path) {
  using gsknn::set_status;
  if (!path) {
    set_status(GSKNN_ERR_ARG, "gsknn_table_open: null path");
    return nullptr;
  }
  const int fd = ::open(path, O_RDONLY);
  if (fd < 0) {
    set_status(GSKNN_ERR_ARG, "gsknn_table_open: cannot open %s", path);
    return nullptr;
  }
  struct stat st {};
  TableHeader h{};
  const bool head_ok = ::fstat(fd, &st) == 0 && (size_t)st.st_size >= sizeof(h) &&
                       ::pread(fd, &h, sizeof(h), 0) == (ssize_t)sizeof(h);
  // sizes are checked before any product is formed, so no header can wrap the arithmetic:
  // d and N fit an int, and N * (d + 1) * 4 bytes (rows and norms) fits 63 bits
  const bool sizes_ok = head_ok && h.d > 0 && h.d <= 0x7fffffffULL && h.N > 0 &&
                        h.N <= 0x7fffffffULL &&
                        h.N <= ((uint64_t)1 << 62) / (4 * ((uint64_t)h.d + 1));
  const bool valid = sizes_ok && std::memcmp(h.magic, kMagic, 8) == 0 && h.version == 1 &&
                     h.rows_off == sizeof(h) &&
                     h.norms_off == h.rows_off + h.N * h.d * 4 &&
                     (uint64_t)st.st_size >= h.norms_off + h.N * 4;
  if (!valid) {
    ::close(fd);
    set_status(GSKNN_ERR_ARG, "gsknn_table_open: %s is not a point table of this format", path);
    return nullptr;
  }
  const size_t bytes = (size_t)(h.norms_off + h.N * 4);
  void *map = ::mmap(nullptr, bytes, PROT_READ, MAP_PRIVATE, fd, 0);
  ::close(fd);
  if (map == MAP_FAILED) {
    set_status(GSKNN_ERR_NOMEM, "gsknn_table_open: mapping %s failed", path);
    return nullptr;
  }
  gsknn_table_t *t = new gsknn_table_t;
  t->map = map;
  t->bytes = bytes;
  t->N = (long long)h.N;
  t->d = (int)h.d;
  t->X = reinterpret_cast<const float *>(static_cast<const char *>(map) + h.rows_off);
  t->X2 = reinterpret_cast<const float *>(static_cast<const char *>(map) + h.norms_off);
  set_status(GSKNN_OK, nullptr);
  return t;
}

long long gsknn_table_rows(const gsknn_table_t *t) { return t ? t->N : 0; }
int gsknn_table_dim(const gsknn_table_t *t) { return t ? t->d : 0; }
const float *gsknn_table_points(const gsknn_table_t *t) { return t ? t->X : nullptr; }
const float *gsknn_table_norms(const gsknn_table_t *t) { return t ? t->X2 : nullptr; }

void gsknn_table_close(gsknn_table_t *t) {
  if (!t) return;
  ::munmap(t->map, t->bytes);
  delete t;
}

}  // extern "C"
