// MatrixMarket input of the reference's test drivers (prepare_matrix.f90:154-321
// prepare_real_GEM and :638-759 prepare_real_symm_MM) on one process: the coordinate
// entries of a MatrixMarket file are placed into a dense column-major matrix; a
// `symmetric` file (which stores one triangle) becomes the full symmetric matrix
// A + A^T with the diagonal halved, as the reference forms it with PDTRAN
// (prepare_matrix.f90:262-275, 730-742); a `general` file is used as stored.  The
// reference reads the file with the NIST mmio routine `mmread` (not in its tree); the
// parser here follows the published MatrixMarket exchange format: the banner line
// "%%MatrixMarket matrix <coordinate|array> <real|integer|double> <general|symmetric|...>",
// '%' comment lines, the size line, then the entries (1-based "i j value" for coordinate,
// column-major values for array).  A later duplicate of an entry replaces the earlier one,
// as the reference's assignment loop does (prepare_matrix.f90:251-260).
#include <cctype>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../include/zolo_b200.h"

namespace {

std::string lower(std::string s) {
  for (auto& ch : s) ch = static_cast<char>(std::tolower(static_cast<unsigned char>(ch)));
  return s;
}

struct MmFile {
  bool coordinate = true;
  int kind = 0;  // ZOLO_MM_GENERAL / _SYMMETRIC / _OTHER
  int m = 0, n = 0;
  int64_t nnz = 0;
};

// Reads the banner and size line; returns 0 or a negative error, the stream left at the entries.
int read_header(FILE* f, MmFile* h) {
  char line[1024];
  if (!std::fgets(line, sizeof line, f)) return -11;
  char b0[64] = {0}, obj[64] = {0}, fmt[64] = {0}, field[64] = {0}, sym[64] = {0};
  if (std::sscanf(line, "%63s %63s %63s %63s %63s", b0, obj, fmt, field, sym) != 5) return -11;
  if (lower(b0) != "%%matrixmarket" || lower(obj) != "matrix") return -11;
  const std::string F = lower(fmt), T = lower(field), S = lower(sym);
  if (F == "coordinate") {
    h->coordinate = true;
  } else if (F == "array") {
    h->coordinate = false;
  } else {
    return -12;
  }
  if (T != "real" && T != "double" && T != "integer") return -13;  // complex / pattern: no real values
  h->kind = S == "general" ? ZOLO_MM_GENERAL : (S == "symmetric" ? ZOLO_MM_SYMMETRIC : ZOLO_MM_OTHER);
  while (std::fgets(line, sizeof line, f)) {
    const char* p = line;
    while (*p == ' ' || *p == '\t') ++p;
    if (*p == '%' || *p == '\n' || *p == '\r' || *p == 0) continue;
    long long a = 0, b = 0, c = 0;
    if (h->coordinate) {
      if (std::sscanf(p, "%lld %lld %lld", &a, &b, &c) != 3) return -14;
      h->nnz = c;
    } else {
      // array: column-major values, only the lower triangle for a symmetric matrix
      if (std::sscanf(p, "%lld %lld", &a, &b) != 2) return -14;
      h->nnz = h->kind == ZOLO_MM_SYMMETRIC ? a * (a + 1) / 2 : a * b;
    }
    if (a < 0 || b < 0 || a > 0x7fffffff || b > 0x7fffffff || h->nnz < 0) return -14;
    h->m = static_cast<int>(a);
    h->n = static_cast<int>(b);
    return 0;
  }
  return -14;
}

}  // namespace

extern "C" int zolo_read_mm(const char* path, int* m, int* n, int* kind, double* a, int64_t lda) {
  if (!path || !m || !n) return -1;
  FILE* f = std::fopen(path, "r");
  if (!f) return -10;
  MmFile h;
  int rc = read_header(f, &h);
  if (rc == 0) {
    *m = h.m;
    *n = h.n;
    if (kind) *kind = h.kind;
    if (a) {
      if (lda < (h.m > 1 ? h.m : 1)) {
        rc = -6;
      } else {
        for (int j = 0; j < h.n; ++j)
          std::memset(a + static_cast<int64_t>(j) * lda, 0, sizeof(double) * h.m);
        long long ai = 1, aj = 1;  // next position of an array file (1-based)
        for (int64_t e = 0; e < h.nnz && rc == 0; ++e) {
          long long i = 0, j = 0;
          double v = 0.0;
          if (h.coordinate) {
            if (std::fscanf(f, "%lld %lld %lf", &i, &j, &v) != 3) rc = -15;
          } else {
            if (std::fscanf(f, "%lf", &v) != 1) rc = -15;
            i = ai;
            j = aj;
            if (++ai > h.m) {
              ++aj;
              ai = h.kind == ZOLO_MM_SYMMETRIC ? aj : 1;
            }
          }
          if (rc == 0 && (i < 1 || i > h.m || j < 1 || j > h.n)) rc = -16;
          if (rc == 0) a[(i - 1) + (j - 1) * lda] = v;
        }
        // symmetric: A <- A + A^T, diagonal halved (prepare_matrix.f90:262-275)
        if (rc == 0 && h.kind == ZOLO_MM_SYMMETRIC) {
          if (h.m != h.n) {
            rc = -17;
          } else {
            for (int j = 0; j < h.n; ++j)
              for (int i = j + 1; i < h.n; ++i) {
                const double s = a[i + static_cast<int64_t>(j) * lda] + a[j + static_cast<int64_t>(i) * lda];
                a[i + static_cast<int64_t>(j) * lda] = s;
                a[j + static_cast<int64_t>(i) * lda] = s;
              }
          }
        }
      }
    }
  }
  std::fclose(f);
  return rc;
}
