// Batched FP64 dense linear algebra built from the DMMA GEMM and the leaf
// kernels.  Every routine works on `batch` column-major matrices laid out with
// a constant stride, runs on ctx.stream() and throws CudaFailure on error.
#pragma once
#include <cstdint>

#include "context.h"

namespace zolo {

struct Mat {
  double* p;
  int64_t ld;
  int64_t stride;  // between batch entries
  Mat at(int i, int j) const { return Mat{p + i + static_cast<int64_t>(j) * ld, ld, stride}; }
};

void gemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
          int batch, const double* alpha_vec = nullptr, int tri = 0, int kfrom_n = 0);

// Lower Cholesky in place (n x n), recursive; info[b] > 0 on failure (LAPACK convention).
void potrf(Context& c, int n, Mat A, int batch, int* dinfo);
// X(m x n) <- X L^{-T}   (out of place: X is destroyed, result in Y)
void trsm_rlt(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch);
// X(m x n) <- X L^{-1}   (out of place: X is destroyed, result in Y)
void trsm_rln(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch);

// Householder QR (in place, panels of 32) of the mtot x n matrices W.  With
// `m_top` >= 0 the matrix is the stack [X (m_top x n); D] where D is upper
// triangular: panel j only touches rows j .. m_top + j + 31 (mpdgeqrf.f).
// tau: n per batch entry; T: ceil(n/32) * 32 * 32 per batch entry.
void geqrf(Context& c, int mtot, int n, int m_top, Mat W, double* tau, double* T, int batch);
// Explicit Q (mtot x n) from the reflectors of geqrf (mpdorgqr.f / dorgqr).
void orgqr(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat Q, int batch);

}  // namespace zolo
