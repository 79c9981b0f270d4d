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

// Inverses of the 64 x 64 diagonal blocks of a lower-triangular factor:
// block k of batch entry b at p + b*stride + k*4096 (ld 64).
struct DiagInv {
  double* p;
  int64_t stride;
  double* block(int k) const { return p + static_cast<int64_t>(k) * 4096; }
};

constexpr int kLeaf = 64;
inline int nblocks(int n) { return (n + kLeaf - 1) / kLeaf; }

void gemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
          int batch, const double* alpha_vec = nullptr, int tri = 0, int kfrom_n = 0,
          cudaStream_t st = nullptr, int kto_m = 0);
// The same product with the FP64 multiplications emulated on the INT8 tensor cores
// (ozaki.cu): `slices` (6..8) digit planes per operand; no alpha_vec.  Runs on ctx.stream()
// or `st`; the digit planes live in the context's workspace ("oz_*", or "ozs_*" on the side
// stream).  A pipeline timeout is recorded in the context's oz status word (oz_status()).
void ozgemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
            int batch, int slices, int tri = 0, int kfrom_n = 0, cudaStream_t st = nullptr, int kto_m = 0);
// Reads (and clears) the oz status word: 0, or the code of the first pipeline timeout.
int oz_status(Context& c);
// Lower Cholesky in place (n x n), recursive; info[b] > 0 on failure (LAPACK convention).
// Dinv receives the inverses of the diagonal blocks of L (used by the solves below).
void potrf(Context& c, int n, Mat A, int batch, int* dinfo, DiagInv Dinv);
// Cholesky A = L L^T (lower, in place) and Y = L^{-1} (lower, upper triangle zero) together;
// D receives the leaves' diagonal-block inverses, dinfo LAPACK INFO per batch entry.
void potrf_inv(Context& c, int n, Mat A, Mat Y, int batch, int* dinfo, DiagInv D);
// Dinv for a lower-triangular L that did not come from potrf.
void diag_inverses(Context& c, int n, Mat L, int batch, DiagInv Dinv);
// Y = X L^{-T}  (X m x n is destroyed; L's diagonal block k has inverse Dinv.block(k0 + k))
void trsm_rlt(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch, DiagInv Dinv, int k0 = 0);
// Y = X L^{-1}
void trsm_rln(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch, DiagInv Dinv, int k0 = 0);
// Y = L^{-1} (lower triangular; Y's strictly upper triangle is set to zero), recursively:
// Y21 = -Y22 (L21 Y11), each product skipping the zero triangle of its triangular
// operand (n^3/3 flops); the 64 x 64 diagonal blocks are Dinv's.
void trtri_lower(Context& c, int n, Mat L, Mat Y, int batch, DiagInv Dinv);

// Householder QR (in place, panels of 32) of the mtot x n matrices W.  With
// `m_top` >= 0 the matrix is the stack [X (m_top rows); D] where D is upper
// triangular: panel j only touches rows j .. m_top + j + 31 (mpdgeqrf.f).
// With `top_tri` the top block is upper triangular too (its rows below n are
// zero): panel j then touches two row segments, j .. j + 31 and
// m_top .. m_top + j + 31, and the rows between them are skipped (the same
// arithmetic as the full stack, whose skipped rows are zero in the panel).
// m_top < 0: dense.
// tau: n per batch entry; T: ceil(n/32) * 32 * 32 per batch entry.
// The next panel is factored on a high-priority side stream while the rest of
// the trailing matrix is updated (look-ahead of depth 1).
void geqrf(Context& c, int mtot, int n, int m_top, Mat W, double* tau, double* T, int batch, bool top_tri = false);
// Explicit Q (mtot x nq, nq >= n; default nq = n) from the n reflectors of geqrf
// (mpdorgqr.f / dorgqr with N >= K).
void orgqr(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat Q, int batch, int nq = -1,
           bool top_tri = false);
// C (mtot x ncols) <- Q C with Q = H_1 ... H_n the reflectors of geqrf (dormqr 'L', 'N').
void ormqr_left(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat C, int ncols, int batch,
                bool top_tri = false);

}  // namespace zolo
