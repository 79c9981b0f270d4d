// Recursive Cholesky / triangular solves and the blocked structured Householder
// QR, expressed as DMMA GEMMs plus small leaf kernels.  See linalg.h.
#include "linalg.h"

#include <algorithm>

namespace zolo {

namespace {
constexpr int NB = kLeaf;  // leaf of the Cholesky / TRSM recursion
constexpr int PW = 32;     // Householder panel width

int split_point(int n) {
  int n1 = ((n / 2) + NB - 1) / NB * NB;
  if (n1 >= n) n1 = n - NB;
  if (n1 <= 0) n1 = n / 2;
  return n1;
}
}  // namespace

void gemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
          int batch, const double* alpha_vec, int tri, int kfrom_n, cudaStream_t st, int kto_m) {
  GemmArgs a;
  a.M = M;
  a.N = N;
  a.K = K;
  a.transA = transA;
  a.transB = transB;
  a.A = A.p;
  a.lda = A.ld;
  a.strideA = A.stride;
  a.B = B.p;
  a.ldb = B.ld;
  a.strideB = B.stride;
  a.C = C.p;
  a.ldc = C.ld;
  a.strideC = C.stride;
  a.alpha = alpha;
  a.beta = beta;
  a.alpha_vec = alpha_vec;
  a.batch = batch;
  a.tri = tri;
  a.kfrom_n = kfrom_n;
  a.kto_m = kto_m;
  const size_t need = dgemm_splitk_bytes(a, num_sms());
  if (need) c.ensure_splitk(need);
  cudaStream_t s = st ? st : c.stream();
  Profiler::Rec rec;
  const int cls = tri ? 6 : (M <= 32 ? 3 : (N <= 64 ? 4 : (K <= 64 ? 5 : 0)));
  if (c.prof.on) {
    // algorithmic flops: lower triangle only (tri); k >= output column (kfrom_n)
    double f = (tri ? 1.0 : 2.0) * M * static_cast<double>(N) * K;
    if (kfrom_n == 2) {
      // row i uses k >= i, over its lower-triangle (tri) or all N columns
      f = 0.0;
      for (int i = 0; i < std::min(M, K); ++i) f += 2.0 * (tri ? std::min(i + 1, N) : N) * (K - i);
    } else if (kfrom_n) {
      const double nn = std::min(N, K);
      f = 2.0 * M * (static_cast<double>(N) * K - nn * (nn - 1.0) / 2.0 - (N - nn) * static_cast<double>(K));
    }
    if (kto_m) {
      // row i uses k <= i: sum over rows of min(K, i + 1)
      const double mm = std::min(M, K);
      f = 2.0 * N * (mm * (mm + 1.0) / 2.0 + (M - mm) * static_cast<double>(K));
    }
    c.prof.begin(cls, f * batch, s, &rec);
  }
  ck(dgemm(a, c.splitk(), s));
  if (c.prof.on) c.prof.end(rec, s);
  c.stats.launches += need ? 2 : 1;
}

static void potrf_rec(Context& c, int n, Mat A, int batch, int* dinfo, int off, DiagInv D) {
  if (n <= NB) {
    Profiler::Rec rec;
    if (c.prof.on) c.prof.begin(2, static_cast<double>(n) * n * n / 3.0 * batch, c.stream(), &rec);
    ck(potrf_leaf(n, A.p, A.ld, A.stride, batch, dinfo, off, D.block(off / NB), D.stride, c.stream()));
    if (c.prof.on) c.prof.end(rec, c.stream());
    c.stats.launches++;
    return;
  }
  const int n1 = split_point(n), n2 = n - n1;
  potrf_rec(c, n1, A, batch, dinfo, off, D);
  // A21 <- A21 L11^{-T}  (out of place through a scratch copy)
  const int64_t ldt = (n2 + 1) / 2 * 2;
  Mat tmp{c.buf("potrf_tmp", static_cast<size_t>(ldt) * n1 * batch), ldt, ldt * n1};
  ck(scale_copy(n2, n1, 1.0, A.at(n1, 0).p, A.ld, A.stride, tmp.p, tmp.ld, tmp.stride, batch, 0.0, c.stream()));
  c.stats.launches++;
  trsm_rlt(c, n2, n1, A, tmp, A.at(n1, 0), batch, D, off / NB);
  // A22 -= A21 A21^T (lower)
  gemm(c, 0, 1, n2, n2, n1, -1.0, A.at(n1, 0), A.at(n1, 0), 1.0, A.at(n1, n1), batch, nullptr, 1, 0);
  potrf_rec(c, n2, A.at(n1, n1), batch, dinfo, off + n1, D);
}

void potrf(Context& c, int n, Mat A, int batch, int* dinfo, DiagInv D) {
  // size the scratch of the largest recursion level first (no growth mid-recursion)
  if (n > NB) {
    const int n1 = split_point(n), n2 = n - n1;
    c.buf("potrf_tmp", static_cast<size_t>((n2 + 1) / 2 * 2) * n1 * batch);
  }
  potrf_rec(c, n, A, batch, dinfo, 0, D);
}

void diag_inverses(Context& c, int n, Mat L, int batch, DiagInv D) {
  ck(trtri_blocks(n, L.p, L.ld, L.stride, D.p, batch, c.stream()));
  c.stats.launches++;
}

void trsm_rlt(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch, DiagInv D, int k0) {
  if (n <= NB) {
    Mat li{D.block(k0), NB, D.stride};
    gemm(c, 0, 1, m, n, n, 1.0, X, li, 0.0, Y, batch);
    return;
  }
  const int n1 = split_point(n), n2 = n - n1;
  trsm_rlt(c, m, n1, L, X, Y, batch, D, k0);
  gemm(c, 0, 1, m, n2, n1, -1.0, Y, L.at(n1, 0), 1.0, X.at(0, n1), batch);
  trsm_rlt(c, m, n2, L.at(n1, n1), X.at(0, n1), Y.at(0, n1), batch, D, k0 + n1 / NB);
}

void trsm_rln(Context& c, int m, int n, Mat L, Mat X, Mat Y, int batch, DiagInv D, int k0) {
  if (n <= NB) {
    Mat li{D.block(k0), NB, D.stride};
    gemm(c, 0, 0, m, n, n, 1.0, X, li, 0.0, Y, batch);
    return;
  }
  const int n1 = split_point(n), n2 = n - n1;
  trsm_rln(c, m, n2, L.at(n1, n1), X.at(0, n1), Y.at(0, n1), batch, D, k0 + n1 / NB);
  gemm(c, 0, 0, m, n1, n2, -1.0, Y.at(0, n1), L.at(n1, 0), 1.0, X, batch);
  trsm_rln(c, m, n1, L, X, Y, batch, D, k0);
}

// Rows of panel j (columns j .. j + jb - 1) in the mtot x n matrix: `mp`
// logical rows, of which the first `split` start at row j and the rest follow
// after `gap` skipped rows (gap = 0: one window).
struct PanelRows {
  int mp, split;
  int64_t gap;
};

static void trtri_rec(Context& c, int n, Mat L, Mat Y, int batch, DiagInv D, int k0, Mat Tmp) {
  if (n <= NB) {
    ck(scale_copy(n, n, 1.0, D.block(k0), NB, D.stride, Y.p, Y.ld, Y.stride, batch, 0.0, c.stream()));
    c.stats.launches++;
    return;
  }
  const int n1 = split_point(n), n2 = n - n1;
  trtri_rec(c, n1, L, Y, batch, D, k0, Tmp);
  trtri_rec(c, n2, L.at(n1, n1), Y.at(n1, n1), batch, D, k0 + n1 / NB, Tmp);
  // Y21 = -Y22 (L21 Y11): Y11 lower (k from the output column), Y22 lower (k up to the row)
  gemm(c, 0, 0, n2, n1, n1, 1.0, L.at(n1, 0), Y, 0.0, Tmp, batch, nullptr, 0, 1);
  gemm(c, 0, 0, n2, n1, n2, -1.0, Y.at(n1, n1), Tmp, 0.0, Y.at(n1, 0), batch, nullptr, 0, 0, nullptr, 1);
}

void trtri_lower(Context& c, int n, Mat L, Mat Y, int batch, DiagInv D) {
  ck(set_identity(n, n, Y.p, Y.ld, Y.stride, batch, 0.0, c.stream()));  // zero upper triangle
  c.stats.launches++;
  const int64_t ldt = (n + 1) / 2 * 2;
  Mat Tmp{c.buf("trtri_tmp", static_cast<size_t>(ldt) * n * batch), ldt, ldt * n};
  trtri_rec(c, n, L, Y, batch, D, 0, Tmp);
}

static inline PanelRows panel_rows(int mtot, int m_top, bool top_tri, int j, int jb) {
  const int hi = m_top >= 0 ? std::min(mtot, m_top + j + jb) : mtot;
  if (!top_tri || m_top < 0 || m_top <= j + jb) return PanelRows{hi - j, hi - j, 0};
  return PanelRows{jb + (hi - m_top), jb, static_cast<int64_t>(m_top) - j - jb};
}

// P = V^T B over the panel rows (B starts at the panel's first row)
static void panel_vt_b(Context& c, const PanelRows& R, int jb, int ncols, Mat V, Mat B, Mat P, int batch) {
  gemm(c, 1, 0, jb, ncols, R.split, 1.0, V, B, 0.0, P, batch);
  if (R.split < R.mp)
    gemm(c, 1, 0, jb, ncols, R.mp - R.split, 1.0, V.at(R.split, 0), B.at(static_cast<int>(R.split + R.gap), 0),
         1.0, P, batch);
}

// B -= V P over the panel rows
static void panel_b_minus_vp(Context& c, const PanelRows& R, int jb, int ncols, Mat V, Mat P, Mat B, int batch) {
  gemm(c, 0, 0, R.split, ncols, jb, -1.0, V, P, 1.0, B, batch);
  if (R.split < R.mp)
    gemm(c, 0, 0, R.mp - R.split, ncols, jb, -1.0, V.at(R.split, 0), P, 1.0,
         B.at(static_cast<int>(R.split + R.gap), 0), batch);
}

void geqrf(Context& c, int mtot, int n, int m_top, Mat W, double* tau, double* T, int batch, bool top_tri) {
  const int npan = (n + PW - 1) / PW;
  const int64_t ldv = (mtot + 1) / 2 * 2;
  // explicit V of consecutive panels alternates between two buffers (look-ahead)
  double* vb = c.buf("qr_v2", static_cast<size_t>(ldv) * PW * batch * 2);
  Mat V[2] = {Mat{vb, ldv, ldv * PW}, Mat{vb + ldv * PW * batch, ldv, ldv * PW}};
  Mat P{c.buf("qr_p", static_cast<size_t>(PW) * n * batch), PW, static_cast<int64_t>(PW) * n};
  const int64_t strideT = static_cast<int64_t>(npan) * PW * PW;
  cudaStream_t ms = c.stream(), ss = c.side_stream();
  auto panel = [&](int pj, cudaStream_t st) {
    const int j = pj * PW;
    const int jb = std::min(PW, n - j);
    const PanelRows R = panel_rows(mtot, m_top, top_tri, j, jb);
    Profiler::Rec rec;
    if (c.prof.on) c.prof.begin(1, 2.0 * R.mp * static_cast<double>(jb) * jb * batch, st, &rec);
    ck(qr_panel(R.mp, jb, W.at(j, j).p, W.ld, W.stride, tau + j, n, T + pj * PW * PW, strideT, V[pj & 1].p,
                V[pj & 1].ld, V[pj & 1].stride, batch, st, R.split, R.gap));
    if (c.prof.on) c.prof.end(rec, st);
    c.stats.launches++;
  };
  panel(0, ms);
  for (int pj = 0; pj < npan; ++pj) {
    const int j = pj * PW;
    const int jb = std::min(PW, n - j);
    const PanelRows R = panel_rows(mtot, m_top, top_tri, j, jb);
    const int nc = n - j - jb;
    if (nc <= 0) break;
    const Mat& Vj = V[pj & 1];
    // P = T^T V^T W_trail
    panel_vt_b(c, R, jb, nc, Vj, W.at(j, j + jb), P, batch);
    ck(apply_t(jb, nc, T + pj * PW * PW, strideT, P.p, P.ld, P.stride, 1, batch, ms));
    c.stats.launches++;
    // next panel's columns first, then the panel on the side stream overlaps the rest
    const int jb2 = std::min(PW, nc);
    panel_b_minus_vp(c, R, jb, jb2, Vj, P, W.at(j, j + jb), batch);
    const bool overlap = nc > jb2;
    if (overlap) {
      ck(cudaEventRecord(c.event(0), ms));
      ck(cudaStreamWaitEvent(ss, c.event(0), 0));
      panel(pj + 1, ss);
      ck(cudaEventRecord(c.event(1), ss));
      panel_b_minus_vp(c, R, jb, nc - jb2, Vj, P.at(0, jb2), W.at(j, j + jb + jb2), batch);
      ck(cudaStreamWaitEvent(ms, c.event(1), 0));
    } else {
      panel(pj + 1, ms);
    }
  }
}

void orgqr(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat Q, int batch, int nq, bool top_tri) {
  if (nq < n) nq = n;
  const int npan = (n + PW - 1) / PW;
  const int64_t ldv = (mtot + 1) / 2 * 2;
  Mat V{c.buf("qr_v2", static_cast<size_t>(ldv) * PW * batch * 2), ldv, ldv * PW};
  Mat P{c.buf("qr_p", static_cast<size_t>(PW) * nq * batch), PW, static_cast<int64_t>(PW) * nq};
  const int64_t strideT = static_cast<int64_t>(npan) * PW * PW;
  ck(set_identity(mtot, nq, Q.p, Q.ld, Q.stride, batch, 1.0, c.stream()));
  c.stats.launches++;
  for (int pj = npan - 1; pj >= 0; --pj) {
    const int j = pj * PW;
    const int jb = std::min(PW, n - j);
    const PanelRows R = panel_rows(mtot, m_top, top_tri, j, jb);
    const int nc = nq - j;
    ck(extract_v(R.mp, jb, W.at(j, j).p, W.ld, W.stride, V.p, V.ld, V.stride, batch, c.stream(), R.split, R.gap));
    c.stats.launches++;
    panel_vt_b(c, R, jb, nc, V, Q.at(j, j), P, batch);
    ck(apply_t(jb, nc, T + pj * PW * PW, strideT, P.p, P.ld, P.stride, 0, batch, c.stream()));
    c.stats.launches++;
    panel_b_minus_vp(c, R, jb, nc, V, P, Q.at(j, j), batch);
  }
}

}  // namespace zolo
