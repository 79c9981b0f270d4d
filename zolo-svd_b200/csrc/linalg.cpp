// Recursive Cholesky / triangular solves and the blocked structured Householder
// QR, expressed as DMMA GEMMs plus small leaf kernels.  See linalg.h.
#include "linalg.h"

#include <algorithm>
#include <string>

namespace zolo {

namespace {
constexpr int NB = kLeaf;  // leaf of the Cholesky / TRSM recursion
constexpr int PW = 32;     // Householder panel width
constexpr int QB = 128;    // Householder block: four panels, one rank-128 trailing update
constexpr int QA = 512;    // reflector block of ormqr under the INT8-emulated GEMM: K = 512 updates

int split_point(int n) {
  int n1 = ((n / 2) + NB - 1) / NB * NB;
  if (n1 >= n) n1 = n - NB;
  if (n1 <= 0) n1 = n / 2;
  return n1;
}
// Algorithmic flops of a product: lower triangle only (tri); k >= output column (kfrom_n); the
// triangular operand's zero k range skipped (kfrom_n / kto_m).
double algo_flops(int M, int N, int K, int tri, int kfrom_n, int kto_m) {
  double f = (tri ? 1.0 : 2.0) * M * static_cast<double>(N) * K;
  if (kfrom_n == 2) {
    // row i uses k >= i, over its lower-triangle (tri) or all N columns
    f = 0.0;
    for (int i = 0; i < std::min(M, K); ++i) f += 2.0 * (tri ? std::min(i + 1, N) : N) * (K - i);
  } else if (kfrom_n == 3) {
    // entry (i, j) uses k >= max(i, j) (no tri)
    f = 0.0;
    for (int i = 0; i < std::min(M, K); ++i) {
      const double jn = std::min(i + 1, N);  // columns j <= i: K - i each
      const double jm = std::max(0, std::min(N, K) - i - 1);  // columns i < j < K: K - j each
      f += 2.0 * (jn * (K - i) + jm * (K - i - 1) - jm * (jm - 1.0) / 2.0);
    }
  } else if (kfrom_n) {
    const double nn = std::min(N, K);
    f = 2.0 * M * (static_cast<double>(N) * K - nn * (nn - 1.0) / 2.0 - (N - nn) * static_cast<double>(K));
  }
  if (kto_m == 2) {
    // column j uses k <= j: sum over columns of min(K, j + 1)
    const double nn = std::min(N, K);
    f = 2.0 * M * (nn * (nn + 1.0) / 2.0 + (N - nn) * static_cast<double>(K));
  } else if (kto_m) {
    // row i uses k <= i: sum over rows of min(K, i + 1)
    const double mm = std::min(M, K);
    f = 2.0 * N * (mm * (mm + 1.0) / 2.0 + (M - mm) * static_cast<double>(K));
  }
  return f;
}
}  // namespace

namespace {
// Products the INT8-emulated GEMM takes while an OzScope is active: long enough K for its
// tile pipeline and at least two waves of 128 x 64 output tiles on the GPU (measured against
// the DMMA GEMM on square products: equal at n = 1024, one wave; 1.7x at n = 2048, 3.5 waves;
// 2.3x at n = 4096).
constexpr int kOzMinK = 256;
bool oz_eligible(int M, int N, int K, int batch, int tri) {
  if (K < kOzMinK || M <= 0 || N <= 0) return false;
  const int64_t tm = (M + 127) / 128, tn = (N + 63) / 64;
  int64_t tiles = tm * tn;
  if (tri) {
    tiles = 0;
    for (int64_t i = 0; i < tm; ++i) tiles += std::min<int64_t>(tn, 2 * i + 2);
  }
  return tiles * batch >= 2 * static_cast<int64_t>(num_sms());
}
}  // namespace

void gemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
          int batch, const double* alpha_vec, int tri, int kfrom_n, cudaStream_t st, int kto_m) {
  if (c.oz_active && !alpha_vec && oz_eligible(M, N, K, batch, tri)) {
    ozgemm(c, transA, transB, M, N, K, alpha, A, B, beta, C, batch, c.oz_active, tri, kfrom_n, st, kto_m);
    return;
  }
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
  cudaStream_t s = st ? st : c.stream();
  const bool side = s == c.side_stream() && s != c.stream();
  if (need) c.ensure_splitk(need, side);
  Profiler::Rec rec;
  const int cls = tri ? 6 : (M <= 32 ? 3 : (N <= 64 ? 4 : (K <= 64 ? 5 : (K <= 256 ? 8 : 0))));
  if (c.prof.on) {
    const double f = algo_flops(M, N, K, tri, kfrom_n, kto_m);
    c.prof.begin(cls, f * batch, s, &rec);
  }
  ck(dgemm(a, c.splitk(side), s));
  if (c.prof.on) c.prof.end(rec, s);
  c.stats.launches += need ? 2 : 1;
}

void ozgemm(Context& c, int transA, int transB, int M, int N, int K, double alpha, Mat A, Mat B, double beta, Mat C,
            int batch, int slices, int tri, int kfrom_n, cudaStream_t st, int kto_m) {
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
  a.batch = batch;
  a.tri = tri;
  a.kfrom_n = kfrom_n;
  a.kto_m = kto_m;
  if (!ozgemm_k_ok(slices, K)) {
    // exact INT32 accumulation bounds K: run K in chunks, accumulating into C (the
    // triangular k-skips refer to the whole K range and are dropped; zeros stay zeros)
    const int kc = 16384;
    for (int k0 = 0; k0 < K; k0 += kc) {
      const int kk = std::min(kc, K - k0);
      const Mat Ak{A.p + (transA ? k0 : static_cast<int64_t>(k0) * A.ld), A.ld, A.stride};
      const Mat Bk{B.p + (transB ? static_cast<int64_t>(k0) * B.ld : k0), B.ld, B.stride};
      ozgemm(c, transA, transB, M, N, kk, alpha, Ak, Bk, k0 == 0 ? beta : 1.0, C, batch, slices, tri, 0, st, 0);
    }
    return;
  }
  cudaStream_t s = st ? st : c.stream();
  const bool side = s == c.side_stream() && s != c.stream();
  const std::string pre = side ? "ozs_" : "oz_";
  OzWorkSizes sz;
  ozgemm_work_bytes(a, slices, &sz);
  OzWork w;
  w.sliceA = reinterpret_cast<int8_t*>(c.buf(pre + "sa", (sz.slice_a + 7) / 8));
  w.sliceB = reinterpret_cast<int8_t*>(c.buf(pre + "sb", (sz.slice_b + 7) / 8));
  unsigned long long* rows =
      reinterpret_cast<unsigned long long*>(c.buf(pre + "rows", (sz.rows_a + sz.rows_b) * 3 / 2 + 2));
  w.maxA = rows;
  w.maxB = rows + sz.rows_a;
  w.expA = reinterpret_cast<int*>(rows + sz.rows_a + sz.rows_b);
  w.expB = w.expA + sz.rows_a;
  w.status = c.oz_status_word();
  // profiled: class 9 from the start to the kernel's launch (splitting), class 7 the kernel
  Profiler::Rec split_rec, rec;
  const bool profile = c.prof.on && M > 0 && N > 0 && K > 0 && batch > 0;  // the kernel runs
  if (profile) {
    c.prof.begin(9, 0.0, s, &split_rec);
    rec.a = c.prof.take();
    rec.b = c.prof.take();
    rec.cls = 7;
    rec.flops = algo_flops(M, N, K, tri, kfrom_n, kto_m) * batch;
    w.before_kernel = split_rec.b;
    w.before_kernel2 = rec.a;
  }
  ck(zolo::ozgemm(a, slices, w, s, num_sms()));
  if (profile) {
    c.prof.recs.push_back(split_rec);
    c.prof.end(rec, s);
  }
  c.stats.launches += 3;
}

int oz_status(Context& c) {
  int* d = c.oz_status_word();
  int v = 0;
  ck(cudaMemcpyAsync(&v, d, sizeof(int), cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  if (v) ck(cudaMemsetAsync(d, 0, sizeof(int), c.stream()));
  return v;
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

// Cholesky and the inverse of its factor together: with L11 and Y11 = L11^{-1} from the
// first half, L21 = A21 Y11^T is one GEMM (no recursive triangular solve), then
// A22 -= L21 L21^T, the second half, and Y21 = -Y22 (L21 Y11).  n^3/3 + n^3/3 flops, as
// Cholesky plus triangular inverse, in about half the launches.
static void potrf_inv_rec(Context& c, int n, Mat A, Mat Y, int batch, int* dinfo, int off, DiagInv D, Mat Tmp) {
  if (n <= NB) {
    Profiler::Rec rec;
    if (c.prof.on) c.prof.begin(2, static_cast<double>(n) * n * n / 3.0 * batch, c.stream(), &rec);
    ck(potrf_leaf(n, A.p, A.ld, A.stride, batch, dinfo, off, D.block(off / NB), D.stride, c.stream()));
    if (c.prof.on) c.prof.end(rec, c.stream());
    ck(scale_copy(n, n, 1.0, D.block(off / NB), NB, D.stride, Y.p, Y.ld, Y.stride, batch, 0.0, c.stream()));
    c.stats.launches += 2;
    return;
  }
  const int n1 = split_point(n), n2 = n - n1;
  potrf_inv_rec(c, n1, A, Y, batch, dinfo, off, D, Tmp);
  // L21 = A21 Y11^T: Y11^T is upper triangular (k up to the column)
  ck(scale_copy(n2, n1, 1.0, A.at(n1, 0).p, A.ld, A.stride, Tmp.p, Tmp.ld, Tmp.stride, batch, 0.0, c.stream()));
  c.stats.launches++;
  gemm(c, 0, 1, n2, n1, n1, 1.0, Tmp, Y, 0.0, A.at(n1, 0), batch, nullptr, 0, 0, nullptr, 2);
  // A22 -= L21 L21^T (lower)
  gemm(c, 0, 1, n2, n2, n1, -1.0, A.at(n1, 0), A.at(n1, 0), 1.0, A.at(n1, n1), batch, nullptr, 1, 0);
  potrf_inv_rec(c, n2, A.at(n1, n1), Y.at(n1, n1), batch, dinfo, off + n1, D, Tmp);
  // Y21 = -Y22 (L21 Y11): Y11 lower (k from the column), Y22 lower (k up to the row)
  gemm(c, 0, 0, n2, n1, n1, 1.0, A.at(n1, 0), Y, 0.0, Tmp, batch, nullptr, 0, 1);
  gemm(c, 0, 0, n2, n1, n2, -1.0, Y.at(n1, n1), Tmp, 0.0, Y.at(n1, 0), batch, nullptr, 0, 0, nullptr, 1);
}

void potrf_inv(Context& c, int n, Mat A, Mat Y, int batch, int* dinfo, DiagInv D) {
  ck(set_identity(n, n, Y.p, Y.ld, Y.stride, batch, 0.0, c.stream()));  // zero upper triangle
  c.stats.launches++;
  const int64_t ldt = (n + 1) / 2 * 2;
  Mat Tmp{c.buf("potrf_inv_tmp", static_cast<size_t>(ldt) * n * batch), ldt, ldt * n};
  potrf_inv_rec(c, n, A, Y, batch, dinfo, 0, D, Tmp);
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

// P = V^T B over the panel rows (B starts at the panel's first row; V holds the rows packed)
static void panel_vt_b(Context& c, const PanelRows& R, int jb, int ncols, Mat V, Mat B, Mat P, int batch,
                       cudaStream_t st = nullptr) {
  gemm(c, 1, 0, jb, ncols, R.split, 1.0, V, B, 0.0, P, batch, nullptr, 0, 0, st);
  if (R.split < R.mp)
    gemm(c, 1, 0, jb, ncols, R.mp - R.split, 1.0, V.at(R.split, 0), B.at(static_cast<int>(R.split + R.gap), 0),
         1.0, P, batch, nullptr, 0, 0, st);
}

// B -= V P over the panel rows
static void panel_b_minus_vp(Context& c, const PanelRows& R, int jb, int ncols, Mat V, Mat P, Mat B, int batch,
                             cudaStream_t st = nullptr) {
  gemm(c, 0, 0, R.split, ncols, jb, -1.0, V, P, 1.0, B, batch, nullptr, 0, 0, st);
  if (R.split < R.mp)
    gemm(c, 0, 0, R.mp - R.split, ncols, jb, -1.0, V.at(R.split, 0), P, 1.0,
         B.at(static_cast<int>(R.split + R.gap), 0), batch, nullptr, 0, 0, st);
}

// T_B (jb x jb upper) of the block reflector I - V_B T_B V_B^T = H_1 H_2 ... of the block's
// 32-column panels (the compact WY recursion of LAPACK DLARFT, by panels): the diagonal
// blocks are the panels' T, and T_B(0:c0, q) = -T_B(0:c0, 0:c0) (V_B(:, 0:c0)^T V_q) T_q.
// VB: the block's explicit V, mp packed rows.  T: the first panel's T (32 x 32 per panel).
static void block_t(Context& c, int jb, Mat VB, int mp, const double* T, int64_t strideT, Mat TB, int batch) {
  const int ldg = std::max(jb, 2);
  Mat G{c.buf("qr_bg", static_cast<size_t>(ldg) * ldg * batch), ldg, static_cast<int64_t>(ldg) * ldg};
  Mat Tmp{c.buf("qr_btmp", static_cast<size_t>(ldg) * PW * batch), ldg, static_cast<int64_t>(ldg) * PW};
  // lower triangle of V_B^T V_B: its transpose gives the blocks above the diagonal
  gemm(c, 1, 0, jb, jb, mp, 1.0, VB, VB, 0.0, G, batch, nullptr, 1, 0);
  ck(block_t_init(jb, T, strideT, TB.p, TB.ld, TB.stride, batch, c.stream()));
  c.stats.launches++;
  for (int c0 = PW; c0 < jb; c0 += PW) {
    const int w = std::min(PW, jb - c0);
    // Tmp = T_B(0:c0, 0:c0) G(c0:c0+w, 0:c0)^T  (T_B upper: k from the row)
    gemm(c, 0, 1, c0, w, c0, 1.0, TB, G.at(c0, 0), 0.0, Tmp, batch, nullptr, 0, 2);
    gemm(c, 0, 0, c0, w, w, -1.0, Tmp, TB.at(c0, c0), 0.0, TB.at(0, c0), batch);
  }
}

// Householder QR in 128-column blocks of four 32-column panels.  Inside a block each panel
// updates only the block's remaining columns (rank-32); the trailing columns take one
// rank-128 update per block, C -= V_B (T_B^T (V_B^T C)), whose GEMMs have K = rows and
// K = 128.  Look-ahead: the next block's columns are updated first, then the next block is
// factored on the side stream while the main stream updates the rest.
void geqrf(Context& c, int mtot, int n, int m_top, Mat W, double* tau, double* T, int batch, bool top_tri) {
  const int npan = (n + PW - 1) / PW;
  const int64_t ldv = (mtot + 1) / 2 * 2;
  const int64_t strideT = static_cast<int64_t>(npan) * PW * PW;
  Mat Vp{c.buf("qr_v2", static_cast<size_t>(ldv) * PW * batch), ldv, ldv * PW};
  Mat Pp{c.buf("qr_p", static_cast<size_t>(PW) * QB * batch), PW, static_cast<int64_t>(PW) * QB};
  Mat VB{c.buf("qr_vb", static_cast<size_t>(ldv) * QB * batch), ldv, ldv * QB};
  Mat TB{c.buf("qr_tb", static_cast<size_t>(QB) * QB * batch), QB, static_cast<int64_t>(QB) * QB};
  Mat WB{c.buf("qr_wb", static_cast<size_t>(QB) * n * batch), QB, static_cast<int64_t>(QB) * n};
  Mat PB{c.buf("qr_pb", static_cast<size_t>(QB) * n * batch), QB, static_cast<int64_t>(QB) * n};
  cudaStream_t ms = c.stream(), ss = c.side_stream();
  auto factor_block = [&](int J, cudaStream_t st) {
    const int jend = std::min(n, J + QB);
    for (int j = J; j < jend; j += PW) {
      const int jb = std::min(PW, n - j);
      const int pj = j / PW;
      const PanelRows R = panel_rows(mtot, m_top, top_tri, j, jb);
      Profiler::Rec rec;
      if (c.prof.on) c.prof.begin(1, 2.0 * R.mp * static_cast<double>(jb) * jb * batch, st, &rec);
      ck(qr_panel(R.mp, jb, W.at(j, j).p, W.ld, W.stride, tau + j, n, T + pj * PW * PW, strideT, Vp.p, Vp.ld,
                  Vp.stride, batch, st, R.split, R.gap));
      if (c.prof.on) c.prof.end(rec, st);
      c.stats.launches++;
      const int nc = jend - j - jb;
      if (nc <= 0) continue;
      panel_vt_b(c, R, jb, nc, Vp, W.at(j, j + jb), Pp, batch, st);
      ck(apply_t(jb, nc, T + pj * PW * PW, strideT, Pp.p, Pp.ld, Pp.stride, 1, batch, st));
      c.stats.launches++;
      panel_b_minus_vp(c, R, jb, nc, Vp, Pp, W.at(j, j + jb), batch, st);
    }
  };
  factor_block(0, ms);
  for (int J = 0; J < n; J += QB) {
    const int jbB = std::min(QB, n - J);
    const int nc = n - J - jbB;
    if (nc <= 0) break;
    const PanelRows R = panel_rows(mtot, m_top, top_tri, J, jbB);
    ck(extract_v(R.mp, jbB, W.at(J, J).p, W.ld, W.stride, VB.p, VB.ld, VB.stride, batch, ms, R.split, R.gap));
    c.stats.launches++;
    block_t(c, jbB, VB, R.mp, T + (J / PW) * PW * PW, strideT, TB, batch);
    panel_vt_b(c, R, jbB, nc, VB, W.at(J, J + jbB), WB, batch, ms);
    // P = T_B^T (V_B^T C): T_B^T is lower triangular (k up to the row)
    gemm(c, 1, 0, jbB, nc, jbB, 1.0, TB, WB, 0.0, PB, batch, nullptr, 0, 0, ms, 1);
    const int jn = std::min(QB, nc);
    panel_b_minus_vp(c, R, jbB, jn, VB, PB, W.at(J, J + jbB), batch, ms);
    if (nc > jn) {
      ck(cudaEventRecord(c.event(0), ms));
      ck(cudaStreamWaitEvent(ss, c.event(0), 0));
      factor_block(J + jbB, ss);
      ck(cudaEventRecord(c.event(1), ss));
      panel_b_minus_vp(c, R, jbB, nc - jn, VB, PB.at(0, jn), W.at(J, J + jbB + jn), batch, ms);
      ck(cudaStreamWaitEvent(ms, c.event(1), 0));
    } else {
      factor_block(J + jbB, ms);
    }
  }
}

// Q = H_1 ... H_k applied to the identity, one 128-column block reflector at a time from the
// last block: Q(rows, J:nq) -= V_B (T_B (V_B^T Q(rows, J:nq))).  Columns left of J are still
// identity columns with their one above the block's rows, so V_B^T leaves them zero.
// C <- H_1 ... H_n C (the Q of geqrf applied from the left), one block reflector of `width`
// columns (a multiple of 32) at a time from the last: C(rows, cols) -= V_B (T_B (V_B^T
// C(rows, cols))), T_B merged from the 32-column panels' T (block_t).  Width 128 gives K = 128
// updates on the DMMA update tiles; 512 gives K = 512 products, which the INT8-emulated GEMM
// takes (K >= 256), for about 1 % more flops in the T product; on DMMA both widths measure
// the same.  from_diag: C starts as the identity, so block J touches columns J .. ncols-1 only
// (left of J they are identity columns with their one above the block's rows, which V_B^T
// leaves zero).
static void apply_q_blocks(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat C, int ncols,
                           bool from_diag, int batch, bool top_tri, int width) {
  const int npan = (n + PW - 1) / PW;
  const int64_t ldv = (mtot + 1) / 2 * 2;
  const int64_t strideT = static_cast<int64_t>(npan) * PW * PW;
  const int bw = std::min(width, (n + PW - 1) / PW * PW);
  Mat VB{c.buf("qr_vb", static_cast<size_t>(ldv) * bw * batch), ldv, ldv * bw};
  Mat TB{c.buf("qr_tb", static_cast<size_t>(bw) * bw * batch), bw, static_cast<int64_t>(bw) * bw};
  Mat WB{c.buf("qr_wb", static_cast<size_t>(bw) * ncols * batch), bw, static_cast<int64_t>(bw) * ncols};
  Mat PB{c.buf("qr_pb", static_cast<size_t>(bw) * ncols * batch), bw, static_cast<int64_t>(bw) * ncols};
  const int nblk = (n + bw - 1) / bw;
  for (int b = nblk - 1; b >= 0; --b) {
    const int J = b * bw;
    const int jbB = std::min(bw, n - J);
    const PanelRows R = panel_rows(mtot, m_top, top_tri, J, jbB);
    const int c0 = from_diag ? J : 0;
    const int nc = ncols - c0;
    ck(extract_v(R.mp, jbB, W.at(J, J).p, W.ld, W.stride, VB.p, VB.ld, VB.stride, batch, c.stream(), R.split,
                 R.gap));
    c.stats.launches++;
    block_t(c, jbB, VB, R.mp, T + (J / PW) * PW * PW, strideT, TB, batch);
    panel_vt_b(c, R, jbB, nc, VB, C.at(J, c0), WB, batch);
    // P = T_B (V_B^T C): T_B is upper triangular (k from the row)
    gemm(c, 0, 0, jbB, nc, jbB, 1.0, TB, WB, 0.0, PB, batch, nullptr, 0, 2);
    panel_b_minus_vp(c, R, jbB, nc, VB, PB, C.at(J, c0), batch);
  }
}

void orgqr(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat Q, int batch, int nq, bool top_tri) {
  if (nq < n) nq = n;
  ck(set_identity(mtot, nq, Q.p, Q.ld, Q.stride, batch, 1.0, c.stream()));
  c.stats.launches++;
  apply_q_blocks(c, mtot, n, m_top, W, T, Q, nq, true, batch, top_tri, QB);
}

void ormqr_left(Context& c, int mtot, int n, int m_top, Mat W, const double* T, Mat C, int ncols, int batch,
                bool top_tri) {
  if (ncols <= 0) return;
  apply_q_blocks(c, mtot, n, m_top, W, T, C, ncols, false, batch, top_tri, c.oz_active ? QA : QB);
}

}  // namespace zolo
