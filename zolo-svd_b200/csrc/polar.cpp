// QDWH-PD (pqdwhfacs.f90:296-466, zolopd.f90:290-440) and Zolo-PD
// (pzolopd1.f90:280-487) on one GPU.  The iteration control is host scalar
// code identical to the reference; every matrix operation is one of the FP64
// kernels.  In Zolo-PD the r independent Zolotarev terms of an iteration are
// batched into the same launches (the reference runs them on r process
// groups and sums them with DGSUM2D); the sum is fused into the FormX2 kernel.
#include "polar.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <map>
#include <thread>
#include <vector>

#include "coeff.h"
#include "linalg.h"

namespace zolo {

namespace {

inline int64_t even(int64_t x) { return (x + 1) / 2 * 2; }

double d2h(Context& c, const double* d) {
  double v = 0.0;
  ck(cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  return v;
}

void h2d(Context& c, double* d, const double* h, int n) {
  ck(cudaMemcpyAsync(d, h, n * sizeof(double), cudaMemcpyHostToDevice, c.stream()));
}

int read_info(Context& c, int* dinfo, int count) {
  std::vector<int> h(count, 0);
  ck(cudaMemcpyAsync(h.data(), dinfo, count * sizeof(int), cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  for (int v : h)
    if (v != 0) return v;
  return 0;
}

int npanels(int n) { return (n + 31) / 32; }

// Host-side fault injection (ZOLO_OPT_INJECT_CHOL_FAIL = k + 1): the Cholesky-form step of
// iteration k reports a failed factorization (INFO = n + 1, beyond any real pivot index)
// and takes the recovery path, as a non-positive-definite shifted Gram would.
int injected_info(const Context& c, int it, int info) {
  return (c.inject_chol_fail == it + 1 && info == 0) ? 1000000 : info;
}

// With the mixed form on: 0, or -2000 - code when a pipeline wait of an INT8-emulated product
// timed out during the solve (its results are then not to be used).
int mixed_status(Context& c) {
  if (!c.zolo_mixed) return 0;
  const int st = oz_status(c);
  return st ? -2000 - st : 0;
}

// Newton-Schulz finish of Zolo-PD (ZOLO_OPT_NS_FINISH): entry threshold on
// ||X^T X - I||_F / sqrt(n) and the cap on the number of steps
constexpr double kNsEnter = 0.1;
constexpr int kNsMaxSteps = 12;

// Term plan of Zolo-PD on one GPU (ZOLO_OPT_TERM_PLAN).  The reference runs the r terms
// of an iteration on r process groups at once, so r costs it no time; on one GPU the terms
// run one after another and an iteration costs a fixed part plus r times a term.  Before
// each iteration the planner searches the term counts of the next iterations (up to three,
// then the Newton-Schulz finish) through the CON recursion and takes the first count of the
// cheapest sequence.  An iteration takes the QR form while CON > kConChol: the Cholesky form
// at CON solves with matrices of condition up to CON^2 and its error grows with it (measured
// backward errors 7e-15, 3e-14 and 5e-13 for a first Cholesky iteration at CON 2, 32 and 224).
// The coefficients come from compute_coeff_kp, exact at any CON, so the recursion predicts
// the iterate.  Costs in units of n^3 flops at the measured GEMM rate, from the kernel times
// at n = 8192; the parts that scale with m are multiplied by m/n.
constexpr double kConChol = 12.0;
class TermPlanner {
 public:
  // `mixed`: the Cholesky iterations and Newton-Schulz steps run their products on the
  // INT8-emulated GEMM (measured at n = 8192: a Cholesky iteration 39 ms + 11.5 ms per term,
  // a Newton-Schulz step 27 ms, the finish's first check 8 ms; 17 ms per unit)
  TermPlanner(int rk, int m, int n, double tol, bool mixed = false)
      : rk_(rk), mu_(static_cast<double>(m) / n), tol_(tol) {
    floor_e_ = std::max(1e-14, 0.5 * eps_precision() * std::sqrt(static_cast<double>(m)));
    if (mixed) {
      ch_term_ = 0.68;
      ch_fixed_ = 2.3;
      ns_step_ = 1.58;
      ns_entry_ = 0.48;
    }
  }
  // the plan from CON is the finish itself (no further iteration predicted)
  bool predicts_finish(double con) const { return 2.0 * (con - 1.0) <= 0.5 * kNsEnter; }
  // terms for the iteration at CON = con; `prefactored`: the QR of X is at hand (first iteration)
  int choose(double con, bool prefactored) {
    int first = rk_;
    plan(con, prefactored, 3, &first);
    return first;
  }
  // cost of the cheapest plan from CON at a Cholesky iteration whose Gram is already formed
  double cost_from(double con) { return plan(con, false, 3, nullptr) - (con > kConChol ? 0.0 : mu_ * ns_entry_); }
  // Newton-Schulz steps from a measured e to the rounding floor
  double ns_cost(double e) const { return mu_ * ns_step_ * ns_steps(e); }
  // CON after an iteration with r terms (the coefficients of compute_coeff_kp)
  double con_after(double con, int r) { return next_con(con, r); }
  // predicted Newton-Schulz steps once CON is within the finish threshold
  int finish_steps(double con) const { return ns_steps(2.0 * (con - 1.0)); }

 private:
  static constexpr double kQrTerm = 2.45, kQrFixedPre = 3.3, kQrOfX = 8.0;
  double ch_term_ = 1.05, ch_fixed_ = 4.3, ns_step_ = 2.95, ns_entry_ = 1.0;
  int rk_;
  double mu_, tol_, floor_e_;
  std::map<std::pair<double, int>, double> next_;

  double next_con(double con, int r) {
    const auto key = std::make_pair(con, r);
    const auto it = next_.find(key);
    if (it != next_.end()) return it->second;
    double cf[24];
    compute_coeff_kp(con, tol_, r, cf);
    const double v = zolo_next_con(con, cf, r, zolo_fone(cf, r));
    next_[key] = v;
    return v;
  }
  int ns_steps(double e) const {
    int k = 0;
    while (e > floor_e_ && k < kNsMaxSteps) {
      e = 0.75 * e * e;
      ++k;
    }
    return k;
  }
  double plan(double con, bool prefactored, int depth, int* first) {
    const double e = 2.0 * (con - 1.0);
    if (e <= 0.5 * kNsEnter) return mu_ * (ns_entry_ + ns_steps(e) * ns_step_);
    if (depth == 0) return 1e300;
    const bool qr = con > kConChol;
    const double fixed = qr ? mu_ * (kQrFixedPre + (prefactored ? 0.0 : kQrOfX)) : mu_ * ch_fixed_;
    double best = 1e300;
    for (int r = 1; r <= rk_; ++r) {
      const double here = fixed + r * (qr ? kQrTerm : ch_term_);
      if (here >= best) break;  // the cost of this iteration grows with r
      const double tot = here + plan(next_con(con, r), false, depth - 1, nullptr);
      if (tot < best) {
        best = tot;
        if (first) *first = r;
      }
    }
    return best;
  }
};

// Q1 * Q2^T of the explicit Q of the stacked matrix (Q2 starts at row mp, upper triangular).
void q1q2t(Context& c, int m, int mp, int n, Mat Qf, Mat Z, int batch) {
  gemm(c, 0, 1, m, n, n, 1.0, Qf, Qf.at(mp, 0), 0.0, Z, batch, nullptr, 0, 1);
}

// One Zolo-PD QR step with the QR of X shared by the r terms.  Each term of
// the reference's QR form (zoloqr.f90:99-111) is Q1_j Q2_j^T / sqrt(c_j) with
// [X; sqrt(c_j) I] = [Q1_j; Q2_j] R_j.  With X = Q_x R_x,
//   [X; sqrt(c_j) I] = diag(Q_x, I) [R_x; sqrt(c_j) I],
// so Q1_j = Q_x Q1'_j and Q2_j = Q2'_j where [Q1'_j; Q2'_j] is the Q factor of
// the stack of two upper-triangular n x n matrices.  That stack keeps the
// reference's row order (R_x on top: its rows are the Householder pivots; an
// interleaved order loses backward stability of the iteration), and panel j
// touches only rows j .. j+31 of R_x and rows 0 .. j+31 of sqrt(c_j) I.
// Result: Z(:, :, 0) = Q_x * sum_j w_j Q1'_j Q2'_j^T / FONE, w_j = hw[j].
// Flops: QR of X 4mn^2 - 4n^3/3, per term 4n^3/3 (structured QR and Q) + 2n^3/3
// (product of two triangular factors), and 2mn^2 for the final product -- against
// r (4mn^2 + n^3) for r independent (m+n) x n stacks.
// With `pf`, X = (the matrix pf factors) / scale: Q_x is pf's Q and R_x = R / scale, and
// d_sqrtc must already hold scale * sqrt(c_j) ([R/scale; sqrt(c) I] and [R; scale sqrt(c) I]
// have the same Q factor).
// s_only (with pf): Z receives S = sum_j w_j Q1'_j Q2'_j^T / FONE itself (n x n) and Q_x is
// never formed: the caller keeps the iterate as X = Q_x Y and updates Y.
void zolo_terms_shared_qr(Context& c, int m, int n, const double* X, int64_t ldx, Mat W, Mat Qf, Mat Z, double* tau,
                          double* T, const double* d_sqrtc, const double* hw, double fone, int rk,
                          const Prefactored* pf = nullptr, bool s_only = false, int m_canon = -1) {
  const int64_t ldn = even(n);
  Mat Xq{c.buf("zq_x", static_cast<size_t>(ldx) * n), ldx, 0};
  Mat Qx{c.buf("zq_q", static_cast<size_t>(ldx) * n), ldx, 0};
  if (pf) {
    Xq = Mat{const_cast<double*>(pf->W), pf->ldw, 0};
    if (!s_only) orgqr(c, m, n, -1, Xq, pf->T, Qx, 1);
  } else {
    ck(scale_copy(m, n, 1.0, X, ldx, 0, Xq.p, Xq.ld, 0, 1, 0.0, c.stream()));
    c.stats.launches++;
    geqrf(c, m, n, -1, Xq, tau, T, 1);
    orgqr(c, m, n, -1, Xq, T, Qx, 1);
  }
  // W and Qf hold r stacks of (m + n) x n with m >= n: room for r stacks [R_x; 0; sqrt(c_j) I]
  // of ldn + n rows (the identity block at the even row offset ldn)
  const int mt = static_cast<int>(ldn), mtot = mt + n;
  const int64_t lds = even(mtot);
  Mat Ws{W.p, lds, lds * n}, Qs{Qf.p, lds, lds * n};
  ck(form_stack(n, mt, n, Xq.p, Xq.ld, Ws.p, Ws.ld, Ws.stride, d_sqrtc, 0.0, rk, c.stream(), 1));
  c.stats.launches++;
  geqrf(c, mtot, n, mt, Ws, tau, T, rk, true);
  orgqr(c, mtot, n, mt, Ws, T, Qs, rk, -1, true);
  const bool direct = pf && s_only;
  Mat S = direct ? Mat{Z.p, Z.ld, 0} : Mat{c.buf("G", static_cast<size_t>(ldn) * n), ldn, 0};
  for (int b = 0; b < rk; ++b) {
    // S += w_b Q1'_b Q2'_b^T.  [R_x; sqrt(c) I] = Q'_b R_b gives Q1'_b = R_x R_b^{-1} and
    // Q2'_b = sqrt(c) R_b^{-1}, both upper triangular: entry (i, j) needs k >= max(i, j)
    const Mat Qb{Qs.p + b * Qs.stride, lds, 0};
    gemm(c, 0, 1, n, n, n, hw[b] / fone, Qb, Qb.at(mt, 0), b == 0 ? 0.0 : 1.0, S, 1, nullptr, 0, 3);
  }
  if (!direct) gemm(c, 0, 0, m, n, n, 1.0, Qx, S, 0.0, Mat{Z.p, Z.ld, 0}, 1);
  const double dm = m, dn = n;
  const double executed = direct ? rk * (2.0 * dn * dn * dn)
                                 : (pf ? 2.0 : 4.0) * dm * dn * dn - (pf ? 2.0 : 4.0) * dn * dn * dn / 3.0 +
                                       rk * (2.0 * dn * dn * dn) + 2.0 * dm * dn * dn;
  const double dmc = m_canon >= 0 ? m_canon : m;  // rows of the reference's stack [X; sqrt(c) I]
  c.stats.flops_exec_delta += executed - rk * (4.0 * dmc * dn * dn + dn * dn * dn);
}

// Finish of the polar iteration by FP64 Newton-Schulz steps X <- X (3I - X^T X)/2.
// e = ||X^T X - I||_F / sqrt(n) is measured before every step (the Gram is the step's
// own first half) and the steps stop once e reaches the rounding floor
// max(1e-14, eps sqrt(m) / 2), once a step no longer halves e (rounding level), after a
// step whose bound on the next e is below a tenth of the floor (its Gram is not formed), or
// after kNsMaxSteps.  Near convergence e -> 0.75 e^2; from e = 0.1 that is four steps.  On entry G holds the lower triangle of X^T X and e0 its
// e.  Records the steps as branch 3 after the `it` Zolo iterations.
void newton_schulz_finish(Context& c, int m, int n, double* X, int64_t ldx, Mat G, Mat Z, double e0, int it) {
  const double floor_e = std::max(1e-14, 0.5 * eps_precision() * std::sqrt(static_cast<double>(m)));
  double* scal = c.dscal();
  double e = e0, e_prev = 2.0 * e0 + 1.0;
  for (int k = 0; k < kNsMaxSteps && e > floor_e && e < 0.5 * e_prev; ++k) {
    e_prev = e;
    ck(ns_prepare(n, G.p, G.ld, c.dpartial(), scal + 2, 1, c.stream()));
    gemm(c, 0, 0, m, n, n, 1.0, Mat{X, ldx, 0}, G, 0.0, Mat{Z.p, Z.ld, 0}, 1);
    ck(scale_copy(m, n, 1.0, Z.p, Z.ld, 0, X, ldx, 0, 1, 0.0, c.stream()));
    c.stats.launches += 3;
    c.stats.flops += 2.0 * m * static_cast<double>(n) * n;
    const int slot = it + c.stats.ns_steps;
    if (slot < 16) {
      c.stats.branch[slot] = 3;
      c.stats.con[slot] = 1.0;
      c.stats.err[slot] = e;
    }
    c.stats.ns_steps++;
    // with d_i = sigma_i^2 - 1 a step maps d to -3/4 d^2 (1 - d/3), so the next e is at most
    // 3/4 e^2 sqrt(n) (1 + e sqrt(n)/3) plus the step's rounding: far below the floor, the next
    // Gram would only confirm the floor and is not formed
    const double rn = std::sqrt(static_cast<double>(n));
    if (0.75 * e * e * rn * (1.0 + e * rn / 3.0) <= 0.1 * floor_e) break;
    // the next Gram: the measurement that decides whether another step is needed
    gemm(c, 1, 0, n, n, m, 1.0, Mat{X, ldx, 0}, Mat{X, ldx, 0}, 0.0, G, 1, nullptr, 1, 0);
    ck(ns_prepare(n, G.p, G.ld, c.dpartial(), scal + 2, 0, c.stream()));
    c.stats.launches += 2;
    c.stats.flops += static_cast<double>(m) * n * n;
    e = std::sqrt(d2h(c, scal + 2) / n);
  }
  // the Gram that measured e0 was counted by the Cholesky branch's SYRK
  c.stats.flops += static_cast<double>(m) * n * n;
}

// Z(b) = X W_b^{-1} (left = false) or W_b^{-1} X (left = true, square X), W_b = L_b L_b^T.
// strideX: X of batch entry b at X + b*strideX (0: one X shared by the r terms); the left
// solve takes a shared X only.
void spd_solve(Context& c, int m, int n, const double* X, int64_t ldx, Mat Lw, DiagInv D, Mat Z, int batch,
               bool left, int64_t strideX = 0) {
  const int64_t ldm = even(m);
  Mat Xc{c.buf("Xc", static_cast<size_t>(ldm) * n * batch), ldm, ldm * n};
  Mat Y{c.buf("Y", static_cast<size_t>(ldm) * n * batch), ldm, ldm * n};
  if (!left) {
    ck(scale_copy(m, n, 1.0, X, ldx, strideX, Xc.p, Xc.ld, Xc.stride, batch, 0.0, c.stream()));
    c.stats.launches++;
    trsm_rlt(c, m, n, Lw, Xc, Y, batch, D);
    trsm_rln(c, m, n, Lw, Y, Z, batch, D);
    return;
  }
  // W^{-1} X = (X^T W^{-1})^T : transpose in, right solves, transpose out
  for (int b = 0; b < batch; ++b) {
    ck(transpose(m, n, X, ldx, Xc.p + b * Xc.stride, Xc.ld, c.stream()));
    c.stats.launches++;
  }
  trsm_rlt(c, n, m, Lw, Xc, Y, batch, D);
  trsm_rln(c, n, m, Lw, Y, Xc, batch, D);
  for (int b = 0; b < batch; ++b) {
    ck(transpose(n, m, Xc.p + b * Xc.stride, Xc.ld, Z.p + b * Z.stride, Z.ld, c.stream()));
    c.stats.launches++;
  }
}

}  // namespace

void form_h(Context& c, int m, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, double* dH,
            int64_t ldh) {
  const int64_t ldn = even(n);
  double* Hb = c.buf("Hbuf", static_cast<size_t>(ldn) * n);
  gemm(c, 1, 0, n, n, m, 1.0, Mat{const_cast<double*>(dQ), ldq, 0}, Mat{const_cast<double*>(dA), lda, 0}, 0.0,
       Mat{Hb, ldn, 0}, 1);
  ck(symmetrize(n, Hb, ldn, c.stream()));
  ck(scale_copy(n, n, 1.0, Hb, ldn, 0, dH, ldh, 0, 1, 0.0, c.stream()));
  c.stats.launches += 2;
  c.stats.flops += 2.0 * m * static_cast<double>(n) * n;
}

namespace {
// Guaranteed upper bound of ||R||_2 for an upper-triangular n x n R (the factor of A/alpha_F,
// so ||R||_2 <= ||R||_F = 1): the power method by repeated squaring, G = R^T R, G^2, G^4, and
// ||G^4||_F^(1/8) = (sum sigma_i^16)^(1/16) >= sigma_max; times 1 + 1e-4 against rounding,
// capped by 1.  The intent of the reference's broken pdnormest.f90:44-79 (a power iteration
// for ||A||_2), made a certain bound.  7n^3/3 flops.
double norm2_upper(Context& c, int n, const double* W, int64_t ldw) {
  const int64_t ldn = even(n);
  double* Ru = c.buf("n2_r", static_cast<size_t>(ldn) * n);
  double* G = c.buf("n2_g", static_cast<size_t>(ldn) * n);
  double* G2 = c.buf("n2_g2", static_cast<size_t>(ldn) * n);
  ck(copy_upper(n, W, ldw, 1.0, Ru, ldn, c.stream()));
  // G = R^T R: op(A) = R^T is lower triangular (k <= row)
  gemm(c, 1, 0, n, n, n, 1.0, Mat{Ru, ldn, 0}, Mat{Ru, ldn, 0}, 0.0, Mat{G, ldn, 0}, 1, nullptr, 1, 0, nullptr, 1);
  ck(mirror_lower(n, G, ldn, c.stream()));
  gemm(c, 0, 0, n, n, n, 1.0, Mat{G, ldn, 0}, Mat{G, ldn, 0}, 0.0, Mat{G2, ldn, 0}, 1, nullptr, 1, 0);
  ck(mirror_lower(n, G2, ldn, c.stream()));
  gemm(c, 0, 0, n, n, n, 1.0, Mat{G2, ldn, 0}, Mat{G2, ldn, 0}, 0.0, Mat{G, ldn, 0}, 1, nullptr, 1, 0);
  ck(mirror_lower(n, G, ldn, c.stream()));
  ck(frob2(n, n, G, ldn, c.dpartial(), c.dscal() + 5, c.stream()));
  c.stats.launches += 8;
  c.stats.flops += 7.0 / 3.0 * static_cast<double>(n) * n * n;
  const double f = d2h(c, c.dscal() + 5);  // ||G^4||_F^2 = sum sigma^16
  if (!(f > 0.0) || !std::isfinite(f)) return 1.0;
  return std::min(1.0, std::pow(f, 1.0 / 16.0) * (1.0 + 1e-4));
}
}  // namespace

int bounds(Context& c, int m, int n, double sigma, const double* dA, int64_t lda, BoundsMode mode, double* alpha,
           double* beta, double* alpha_fro) {
  const int64_t ldx = even(m), ldn = even(n);
  double* X = c.buf("bnd_x", static_cast<size_t>(ldx) * n);
  double* scal = c.dscal();
  double* part = c.dpartial();
  ck(scale_copy(m, n, 1.0, dA, lda, 0, X, ldx, 0, 1, -sigma, c.stream()));
  ck(frob2(m, n, X, ldx, part, scal, c.stream()));
  c.stats.launches += 3;
  const double a = std::sqrt(d2h(c, scal));
  *alpha = a;
  if (alpha_fro) *alpha_fro = a;
  if (!(a > 0.0) || !std::isfinite(a)) {
    *beta = 0.0;
    return 1;
  }
  ck(scale_copy(m, n, 1.0 / a, X, ldx, 0, X, ldx, 0, 1, 0.0, c.stream()));
  c.stats.launches++;
  double temp_beta = 1.0;
  if (mode == BOUNDS_PQDWHFACS) {
    double* colsum = c.buf("bnd_colsum", n);
    ck(norm1(m, n, X, ldx, colsum, scal + 1, c.stream()));
    c.stats.launches += 2;
    temp_beta = d2h(c, scal + 1);
  }
  // R of X = QR (unstructured Householder), then R^{-T} = (R^T)^{-1} by the blocked triangular
  // inverse and R^{-1} as its transpose for ||R^{-1}||_1 and ||R^{-1}||_F
  double* tau = c.buf("bnd_tau", n);
  double* T = c.buf("bnd_t", static_cast<size_t>(npanels(n)) * 1024);
  geqrf(c, m, n, -1, Mat{X, ldx, 0}, tau, T, 1);
  double* Lt = c.buf("bnd_lt", static_cast<size_t>(ldn) * n);
  double* I = c.buf("bnd_i", static_cast<size_t>(ldn) * n);
  double* Ri = c.buf("bnd_rinv", static_cast<size_t>(ldn) * n);
  ck(transpose(n, n, X, ldx, Lt, ldn, c.stream()));
  c.stats.launches++;
  DiagInv D{c.buf("bnd_dinv", static_cast<size_t>(nblocks(n)) * 4096), 0};
  diag_inverses(c, n, Mat{Lt, ldn, 0}, 1, D);
  trtri_lower(c, n, Mat{Lt, ldn, 0}, Mat{I, ldn, 0}, 1, D);
  ck(transpose(n, n, I, ldn, Ri, ldn, c.stream()));
  c.stats.launches++;
  double* colsum = c.buf("bnd_colsum", n);
  ck(norm1(n, n, Ri, ldn, colsum, scal + 2, c.stream()));
  ck(frob2(n, n, Ri, ldn, part, scal + 3, c.stream()));
  c.stats.launches += 4;
  const double inv1 = d2h(c, scal + 2);
  const double fr = d2h(c, scal + 3);
  c.stats.flops += 4.0 / 3.0 * static_cast<double>(n) * n * n + 2.0 * m * static_cast<double>(n) * n;
  if (!std::isfinite(fr) || !std::isfinite(inv1) || !(inv1 > 0.0)) {
    *beta = 0.0;
    return 1;
  }
  // sigma_min(X) = 1/||R^{-1}||_2 >= 1/||R^{-1}||_F >= 1/(sqrt(n) ||R^{-1}||_1)
  *beta = (mode == BOUNDS_FROB || mode == BOUNDS_NORM2) ? 1.0 / std::sqrt(fr)
                                                        : temp_beta / (std::sqrt(static_cast<double>(n)) * inv1);
  if (mode == BOUNDS_NORM2) {
    // A/alpha' with alpha' = alpha s2 >= ||A||_2 has sigma_min >= beta / s2
    const double s2 = norm2_upper(c, n, X, ldx);
    *alpha = a * s2;
    *beta /= s2;
  }
  return 0;
}

int qdwh(Context& c, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq, double* dH, int64_t ldh,
         const QdwhOpts& o) {
  if (m < n) return -1;
  if (m == 0 || n == 0) return 0;
  c.stats = Stats{};
  EventTimer total(c.stream());
  // internal copies with an even leading dimension (16-byte aligned GEMM tiles)
  const int64_t ldx = even(m);
  double* Ain = c.buf("Ain", static_cast<size_t>(ldx) * n);
  double* X = c.buf("Xit", static_cast<size_t>(ldx) * n);
  ck(scale_copy(m, n, 1.0, dA, lda, 0, Ain, ldx, 0, 1, 0.0, c.stream()));
  c.stats.launches++;
  double alpha = 0, beta = 0;
  {
    EventTimer tb(c.stream());
    const int info = bounds(c, m, n, o.sigma, Ain, ldx, o.bounds, &alpha, &beta);
    c.stats.ms_bounds = tb.stop();
    c.stats.alpha = alpha;
    c.stats.beta = beta;
    if (info != 0) {
      c.stats.info = info;
      return info;
    }
  }
  ck(scale_copy(m, n, 1.0, Ain, ldx, 0, X, ldx, 0, 1, -o.sigma, c.stream()));
  ck(scale_copy(m, n, 1.0 / alpha, X, ldx, 0, X, ldx, 0, 1, 0.0, c.stream()));
  c.stats.launches += 2;

  const double eps = eps_precision();
  const double tol1 = 10.0 * eps / 2.0;
  const double tol2 = std::exp(std::log(tol1) / 3.0);
  const int mp = static_cast<int>(even(m));  // row offset of the sqrt(c) I block in the stack
  const int64_t ldw = even(static_cast<int64_t>(mp) + n), ldz = even(m), ldn = even(n);
  Mat W{c.buf("W", static_cast<size_t>(ldw) * n), ldw, 0};
  Mat Qf{c.buf("Qf", static_cast<size_t>(ldw) * n), ldw, 0};
  Mat Z{c.buf("Z", static_cast<size_t>(ldz) * n), ldz, 0};
  Mat G{c.buf("G", static_cast<size_t>(ldn) * n), ldn, 0};
  DiagInv Dg{c.buf("dinv", static_cast<size_t>(nblocks(n)) * 4096), 0};
  double* tau = c.buf("tau", n);
  double* T = c.buf("qr_t", static_cast<size_t>(npanels(n)) * 1024);
  int* dinfo = c.dinfo();
  double* scal = c.dscal();
  double* part = c.dpartial();
  const bool left = (o.left_solve || o.sym == 'S' || o.sym == 's') && m == n;

  EventTimer ti(c.stream());
  double lowk = beta, err = 1.0, err2 = std::fabs(1.0 - lowk);
  int it = 0;
  while ((it == 0 || err > tol2 || err2 > tol1) && (o.maxit < 0 || it <= o.maxit) && it < 100) {
    EventTimer tstep(c.stream());
    double ak, bk, ckk, lnext;
    qdwh_weights(lowk, &ak, &bk, &ckk, &lnext);
    lowk = lnext;
    double akk, bkk;
    bool use_qr = ckk > 100.0;
    if (!use_qr) {
      OzScope mixed_ch(c, c.zolo_mixed >= 1);  // the mixed form's products of this Cholesky step
      gemm(c, 1, 0, n, n, m, ckk, Mat{X, ldx, 0}, Mat{X, ldx, 0}, 0.0, G, 1, nullptr, 1, 0);
      ck(add_diag(n, G.p, G.ld, 1.0, c.stream()));
      ck(cudaMemsetAsync(dinfo, 0, sizeof(int), c.stream()));
      c.stats.launches += 2;
      potrf(c, n, G, 1, dinfo, Dg);
      const int pinfo = injected_info(c, it, read_info(c, dinfo, 1));
      if (pinfo != 0) {
        // not numerically SPD: redo this step with the QR form (the reference ignores PDPOSV's INFO)
        if (c.stats.info == 0) c.stats.info = pinfo;
        use_qr = true;
      } else {
        spd_solve(c, m, n, X, ldx, G, Dg, Z, 1, left);
        akk = ak - bk / ckk;
        bkk = bk / ckk;
        c.stats.chol_iterations++;
        if (it < 16) c.stats.branch[it] = 2;
        c.stats.flops += 2.0 * m * static_cast<double>(n) * n + static_cast<double>(n) * n * n / 3.0 +
                         static_cast<double>(m) * n * n;
      }
    }
    if (use_qr) {
      const double sck = std::sqrt(ckk);
      ck(form_stack(m, mp, n, X, ldx, W.p, W.ld, 0, nullptr, 1.0 / sck, 1, c.stream()));
      c.stats.launches++;
      geqrf(c, mp + n, n, mp, W, tau, T, 1);
      orgqr(c, mp + n, n, mp, W, T, Qf, 1);
      q1q2t(c, m, mp, n, Qf, Z, 1);
      akk = (ak - bk / ckk) / sck;
      bkk = bk / ckk;
      c.stats.qr_iterations++;
      if (it < 16) c.stats.branch[it] = 1;
      c.stats.flops += 4.0 * m * static_cast<double>(n) * n + static_cast<double>(n) * n * n;
    }
    ck(combine_update(m, n, X, ldx, Z.p, Z.ld, 0, 1, bkk, akk, nullptr, part, scal, c.stream()));
    c.stats.launches += 2;
    err = std::sqrt(d2h(c, scal));
    if (it < 16) {
      c.stats.con[it] = ckk;
      c.stats.err[it] = err;
      c.stats.ms_step[it] = tstep.stop();
    }
    ++it;
    err2 = std::fabs(1.0 - lowk);
  }
  c.stats.ms_iter = ti.stop();
  c.stats.iterations = it;
  c.stats.last_err = err;
  ck(scale_copy(m, n, 1.0, X, ldx, 0, dQ, ldq, 0, 1, 0.0, c.stream()));
  c.stats.launches++;
  if (dH) {
    EventTimer th(c.stream());
    OzScope mixed_h(c, c.zolo_mixed >= 1);
    form_h(c, m, n, X, ldx, Ain, ldx, dH, ldh);
    c.stats.ms_h = th.stop();
  }
  c.stats.ms_total = total.stop();
  return mixed_status(c);
}

int zolo_pd(Context& c, char sym, int rk, int m, int n, double alpha, double beta, const double* dA, int64_t lda,
            double* dQ, int64_t ldq, double* dH, int64_t ldh, int maxit, const Prefactored* pf) {
  if (m < n) return -3;
  if (rk < 1 || rk > 8) return -2;
  if (m == 0 || n == 0) return 0;
  if (!(alpha > 0.0) || !(beta > 0.0)) return -5;
  c.stats = Stats{};
  c.stats.alpha = alpha;
  c.stats.beta = beta;
  EventTimer total(c.stream());
  // Factored iterate (with the bounds' QR at hand and the shared QR form): X = Q_x Y with
  // Q_x the Q of A/alpha = Q_x R, so X0 = A/(alpha beta) has Y0 = R/beta.  Every step keeps
  // Q_x on the left (the QR of X is Q_x times the QR of Y; X^T X = Y^T Y; X S = Q_x (Y S)),
  // so the iteration runs on the n x n Y; at the end Q = Q_x Y through the reflectors and
  // H = sym(Q^T A) = sym(alpha R^T Y).  That saves forming Q_x, the m x n products with it
  // and H's 2mn^2.
  const bool factored = pf && c.zolo_shared_qr && !(sym == 'S' || sym == 's');
  const int mx = factored ? n : m;  // rows of the iterate
  const int64_t ldx = even(mx);
  double* X = c.buf("Xit", static_cast<size_t>(ldx) * n);
  // R with its zeros below the diagonal (the reflectors live there), for H at the end
  double* Rx = factored && dH ? c.buf("zf_r", static_cast<size_t>(even(n)) * n) : nullptr;
  // X0 = A/(alpha beta) = Q_x R (pf->alpha / (alpha beta)): Y0 = R / ys
  const double ys = pf ? beta * alpha / pf->alpha : 1.0;
  if (factored) {
    ck(copy_upper(n, pf->W, pf->ldw, 1.0 / ys, X, ldx, c.stream()));
    if (Rx) ck(copy_upper(n, pf->W, pf->ldw, 1.0, Rx, even(n), c.stream()));
    c.stats.launches += 2;
  } else {
    ck(scale_copy(m, n, 1.0 / (alpha * beta), dA, lda, 0, X, ldx, 0, 1, 0.0, c.stream()));
    c.stats.launches++;
  }

  const double eps = eps_precision();
  const double tol = eps;
  const double tol1 = 10.0 * eps / 2.0;
  const double tol2 = std::exp(std::log(tol1) / (2.0 * rk + 1.0));
  const int mp = static_cast<int>(even(m));  // row offset of the sqrt(c) I block in the stack
  const int64_t ldw = even(static_cast<int64_t>(mp) + n), ldz = even(m), ldn = even(n);
  const int64_t sW = ldw * n, sZ = ldz * n;
  Mat W{c.buf("W", static_cast<size_t>(sW) * rk), ldw, sW};
  Mat Qf{c.buf("Qf", static_cast<size_t>(sW) * rk), ldw, sW};
  Mat Z{c.buf("Z", static_cast<size_t>(sZ) * rk), ldz, sZ};
  Mat G{c.buf("G", static_cast<size_t>(ldn) * n), ldn, 0};
  Mat Wc{W.p, ldn, ldn * n};  // shifted Gram matrices reuse the QR workspace
  const int64_t sD = static_cast<int64_t>(nblocks(n)) * 4096;
  DiagInv Dz{c.buf("dinv", static_cast<size_t>(sD) * rk), sD};
  double* tau = c.buf("tau", static_cast<size_t>(n) * rk);
  double* T = c.buf("qr_t", static_cast<size_t>(npanels(n)) * 1024 * rk);
  double* dvec = c.buf("zolo_vec", 64);
  int* dinfo = c.dinfo();
  double* scal = c.dscal();
  double* part = c.dpartial();
  const bool left = (sym == 'S' || sym == 's') && m == n;

  std::vector<double> coeff(3 * rk), hv(64, 0.0);
  double con = 1.0 / beta, err = 1.0;
  int it = 0;
  const bool ns_finish = c.zolo_ns_finish != 0;
  EventTimer ti(c.stream());
  // term plan (ZOLO_OPT_TERM_PLAN): needs the measured Newton-Schulz finish to end the loop;
  // its coefficients come from the complementary modulus (exact at any CON)
  const bool plan_terms = ns_finish && c.zolo_term_plan && c.zolo_chol_inverse && !left;
  TermPlanner planner(rk, mx, n, tol, c.zolo_mixed >= 1);
  int planned = 0;
  // with the Newton-Schulz finish the loop ends at the measured check, not on ||X_{k+1} - X_k||
  while ((ns_finish || err > tol2) && it < maxit) {
    EventTimer tstep(c.stream());
    int rk_it = rk;  // terms of this iteration
    if (plan_terms) rk_it = planned > 0 ? planned : planner.choose(con, it == 0 && pf && c.zolo_shared_qr);
    if (plan_terms) compute_coeff_kp(con, tol, rk_it, coeff.data());
    else compute_coeff(con, tol, rk_it, coeff.data());
    double maxc = coeff[0];
    for (int i = 1; i < 2 * rk_it; ++i) maxc = std::max(maxc, coeff[i]);
    bool use_qr = plan_terms ? con > kConChol : (it == 0 || con > 1.0e3) && maxc > 3.0e2;
    bool z_summed = false;  // Z holds sum_j w_j Z_j / FONE already (one Z instead of r)
    if (!use_qr) {
      // the mixed form's products of the Cholesky iteration (and of the finish entered here)
      OzScope mixed_ch(c, c.zolo_mixed >= 1);
      gemm(c, 1, 0, n, n, mx, 1.0, Mat{X, ldx, 0}, Mat{X, ldx, 0}, 0.0, G, 1, nullptr, 1, 0);
      if (ns_finish) {
        // G = X^T X is in hand: once X is within 0.1 of orthogonal (RMS of sigma^2 - 1),
        // the rest of the iteration is FP64 Newton-Schulz (the polar factor of X is that of A)
        ck(ns_prepare(n, G.p, G.ld, part, scal + 2, 0, c.stream()));
        c.stats.launches += 2;
        const double e0 = std::sqrt(d2h(c, scal + 2) / n);
        // with the term plan: Newton-Schulz from the measured e0 only when cheaper than the plan
        // (the plan's prediction can be reached only to rounding: when it predicts the finish,
        // the measured e0 decides the steps)
        if (e0 <= kNsEnter &&
            (!plan_terms || planner.predicts_finish(con) || planner.ns_cost(e0) <= planner.cost_from(con))) {
          newton_schulz_finish(c, mx, n, X, ldx, G, Z, e0, it);
          c.stats.ns_finish = 1;
          c.stats.ms_finish = tstep.stop();
          break;
        }
      }
      const bool inverse_form = c.zolo_chol_inverse && !left;
      for (int b = 0; b < rk_it; ++b) hv[b] = coeff[2 * b];
      h2d(c, dvec, hv.data(), rk_it);
      ck(shift_lower(n, G.p, G.ld, Wc.p, Wc.ld, Wc.stride, dvec, rk_it, c.stream()));
      ck(cudaMemsetAsync(dinfo, 0, sizeof(int) * rk_it, c.stream()));
      c.stats.launches += 2;
      // the explicit-inverse form takes the factors' inverses from the same recursion
      Mat Y{nullptr, ldn, ldn * n};
      if (inverse_form) {
        Y.p = c.buf("zc_y", static_cast<size_t>(ldn) * n * rk_it);
        potrf_inv(c, n, Wc, Y, rk_it, dinfo, Dz);
      } else {
        potrf(c, n, Wc, rk_it, dinfo, Dz);
      }
      const int pinfo = injected_info(c, it, read_info(c, dinfo, rk_it));
      if (pinfo != 0) {
        if (c.stats.info == 0) c.stats.info = pinfo;
        use_qr = true;  // fall back to the QR form for this step
      } else if (inverse_form) {
        // explicit form: S = sum_b w_b W_b^{-1}, W_b^{-1} = L_b^{-T} L_b^{-1}, then one Z = X S
        const double fone_c = zolo_fone(coeff.data(), rk_it);
        Mat S{c.buf("zc_s", static_cast<size_t>(ldn) * n), ldn, 0};
        for (int b = 0; b < rk_it; ++b) {
          const double w = -coeff[2 * rk_it + b] / fone_c;
          gemm(c, 1, 0, n, n, n, w, Mat{Y.p + b * Y.stride, ldn, 0}, Mat{Y.p + b * Y.stride, ldn, 0},
               b == 0 ? 0.0 : 1.0, S, 1, nullptr, 1, 2);
        }
        ck(mirror_lower(n, S.p, S.ld, c.stream()));
        c.stats.launches++;
        gemm(c, 0, 0, mx, n, n, 1.0, Mat{X, ldx, 0}, S, 0.0, Mat{Z.p, Z.ld, 0}, 1);
        z_summed = true;
        c.stats.chol_iterations++;
        if (it < 16) c.stats.branch[it] = 2;
        const double dm = m, dmx = mx, dn = n;
        const double canonical = dm * dn * dn + rk_it * (dn * dn * dn / 3.0 + 2.0 * dm * dn * dn);
        c.stats.flops += canonical;
        c.stats.flops_exec_delta += 3.0 * dmx * dn * dn + rk_it * dn * dn * dn - canonical;
      } else {
        spd_solve(c, mx, n, X, ldx, Wc, Dz, Z, rk_it, left);
        for (int b = 0; b < rk_it; ++b) hv[16 + b] = -coeff[2 * rk_it + b];
        c.stats.chol_iterations++;
        if (it < 16) c.stats.branch[it] = 2;
        c.stats.flops += static_cast<double>(m) * n * n +
                         rk_it * (static_cast<double>(n) * n * n / 3.0 + 2.0 * m * static_cast<double>(n) * n);
      }
    }
    const double fone = zolo_fone(coeff.data(), rk_it);
    const double con_next = zolo_next_con(con, coeff.data(), rk_it, fone);
    if (use_qr) {
      const bool shared = c.zolo_shared_qr != 0;
      z_summed = shared;
      // the first iteration may reuse the QR of A/alpha: X0 = (A/alpha)/beta
      const Prefactored* pfi = (shared && it == 0) ? pf : nullptr;
      for (int b = 0; b < rk_it; ++b) hv[b] = std::sqrt(coeff[2 * b]) * (pfi ? ys : 1.0);
      h2d(c, dvec, hv.data(), rk_it);
      for (int b = 0; b < rk_it; ++b) hv[16 + b] = -coeff[2 * rk_it + b] / std::sqrt(coeff[2 * b]);
      if (shared) {
        zolo_terms_shared_qr(c, mx, n, X, ldx, W, Qf, Z, tau, T, dvec, hv.data() + 16, fone, rk_it, pfi, factored,
                             m);
      } else {
        ck(form_stack(m, mp, n, X, ldx, W.p, W.ld, W.stride, dvec, 0.0, rk_it, c.stream()));
        c.stats.launches++;
        geqrf(c, mp + n, n, mp, W, tau, T, rk_it);
        orgqr(c, mp + n, n, mp, W, T, Qf, rk_it);
        q1q2t(c, m, mp, n, Qf, Z, rk_it);
      }
      // canonical: the reference's structured QR form, 4mn^2 + n^3 per term (the shared form
      // records what it executes beyond this in flops_exec_delta)
      c.stats.flops += rk_it * (4.0 * m * static_cast<double>(n) * n + static_cast<double>(n) * n * n);
      c.stats.qr_iterations++;
      if (it < 16) c.stats.branch[it] = 1;
    }
    if (z_summed) {
      // Z already holds sum_j w_j Z_j / FONE
      ck(combine_update(mx, n, X, ldx, Z.p, Z.ld, 0, 1, 1.0 / fone, 1.0, nullptr, part, scal, c.stream()));
    } else {
      for (int b = 0; b < rk_it; ++b) hv[16 + b] /= fone;
      h2d(c, dvec + 16, hv.data() + 16, rk_it);
      ck(combine_update(mx, n, X, ldx, Z.p, Z.ld, Z.stride, rk_it, 1.0 / fone, 0.0, dvec + 16, part, scal,
                        c.stream()));
    }
    c.stats.launches += 2;
    // plan the next iteration while this one runs
    if (plan_terms) planned = planner.choose(con_next, false);
    err = std::sqrt(d2h(c, scal));
    if (it < 16) {
      c.stats.con[it] = con;
      c.stats.err[it] = err;
      c.stats.ms_step[it] = tstep.stop();
      c.stats.terms[it] = rk_it;
    }
    con = con_next;
    ++it;
  }
  c.stats.ms_iter = ti.stop();
  c.stats.iterations = it;
  c.stats.last_err = err;
  OzScope mixed_h(c, c.zolo_mixed >= 1);  // forming Q and H
  if (factored) {
    EventTimer th(c.stream());  // ms_h covers Q = Q_x Y and H here
    // Q = Q_x Y: [Y; 0] through the reflectors of A/alpha = Q_x R
    ck(set_identity(m, n, dQ, ldq, 0, 1, 0.0, c.stream()));
    ck(scale_copy(n, n, 1.0, X, ldx, 0, dQ, ldq, 0, 1, 0.0, c.stream()));
    c.stats.launches += 2;
    ormqr_left(c, m, n, -1, Mat{const_cast<double*>(pf->W), pf->ldw, 0}, pf->T, Mat{dQ, ldq, 0}, n, 1);
    const double dm = m, dn = n;
    c.stats.flops_exec_delta += 4.0 * dm * dn * dn - 2.0 * dn * dn * dn;
    if (dH) {
      // H = sym(Q^T A) = sym(a Y^T R) = sym(a R^T Y), a = pf->alpha (A = a Q_x R): R^T is lower
      // triangular (k up to the row)
      const int64_t ldh_i = even(n);
      double* Hb = c.buf("Hbuf", static_cast<size_t>(ldh_i) * n);
      gemm(c, 1, 0, n, n, n, pf->alpha, Mat{Rx, even(n), 0}, Mat{X, ldx, 0}, 0.0, Mat{Hb, ldh_i, 0}, 1, nullptr, 0,
           0, nullptr, 1);
      ck(symmetrize(n, Hb, ldh_i, c.stream()));
      ck(scale_copy(n, n, 1.0, Hb, ldh_i, 0, dH, ldh, 0, 1, 0.0, c.stream()));
      c.stats.launches += 2;
      c.stats.flops += 2.0 * dm * dn * dn;
      c.stats.flops_exec_delta += dn * dn * dn - 2.0 * dm * dn * dn;
    }
    c.stats.ms_h = th.stop();
    c.stats.ms_total = total.stop();
    return mixed_status(c);
  }
  ck(scale_copy(m, n, 1.0, X, ldx, 0, dQ, ldq, 0, 1, 0.0, c.stream()));
  c.stats.launches++;
  if (dH) {
    EventTimer th(c.stream());
    const int64_t lda_i = even(m);
    double* Ain = c.buf("Ain", static_cast<size_t>(lda_i) * n);
    ck(scale_copy(m, n, 1.0, dA, lda, 0, Ain, lda_i, 0, 1, 0.0, c.stream()));
    form_h(c, m, n, X, ldx, Ain, lda_i, dH, ldh);
    c.stats.ms_h = th.stop();
  }
  c.stats.ms_total = total.stop();
  return mixed_status(c);
}

int plan_terms(double con, int rk, int m, int n, bool prefactored, int* terms, int* qr_form, int maxlen,
               int* ns_steps) {
  if (rk < 1 || rk > 8 || m < n || n < 1 || !(con >= 1.0) || maxlen < 0) return -1;
  TermPlanner planner(rk, m, n, eps_precision());
  int len = 0;
  while (2.0 * (con - 1.0) > 0.5 * kNsEnter && len < maxlen) {
    const int r = planner.choose(con, prefactored && len == 0);
    if (terms) terms[len] = r;
    if (qr_form) qr_form[len] = con > kConChol ? 1 : 0;
    con = planner.con_after(con, r);
    ++len;
  }
  if (ns_steps) *ns_steps = planner.finish_steps(con);
  return len;
}

int zolo_polar(Context& c, int rk, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq, double* dH,
               int64_t ldh) {
  if (m < n) return -3;
  if (rk < 1 || rk > 8) return -2;
  if (m == 0 || n == 0) return 0;
  EventTimer total(c.stream());
  double alpha = 0.0, beta = 0.0, alpha_fro = 0.0;
  EventTimer tb(c.stream());
  const BoundsMode bm = c.zolo_norm2 ? BOUNDS_NORM2 : (c.zolo_beta_frob ? BOUNDS_FROB : BOUNDS_ZOLOPD);
  const int binfo = bounds(c, m, n, 0.0, dA, lda, bm, &alpha, &beta, &alpha_fro);
  const double ms_bounds = tb.stop();
  const double bflops = 4.0 / 3.0 * static_cast<double>(n) * n * n + 2.0 * m * static_cast<double>(n) * n;
  if (binfo != 0) {
    c.stats = Stats{};
    c.stats.info = binfo;
    return binfo;
  }
  // bounds left the factored A/alpha in its workspace ("bnd_x", ld even(m)) and the panel factors in "bnd_t"
  const Prefactored pf{c.buf("bnd_x", static_cast<size_t>(even(m)) * n), even(m),
                       c.buf("bnd_t", static_cast<size_t>(npanels(n)) * 1024), alpha_fro};
  const int info = zolo_pd(c, 'N', rk, m, n, alpha, beta, dA, lda, dQ, ldq, dH, ldh, 6, &pf);
  c.stats.ms_bounds = ms_bounds;
  c.stats.flops += bflops;
  c.stats.ms_total = total.stop();
  return info;
}

namespace {

constexpr int kMaxBatch = 1024;  // members per launch (the device INFO array holds 1024)

void h2d_bytes(Context& c, void* d, const void* h, size_t bytes) {
  ck(cudaMemcpyAsync(d, h, bytes, cudaMemcpyHostToDevice, c.stream()));
}

std::vector<double> d2h_vec(Context& c, const double* d, int count) {
  std::vector<double> h(count);
  ck(cudaMemcpyAsync(h.data(), d, sizeof(double) * count, cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  return h;
}

// One bucket: B members padded to MB x NB, solved together (pqdwhfacs.f90:318-457 per member).
void qdwh_bucket(Context& c, const std::vector<int>& idx, int MB, int NB, const int* m, const int* n,
                 const double* const* dA, const int64_t* lda, double* const* dQ, const int64_t* ldq,
                 double* const* dH, const int64_t* ldh, int* info, int* iterations, BatchStats* bs) {
  const int B = static_cast<int>(idx.size());
  const cudaStream_t st = c.stream();
  const int64_t ldp = MB, sP = ldp * NB, ldn = NB, sN = ldn * NB;
  double* Ap = c.buf("bat_a", static_cast<size_t>(sP) * B);
  double* X = c.buf("bat_x", static_cast<size_t>(sP) * B);
  double* vals = c.buf("bat_vec", static_cast<size_t>(8) * B);
  double* part = c.buf("bat_part", 8192);
  const size_t mem_doubles = (sizeof(BatchMember) * B + 7) / 8;
  auto* dmem = reinterpret_cast<BatchMember*>(c.buf("bat_mem", mem_doubles));
  std::vector<BatchMember> hm(B);
  for (int b = 0; b < B; ++b) {
    const int i = idx[b];
    hm[b] = BatchMember{m[i], n[i], dA[i], lda[i], 0.0, dQ[i], ldq[i], dH ? dH[i] : nullptr, dH ? ldh[i] : 0};
  }
  // pad with tau = ||A||_F / sqrt(n), a value inside [sigma_min, sigma_max]
  h2d_bytes(c, dmem, hm.data(), sizeof(BatchMember) * B);
  ck(batch_pack(dmem, B, MB, NB, Ap, ldp, sP, st));
  ck(batch_frob2(MB, NB, Ap, ldp, sP, B, part, 8192, vals, st));
  const std::vector<double> fa = d2h_vec(c, vals, B);
  bool padded = false;
  for (int b = 0; b < B; ++b) {
    hm[b].tau = std::sqrt(fa[b] / hm[b].n);
    padded = padded || hm[b].n < NB;
  }
  if (padded) {
    h2d_bytes(c, dmem, hm.data(), sizeof(BatchMember) * B);
    ck(batch_pack(dmem, B, MB, NB, Ap, ldp, sP, st));
  }
  c.stats.launches += padded ? 4 : 3;

  // ---- bounds, PQDWHFACS form: alpha = ||A'||_F, beta = ||X0||_1 / (sqrt(NB) ||R^-1||_1) ----
  ck(batch_frob2(MB, NB, Ap, ldp, sP, B, part, 8192, vals, st));
  std::vector<double> alpha = d2h_vec(c, vals, B);
  std::vector<double> hv(8 * B, 0.0);
  std::vector<char> done(B, 0);
  for (int b = 0; b < B; ++b) {
    alpha[b] = std::sqrt(alpha[b]);
    if (!(alpha[b] > 0.0) || !std::isfinite(alpha[b])) {
      info[idx[b]] = 1;
      done[b] = 1;
    }
    hv[b] = done[b] ? 1.0 : 1.0 / alpha[b];
  }
  const std::vector<double> xscale(hv.begin(), hv.begin() + B);  // X_0 = A' xscale
  h2d(c, vals, hv.data(), B);
  ck(scale_copy(MB, NB, 1.0, Ap, ldp, sP, X, ldp, sP, B, 0.0, st));
  ck(batch_scale(MB, NB, X, ldp, sP, B, vals, st));
  ck(batch_norm1(MB, NB, X, ldp, sP, B, vals + B, st));
  double* Xq = c.buf("bat_xq", static_cast<size_t>(sP) * B);
  ck(scale_copy(MB, NB, 1.0, X, ldp, sP, Xq, ldp, sP, B, 0.0, st));
  c.stats.launches += 5;
  double* tau = c.buf("bat_tau", static_cast<size_t>(NB) * B);
  const int np = (NB + 31) / 32;
  double* T = c.buf("bat_t", static_cast<size_t>(np) * 1024 * B);
  geqrf(c, MB, NB, -1, Mat{Xq, ldp, sP}, tau, T, B);
  double* Lt = c.buf("bat_lt", static_cast<size_t>(sN) * B);
  double* Id = c.buf("bat_i", static_cast<size_t>(sN) * B);
  double* Ri = c.buf("bat_ri", static_cast<size_t>(sN) * B);
  ck(batch_transpose(NB, NB, Xq, ldp, sP, Lt, ldn, sN, B, st));
  ck(set_identity(NB, NB, Id, ldn, sN, B, 1.0, st));
  c.stats.launches += 2;
  const int64_t sD = static_cast<int64_t>(nblocks(NB)) * 4096;
  DiagInv D{c.buf("bat_dinv", static_cast<size_t>(sD) * B), sD};
  diag_inverses(c, NB, Mat{Lt, ldn, sN}, B, D);
  trsm_rlt(c, NB, NB, Mat{Lt, ldn, sN}, Mat{Id, ldn, sN}, Mat{Ri, ldn, sN}, B, D);
  ck(batch_norm1(NB, NB, Ri, ldn, sN, B, vals + 2 * B, st));
  c.stats.launches++;
  const std::vector<double> nv = d2h_vec(c, vals + B, 2 * B);
  std::vector<double> lowk(B, 1.0), err(B, 1.0);
  std::vector<int> its(B, 0);
  for (int b = 0; b < B; ++b) {
    const double beta = nv[b] / (std::sqrt(static_cast<double>(NB)) * nv[B + b]);
    if (!done[b] && (!std::isfinite(beta) || !(beta > 0.0))) {
      info[idx[b]] = 1;
      done[b] = 1;
    }
    lowk[b] = done[b] ? 1.0 : beta;
  }
  double flops = 4.0 / 3.0 * NB * static_cast<double>(NB) * NB + 2.0 * MB * static_cast<double>(NB) * NB;
  double useful = 0.0;
  for (int b = 0; b < B; ++b) {
    const double mm = m[idx[b]], nn = n[idx[b]];
    useful += 4.0 / 3.0 * nn * nn * nn + 2.0 * mm * nn * nn;
  }
  flops *= B;

  // ---- the iteration, all members together ----
  const double eps = eps_precision();
  const double tol1 = 10.0 * eps / 2.0;
  const double tol2 = std::exp(std::log(tol1) / 3.0);
  const int maxit = 12;
  const int mp = MB;  // the sqrt(c) I block of the QR stack starts at row MB (even)
  const int64_t ldw = even(static_cast<int64_t>(mp) + NB), sW = ldw * NB;
  Mat W{c.buf("bat_w", static_cast<size_t>(sW) * B), ldw, sW};
  Mat Qf{c.buf("bat_qf", static_cast<size_t>(sW) * B), ldw, sW};
  Mat Z{c.buf("bat_z", static_cast<size_t>(sP) * B), ldp, sP};
  Mat G{c.buf("bat_g", static_cast<size_t>(sN) * B), ldn, sN};
  DiagInv Dg{c.buf("bat_dinv2", static_cast<size_t>(sD) * B), sD};
  int* dinfo = c.dinfo();
  std::vector<double> ak(B), bk(B), ckv(B), ln(B);
  std::vector<double> cx(B), cz(B);
  const std::vector<char> done0 = done;
  const std::vector<double> lowk0 = lowk;

  // The steps on the device, their coefficients read from device arrays: the Cholesky form
  // Z = X (I + c X^T X)^{-1} (pqdwhfacs.f90:408-431) and the QR form from the stack
  // [sqrt(c) X; I] (pqdwhfacs.f90:375-404), then X <- cx X + cz Z and ||X_new - X||_F^2.
  auto chol_factor = [&](const double* dck, int* dinf) {
    gemm(c, 1, 0, NB, NB, MB, 1.0, Mat{X, ldp, sP}, Mat{X, ldp, sP}, 0.0, G, B, dck, 1, 0);
    ck(batch_add_diag(NB, G.p, G.ld, G.stride, B, 1.0, st));
    ck(cudaMemsetAsync(dinf, 0, sizeof(int) * B, st));
    c.stats.launches += 2;
    potrf(c, NB, G, B, dinf, Dg);
  };
  auto chol_solve = [&]() { spd_solve(c, MB, NB, X, ldp, G, Dg, Z, B, false, sP); };
  auto qr_step = [&](const double* dsc) {
    ck(form_stack(MB, mp, NB, X, ldp, W.p, W.ld, W.stride, dsc, 0.0, B, st, 0, sP));
    c.stats.launches++;
    geqrf(c, mp + NB, NB, mp, W, tau, T, B);
    orgqr(c, mp + NB, NB, mp, W, T, Qf, B);
    q1q2t(c, MB, mp, NB, Qf, Z, B);
  };
  auto combine = [&](const double* dcx, const double* dcz, double* de2) {
    ck(batch_combine(MB, NB, X, ldp, sP, Z.p, Z.ld, Z.stride, B, dcx, dcz, part, 8192, de2, st));
    c.stats.launches += 2;
  };
  auto count_step = [&](bool qr, const std::vector<char>& active) {
    flops += B * (qr ? 4.0 * MB * static_cast<double>(NB) * NB + static_cast<double>(NB) * NB * NB
                     : 2.0 * MB * static_cast<double>(NB) * NB + NB * static_cast<double>(NB) * NB / 3.0 +
                           static_cast<double>(MB) * NB * NB);
    for (int b = 0; b < B; ++b) {
      if (!active[b]) continue;
      const double mm = m[idx[b]], nn = n[idx[b]];
      useful += qr ? 4.0 * mm * nn * nn + nn * nn * nn : 3.0 * mm * nn * nn + nn * nn * nn / 3.0;
    }
  };
  // H' = sym(Q'^T A') and the unpadded outputs
  double* Hp = dH ? c.buf("bat_h", static_cast<size_t>(sN) * B) : nullptr;
  auto finish = [&]() {
    if (dH) {
      gemm(c, 1, 0, NB, NB, MB, 1.0, Mat{X, ldp, sP}, Mat{Ap, ldp, sP}, 0.0, Mat{Hp, ldn, sN}, B);
      ck(batch_symmetrize(NB, Hp, ldn, sN, B, st));
      c.stats.launches++;
    }
    ck(batch_unpack(dmem, B, MB, NB, X, ldp, sP, Hp, ldn, sN, st));
    c.stats.launches++;
  };
  auto count_finish = [&]() {
    if (!dH) return;
    flops += B * 2.0 * MB * static_cast<double>(NB) * NB;
    for (int b = 0; b < B; ++b) useful += 2.0 * m[idx[b]] * static_cast<double>(n[idx[b]]) * n[idx[b]];
  };

  // The host-synchronized loop (pqdwhfacs.f90:359-457 per member): the weights and the form
  // of each step from the members' current L, the Cholesky INFO read back before the solve (a
  // factorization that fails for any member turns the step into the QR form) and the errors
  // read back after the update.
  int it = 0;
  auto sync_loop = [&]() {
    while (true) {
      bool any = false, use_qr = false;
      for (int b = 0; b < B; ++b) {
        if (done[b]) continue;
        any = true;
        qdwh_weights(lowk[b], &ak[b], &bk[b], &ckv[b], &ln[b]);
        use_qr = use_qr || ckv[b] > 100.0;
      }
      if (!any) break;
      std::vector<char> active(B);
      for (int b = 0; b < B; ++b) active[b] = !done[b];
      if (!use_qr) {
        for (int b = 0; b < B; ++b) hv[b] = done[b] ? 0.0 : ckv[b];
        h2d(c, vals, hv.data(), B);
        chol_factor(vals, dinfo);
        std::vector<int> pin(B, 0);
        ck(cudaMemcpyAsync(pin.data(), dinfo, sizeof(int) * B, cudaMemcpyDeviceToHost, st));
        ck(cudaStreamSynchronize(st));
        bool fail = false;
        for (int b = 0; b < B; ++b) fail = fail || (!done[b] && pin[b] != 0);
        fail = fail || injected_info(c, it, 0) != 0;
        if (fail) {
          use_qr = true;  // not numerically SPD for some member: this step takes the QR form
        } else {
          chol_solve();
          for (int b = 0; b < B; ++b) {
            cx[b] = done[b] ? 1.0 : bk[b] / ckv[b];
            cz[b] = done[b] ? 0.0 : ak[b] - bk[b] / ckv[b];
          }
          count_step(false, active);
        }
      }
      if (use_qr) {
        for (int b = 0; b < B; ++b) hv[b] = done[b] ? 1.0 : 1.0 / std::sqrt(ckv[b]);
        h2d(c, vals, hv.data(), B);
        qr_step(vals);
        for (int b = 0; b < B; ++b) {
          const double sck = done[b] ? 1.0 : std::sqrt(ckv[b]);
          cx[b] = done[b] ? 1.0 : bk[b] / ckv[b];
          cz[b] = done[b] ? 0.0 : (ak[b] - bk[b] / ckv[b]) / sck;
        }
        count_step(true, active);
      }
      for (int b = 0; b < B; ++b) {
        hv[B + b] = cx[b];
        hv[2 * B + b] = cz[b];
      }
      h2d(c, vals + B, hv.data() + B, 2 * B);
      combine(vals + B, vals + 2 * B, vals + 3 * B);
      const std::vector<double> e2 = d2h_vec(c, vals + 3 * B, B);
      ++it;
      for (int b = 0; b < B; ++b) {
        if (done[b]) continue;
        err[b] = std::sqrt(e2[b]);
        lowk[b] = ln[b];
        ++its[b];
        // pqdwhfacs.f90:359: continue while ERR > TOL1^(1/3) or |1 - L| > TOL1, IT <= 12
        const bool more = (err[b] > tol2 || std::fabs(1.0 - lowk[b]) > tol1) && its[b] <= maxit;
        if (!more) done[b] = 1;
      }
    }
  };

  if (!c.batch_graph) {
    sync_loop();
    finish();
    count_finish();
    bs->sync_loops++;
  } else {
    // The schedule (qdwh_schedule): every step's form and weights from the members' L_0; a
    // step after a member's L has converged is conditional, and a gate kernel makes it neutral
    // for the member on the device when the error just measured is already below TOL1^(1/3).
    const QdwhSchedule S = qdwh_schedule(B, lowk.data(), done.data(), tol1, maxit);
    const int K = S.steps;
    const std::vector<char>& sqr = S.qr;
    const std::vector<int>&cnt = S.count, &last = S.last, &kc = S.cond;
    std::vector<char> hascond(B);
    for (int b = 0; b < B; ++b) hascond[b] = kc[b] >= 0;
    double* sched = c.buf("bat_sched", static_cast<size_t>(std::max(K, 1)) * 5 * B);
    int* sinfo = c.ibuf("bat_sinfo", static_cast<size_t>(std::max(K, 1)) * B);
    if (K > 0) h2d(c, sched, S.table.data(), K * 5 * B);
    std::vector<char> gated(K, 0);
    for (int b = 0; b < B; ++b)
      if (kc[b] >= 0) gated[kc[b]] = 1;
    auto run_steps = [&](int k0, int k1) {
      for (int k = k0; k < k1; ++k) {
        double* row = sched + static_cast<size_t>(k) * 5 * B;
        if (gated[k]) {
          ck(batch_gate(B, row - 5 * B + 3 * B, row + 4 * B, row, sqr[k], tol2, st));
          c.stats.launches++;
        }
        if (sqr[k]) {
          qr_step(row);
        } else {
          chol_factor(row, sinfo + static_cast<size_t>(k) * B);
          chol_solve();
        }
        combine(row + B, row + 2 * B, row + 3 * B);
      }
    };
    // When the last step is conditional for every member in it, it runs only if one of them
    // takes it (one read-back of the previous step's errors); the rest is one launch sequence.
    bool tail = K > 0 && gated[K - 1];
    for (int b = 0; b < B && tail; ++b) tail = last[b] < K - 1;
    const int Ka = tail ? K - 1 : K;
    auto scheduled = [&]() {
      run_steps(0, Ka);
      if (!tail) finish();
    };
    // one graph per bucket shape and schedule, captured on the second call of that shape (the
    // first runs eagerly and sizes the workspace), replayed while the workspace is unchanged
    std::string key = "qdwh " + std::to_string(MB) + " " + std::to_string(NB) + " " + std::to_string(B) + " " +
                      (dH ? "h " : "- ") + (tail ? "t " : "- ");
    for (int k = 0; k < Ka; ++k) key += sqr[k] ? (gated[k] ? 'Q' : 'q') : (gated[k] ? 'C' : 'c');
    // a bounded cache: a caller cycling through many bucket shapes keeps at most 256 graphs
    if (c.graphs.size() >= 256 && c.graphs.find(key) == c.graphs.end()) {
      ck(cudaStreamSynchronize(st));
      c.drop_graphs();
    }
    Context::CachedGraph& g = c.graphs[key];
    cudaGraphExec_t once = nullptr;  // a graph captured while the workspace grew: run once
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    ck(cudaStreamIsCapturing(st, &cap));
    // no capture under an injected CUDA tool (a profiler sets CUDA_INJECTION64_PATH): the
    // worker threads' concurrent captures ended the process under one; the same schedule then
    // runs eagerly
    static const bool tool = std::getenv("CUDA_INJECTION64_PATH") != nullptr;
    const bool capturable = c.batch_graph == 1 && !c.prof.on && !tool && st != cudaStreamLegacy && st != nullptr &&
                            cap == cudaStreamCaptureStatusNone;
    if (capturable && g.seen) {
      if (g.exec && g.gen != c.alloc_gen()) {
        ck(cudaGraphExecDestroy(g.exec));
        g.exec = nullptr;
      }
      if (g.exec) {
        ck(cudaGraphLaunch(g.exec, st));
        c.stats.launches += g.launches;
        bs->graph_replays++;
      } else {
        const uint64_t gen0 = c.alloc_gen();
        const int64_t l0 = c.stats.launches;
        cudaGraph_t graph = nullptr;
        ck(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
        c.capturing = true;
        try {
          scheduled();
        } catch (...) {
          c.capturing = false;
          cudaStreamEndCapture(st, &graph);
          if (graph) cudaGraphDestroy(graph);
          throw;
        }
        c.capturing = false;
        ck(cudaStreamEndCapture(st, &graph));
        cudaGraphExec_t exec = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        ck(e);
        ck(cudaGraphLaunch(exec, st));
        bs->graph_captures++;
        if (c.alloc_gen() == gen0) {
          g.exec = exec;
          g.gen = gen0;
          g.launches = c.stats.launches - l0;
        } else {
          once = exec;
        }
      }
    } else {
      scheduled();
      g.seen = true;
      bs->eager_scheduled++;
    }
    int Kr = K;  // steps that ran
    if (tail) {
      std::vector<double> e2p(B);
      ck(cudaMemcpyAsync(e2p.data(), sched + static_cast<size_t>(K - 2) * 5 * B + 3 * B, sizeof(double) * B,
                         cudaMemcpyDeviceToHost, st));
      ck(cudaStreamSynchronize(st));
      bool need = false;
      for (int b = 0; b < B; ++b) need = need || (kc[b] == K - 1 && std::sqrt(e2p[b]) > tol2);
      if (need) {
        run_steps(K - 1, K);
      } else {
        Kr = K - 1;
      }
      finish();
    }
    // the last synchronization of the bucket's iterations: every step's INFO and error
    std::vector<int> hinfo(static_cast<size_t>(K) * B, 0);
    std::vector<double> hs(static_cast<size_t>(K) * 5 * B, 0.0);
    if (K > 0) {
      ck(cudaMemcpyAsync(hinfo.data(), sinfo, sizeof(int) * hinfo.size(), cudaMemcpyDeviceToHost, st));
      ck(cudaMemcpyAsync(hs.data(), sched, sizeof(double) * hs.size(), cudaMemcpyDeviceToHost, st));
    }
    ck(cudaStreamSynchronize(st));
    if (once) ck(cudaGraphExecDestroy(once));
    c.free_retired();
    auto e2_at = [&](int k, int b) { return hs[static_cast<size_t>(k) * 5 * B + 3 * B + b]; };
    // which members took their conditional step (the gate's test, repeated on the host)
    std::vector<char> took(B, 0);
    for (int b = 0; b < B; ++b) took[b] = hascond[b] && std::sqrt(e2_at(last[b], b)) > tol2;
    for (int k = 0; k < Kr; ++k) {
      std::vector<char> active(B, 0);
      for (int b = 0; b < B; ++b) active[b] = (last[b] >= k) || (took[b] && kc[b] == k);
      count_step(sqr[k], active);
    }
    count_finish();
    bool fail = false;
    for (int k = 0; k < Kr && !fail; ++k) {
      if (sqr[k]) continue;
      for (int b = 0; b < B; ++b) {
        const bool active = (last[b] >= k) || (took[b] && kc[b] == k);
        fail = fail || (active && hinfo[static_cast<size_t>(k) * B + b] != 0);
      }
      fail = fail || injected_info(c, k, 0) != 0;
    }
    if (fail) {
      // a Cholesky step failed for some member: the whole bucket again from X_0 = A'/alpha
      // through the synchronized loop, which takes the QR form at that step
      h2d(c, vals, xscale.data(), B);
      ck(scale_copy(MB, NB, 1.0, Ap, ldp, sP, X, ldp, sP, B, 0.0, st));
      ck(batch_scale(MB, NB, X, ldp, sP, B, vals, st));
      c.stats.launches += 2;
      done = done0;
      lowk = lowk0;
      std::fill(its.begin(), its.end(), 0);
      it = 0;
      sync_loop();
      finish();
      count_finish();
      bs->restarts++;
    } else {
      bool resume = false;
      it = Kr;
      for (int b = 0; b < B; ++b) {
        if (last[b] < 0) continue;
        const int kf = took[b] ? kc[b] : last[b];
        its[b] = cnt[b] + (took[b] ? 1 : 0);
        lowk[b] = took[b] ? S.l_cond[b] : S.l_uncond[b];
        err[b] = std::sqrt(e2_at(kf, b));
        // pqdwhfacs.f90:359 after the member's last step
        const bool high = err[b] > tol2 || (c.inject_batch_err && b == 0);
        done[b] = !((high || std::fabs(1.0 - lowk[b]) > tol1) && its[b] <= maxit);
        resume = resume || !done[b];
      }
      if (resume) {
        // a member whose error was still above TOL1^(1/3) after its conditional step: its
        // further steps through the synchronized loop (the others are complete and unchanged)
        sync_loop();
        finish();
        count_finish();
        bs->resumes++;
      }
    }
  }
  for (int b = 0; b < B; ++b)
    if (iterations) iterations[idx[b]] = its[b];
  bs->buckets++;
  bs->max_iterations = std::max(bs->max_iterations, it);
  bs->flops += flops;
  bs->flops_useful += useful;
}

}  // namespace

int qdwh_batch(Context& c, int count, const int* m, const int* n, const double* const* dA, const int64_t* lda,
               double* const* dQ, const int64_t* ldq, double* const* dH, const int64_t* ldh, int* info,
               int* iterations, BatchStats* bs) {
  if (count < 0) return -2;
  for (int i = 0; i < count; ++i) {
    if (n[i] < 1 || m[i] < n[i]) return -3;
    if (lda[i] < m[i] || ldq[i] < m[i] || (dH && ldh[i] < n[i])) return -4;
    info[i] = 0;
  }
  BatchStats local;
  if (!bs) bs = &local;
  *bs = BatchStats{};
  c.stats = Stats{};
  EventTimer total(c.stream());
  // buckets from the cost model (dynamic programming over the members sorted by n)
  const BucketPlan plan = plan_buckets(c.batch_model, count, m, n, kMaxBatch);
  const int nbk = static_cast<int>(plan.nb.size());
  const int W = std::min(std::max(1, c.batch_model.streams), nbk);
  if (nbk > 0) {
    // the buckets are independent: spread them over W worker contexts (own stream and
    // workspace each, driven by one host thread each) so that their launch chains overlap;
    // a single bucket too runs on a worker's own stream, which its graph capture then holds
    // alone (a capture of the caller's stream would take in other threads' work on it)
    while (static_cast<int>(c.workers.size()) < W) c.workers.emplace_back(new Context(c.device()));
    std::vector<int> order(nbk);
    for (int b = 0; b < nbk; ++b) order[b] = b;
    std::sort(order.begin(), order.end(), [&](int a, int b) { return plan.ms[a] > plan.ms[b]; });
    std::vector<std::vector<int>> assign(W);
    std::vector<double> load(W, 0.0);
    for (int b : order) {
      const int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
      assign[w].push_back(b);
      load[w] += plan.ms[b];
    }
    // the members' inputs are ready on the caller's stream; the outputs are ready for it after
    cudaEvent_t ready = c.event(0);
    ck(cudaEventRecord(ready, c.stream()));
    std::vector<BatchStats> wbs(W);
    std::vector<int64_t> wl(W, 0);
    std::vector<cudaError_t> werr(W, cudaSuccess);
    std::vector<std::thread> th;
    for (int w = 0; w < W; ++w) {
      th.emplace_back([&, w] {
        try {
          Context& wc = *c.workers[w];
          ck(cudaSetDevice(wc.device()));
          ck(cudaStreamWaitEvent(wc.stream(), ready, 0));
          wc.stats = Stats{};
          wc.batch_graph = c.batch_graph;
          wc.inject_chol_fail = c.inject_chol_fail;
          wc.inject_batch_err = c.inject_batch_err;
          for (int b : assign[w])
            qdwh_bucket(wc, plan.members[b], plan.mb[b], plan.nb[b], m, n, dA, lda, dQ, ldq, dH, ldh, info,
                        iterations, &wbs[w]);
          wl[w] = wc.stats.launches;
        } catch (const CudaFailure& e) {
          werr[w] = e.err;
        } catch (...) {
          werr[w] = cudaErrorUnknown;
        }
      });
    }
    for (auto& t : th) t.join();
    for (int w = 0; w < W; ++w) {
      Context& wc = *c.workers[w];
      ck(cudaEventRecord(wc.event(0), wc.stream()));
      ck(cudaStreamWaitEvent(c.stream(), wc.event(0), 0));
    }
    for (int w = 0; w < W; ++w)
      if (werr[w] != cudaSuccess) throw CudaFailure{werr[w]};
    for (int w = 0; w < W; ++w) {
      bs->buckets += wbs[w].buckets;
      bs->max_iterations = std::max(bs->max_iterations, wbs[w].max_iterations);
      bs->flops += wbs[w].flops;
      bs->flops_useful += wbs[w].flops_useful;
      bs->graph_replays += wbs[w].graph_replays;
      bs->graph_captures += wbs[w].graph_captures;
      bs->eager_scheduled += wbs[w].eager_scheduled;
      bs->sync_loops += wbs[w].sync_loops;
      bs->restarts += wbs[w].restarts;
      bs->resumes += wbs[w].resumes;
      c.stats.launches += wl[w];
    }
  }
  bs->ms = total.stop();
  bs->predicted_ms = plan.total_ms;
  c.stats.ms_total = bs->ms;
  c.stats.flops = bs->flops_useful;
  c.stats.flops_exec_delta = bs->flops - bs->flops_useful;
  c.stats.iterations = bs->max_iterations;
  return 0;
}

int batch_autotune(Context& c) {
  // probe buckets of graded diagonal members (kappa 1e8, m = 1.5 n) at three sizes with 1 and
  // 8 members: the difference gives the per-member work, the rest the launch-chain latency
  const int sizes[3] = {64, 256, 1024};
  double lat[3], rate[3];
  double flops_at[3];
  // the probes run on a worker context (own stream), as the solver's buckets do
  if (c.workers.empty()) c.workers.emplace_back(new Context(c.device()));
  Context& wc = *c.workers[0];
  wc.batch_graph = c.batch_graph;
  wc.inject_chol_fail = 0;
  wc.inject_batch_err = 0;
  for (int k = 0; k < 3; ++k) {
    const int NB = sizes[k], MB = NB + NB / 2;
    std::vector<double> host(static_cast<size_t>(MB) * NB, 0.0);
    for (int j = 0; j < NB; ++j) host[j + static_cast<size_t>(j) * MB] = std::pow(10.0, -8.0 * j / std::max(1, NB - 1));
    const int B = 8;
    double* dA = c.buf("tune_a", static_cast<size_t>(MB) * NB * B);
    double* dQ = c.buf("tune_q", static_cast<size_t>(MB) * NB * B);
    for (int b = 0; b < B; ++b)
      ck(cudaMemcpyAsync(dA + static_cast<size_t>(b) * MB * NB, host.data(), host.size() * sizeof(double),
                         cudaMemcpyHostToDevice, c.stream()));
    std::vector<const double*> pa(B);
    std::vector<double*> pq(B);
    std::vector<int64_t> ld(B, MB);
    std::vector<int> mm(B, MB), nn(B, NB), inf(B, 0), its(B, 0);
    for (int b = 0; b < B; ++b) {
      pa[b] = dA + static_cast<size_t>(b) * MB * NB;
      pq[b] = dQ + static_cast<size_t>(b) * MB * NB;
    }
    ck(cudaEventRecord(c.event(0), c.stream()));  // the probe inputs are on the device
    ck(cudaStreamWaitEvent(wc.stream(), c.event(0), 0));
    double t[2];
    for (int rep = 0; rep < 2; ++rep) {
      const int nb_members = rep == 0 ? 1 : B;
      std::vector<int> idx(nb_members);
      for (int b = 0; b < nb_members; ++b) idx[b] = b;
      BatchStats bs;
      // warm-up to the steady state the solver runs in: the first call sizes the workspace,
      // the second captures the bucket's graph (ZOLO_OPT_BATCH_GRAPH), the timed one replays it
      for (int w = 0; w < 2; ++w)
        qdwh_bucket(wc, idx, MB, NB, mm.data(), nn.data(), pa.data(), ld.data(), pq.data(), ld.data(), nullptr,
                    nullptr, inf.data(), its.data(), &bs);
      EventTimer tm(wc.stream());
      qdwh_bucket(wc, idx, MB, NB, mm.data(), nn.data(), pa.data(), ld.data(), pq.data(), ld.data(), nullptr,
                  nullptr, inf.data(), its.data(), &bs);
      t[rep] = tm.stop();
    }
    const double w = std::max(1e-3, (t[1] - t[0]) / (B - 1));
    lat[k] = std::max(0.0, t[0] - w);
    flops_at[k] = batch_member_flops(MB, NB);
    rate[k] = flops_at[k] / w / 1e9;  // TFLOP/s
  }
  BatchCostModel md = c.batch_model;
  // latency: least-squares line in NB/32 through the three probes
  double sx = 0, sy = 0, sxx = 0, sxy = 0;
  for (int k = 0; k < 3; ++k) {
    const double x = sizes[k] / 32.0;
    sx += x;
    sy += lat[k];
    sxx += x * x;
    sxy += x * lat[k];
  }
  const double den = 3.0 * sxx - sx * sx;
  md.lat1 = std::max(0.0, (3.0 * sxy - sx * sy) / den);
  md.lat0 = std::max(0.0, (sy - md.lat1 * sx) / 3.0);
  // rate(NB) = R NB / (NB + h) through the two larger probes
  const double n1 = sizes[1], n2 = sizes[2], r1 = rate[1], r2 = rate[2];
  const double h = (r2 - r1) / (r1 / n1 - r2 / n2);
  if (std::isfinite(h) && h > 0.0 && r2 > 0.0) {
    md.nhalf = h;
    md.rate_tflops = r2 * (n2 + h) / n2;
  } else if (r2 > 0.0) {
    md.nhalf = 0.0;
    md.rate_tflops = r2;
  }
  // a fit outside what the FP64 tensor path can do (noise in the small probes) keeps the
  // previous rate terms
  if (!(md.rate_tflops > 0.5 && md.rate_tflops < 60.0 && md.nhalf < 8192.0)) {
    md.rate_tflops = c.batch_model.rate_tflops;
    md.nhalf = c.batch_model.nhalf;
  }
  c.batch_model = md;
  return 0;
}

}  // namespace zolo
