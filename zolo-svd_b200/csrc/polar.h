// Device-side drivers of the polar decompositions (QDWH-PD and Zolo-PD) and
// the singular-value bounds they start from.
#pragma once
#include <cstdint>

#include "context.h"

namespace zolo {

enum BoundsMode {
  BOUNDS_PQDWHFACS = 0,  // beta = ||X0||_1 / (sqrt(n) ||R^-1||_1)   (pqdwhfacs.f90:325-344 form)
  BOUNDS_ZOLOPD = 1,     // beta = 1 / (sqrt(n) ||R^-1||_1)           (zolopd.f90 / test_zolodrv1.f90 form)
  BOUNDS_FROB = 2,       // beta = 1 / ||R^-1||_F: still <= sigma_min(X0), never below mode 1's
  BOUNDS_NORM2 = 3,      // mode 2's beta, and alpha lowered from ||A||_F to a guaranteed upper bound of
                         // ||A||_2, (sum_i sigma_i^16)^(1/16) from (R^T R)^4 (norm2_upper in polar.cpp)
};

// alpha = ||A - sigma I||_F ; beta from R of (A - sigma I)/alpha = QR.  Returns info (0 ok).
// BOUNDS_NORM2: alpha is then the two-norm bound and beta the sigma_min bound of A/alpha; the
// QR left in the workspace is that of A/alpha_fro (reported in *alpha_fro when not null).
int bounds(Context& c, int m, int n, double sigma, const double* dA, int64_t lda, BoundsMode mode, double* alpha,
           double* beta, double* alpha_fro = nullptr);

struct QdwhOpts {
  char sym = 'N';
  double sigma = 0.0;
  BoundsMode bounds = BOUNDS_PQDWHFACS;
  int maxit = 12;           // loop runs while IT <= maxit; < 0 = no cap (zolopd.f90)
  bool left_solve = false;  // zolopd.f90: W^{-1} X instead of X W^{-1}
};

// Q = polar factor of A - sigma I (m x n, m >= n); H = sym(Q^T A) when dH != nullptr.
int qdwh(Context& c, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq, double* dH, int64_t ldh,
         const QdwhOpts& o);

// A Householder QR of A/alpha already computed (by bounds): the factored matrix W
// (R on and above the diagonal, reflectors below; ld ldw) and its panel factors T.
struct Prefactored {
  const double* W;
  int64_t ldw;
  const double* T;
  double alpha;  // the factored matrix is A / alpha
};

// Zolo-PD of As/(alpha*beta) with rk terms (pzolopd1.f90:280-487); H as above.  With
// `pf` (the QR of A/alpha) the first iteration, if it takes the QR form with the QR of
// X shared by the terms, reuses it: X0 = A/(alpha beta) has the same Q and R/beta.
int zolo_pd(Context& c, char sym, int rk, int m, int n, double alpha, double beta, const double* dA, int64_t lda,
            double* dQ, int64_t ldq, double* dH, int64_t ldh, int maxit = 6, const Prefactored* pf = nullptr);

// bounds (ZOLOPD form) + Zolo-PD + H in one call, the flow of the reference's driver
// (test_zolodrv1.f90:167-198): the QR of A/alpha that gives beta is reused by the first
// Zolo-PD iteration.  Returns INFO; alpha and beta are reported in the stats.
// The term plan (ZOLO_OPT_TERM_PLAN) from CON on: terms[k] and qr_form[k] (1 = QR form) of
// each predicted Zolo-PD iteration and the predicted Newton-Schulz steps; returns the number
// of iterations (at most maxlen), or -1 for bad arguments.  Host only.
int plan_terms(double con, int rk, int m, int n, bool prefactored, int* terms, int* qr_form, int maxlen,
               int* ns_steps);
int zolo_polar(Context& c, int rk, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq, double* dH,
               int64_t ldh);

// QDWH-PD (PQDWHFACS steps and bounds, SYM = 'N', SIGMA = 0) of `count` matrices of
// different sizes.  Members are grouped into buckets of one padded size NB (a ladder of
// multiples of 32) and padded exactly: A' = [[A, 0], [0, tau I], [0, 0]] with
// tau = ||A||_F / sqrt(n), which lies in [sigma_min, sigma_max], so the condition number
// is unchanged and polar(A') = diag(polar(A), I), H' = diag(H, tau I).  Each bucket runs
// as one batched solve with per-member weights and convergence.  info[i] = 0, or > 0
// when member i's bounds or Cholesky failed (its outputs are then undefined).
struct BatchStats {
  int buckets = 0;
  int max_iterations = 0;
  double flops = 0.0;       // executed FP64 flops, padding included
  double flops_useful = 0.0;  // the same work counted on the unpadded sizes
  double ms = 0.0;
  double predicted_ms = 0.0;  // the bucket plan's predicted time (cost model)
  // buckets by how their iterations ran (ZOLO_OPT_BATCH_GRAPH)
  int graph_replays = 0;    // a cached graph launched
  int graph_captures = 0;   // captured, instantiated and launched
  int eager_scheduled = 0;  // the schedule's launches issued eagerly (first call of a shape)
  int sync_loops = 0;       // the host-synchronized loop (option off, or profiling)
  int restarts = 0;         // a Cholesky step failed: rerun through the synchronized loop
  int resumes = 0;          // a member continued in the synchronized loop after the schedule
};
int qdwh_batch(Context& c, int count, const int* m, const int* n, const double* const* dA, const int64_t* lda,
               double* const* dQ, const int64_t* ldq, double* const* dH, const int64_t* ldh, int* info,
               int* iterations, BatchStats* bs);

// Measures the batched solver's cost model on this GPU (probe buckets at three sizes) into
// c.batch_model; the bucket plan of qdwh_batch uses it.  Returns 0.
int batch_autotune(Context& c);

// H = (Q^T A + A^T Q)/2
void form_h(Context& c, int m, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, double* dH,
            int64_t ldh);

}  // namespace zolo
