// Device-side drivers of the polar decompositions (QDWH-PD and Zolo-PD) and
// the singular-value bounds they start from.
#pragma once
#include <cstdint>

#include "context.h"

namespace zolo {

enum BoundsMode {
  BOUNDS_PQDWHFACS = 0,  // beta = ||X0||_1 / (sqrt(n) ||R^-1||_1)   (pqdwhfacs.f90:325-344 form)
  BOUNDS_ZOLOPD = 1,     // beta = 1 / (sqrt(n) ||R^-1||_1)           (zolopd.f90 / test_zolodrv1.f90 form)
};

// alpha = ||A - sigma I||_F ; beta from R of (A - sigma I)/alpha = QR.  Returns info (0 ok).
int bounds(Context& c, int m, int n, double sigma, const double* dA, int64_t lda, BoundsMode mode, double* alpha,
           double* beta);

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

// Zolo-PD of As/(alpha*beta) with rk terms (pzolopd1.f90:280-487); H as above.
int zolo_pd(Context& c, char sym, int rk, int m, int n, double alpha, double beta, const double* dA, int64_t lda,
            double* dQ, int64_t ldq, double* dH, int64_t ldh, int maxit = 6);

// H = (Q^T A + A^T Q)/2
void form_h(Context& c, int m, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, double* dH,
            int64_t ldh);

}  // namespace zolo
