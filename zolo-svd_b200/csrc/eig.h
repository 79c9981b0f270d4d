// Symmetric eigensolver (spectral divide-and-conquer with Jacobi leaves),
// ZoloEig and the SVD assembly.  See eig.cpp.
#pragma once
#include <cstdint>

#include "context.h"

namespace zolo {

constexpr int kJacobiLeaf = 64;

struct EigStats {
  int splits = 0;
  int leaves = 0;
  int qdwh_calls = 0;
  int qdwh_iterations = 0;
  int subspace_passes = 0;
  int max_jacobi_sweeps = 0;
  double max_split_residual = 0.0;  // max ||V2^T H V1||_F / ||H||_F over the splits
  double flops = 0.0;
  int batched_nodes = 0;  // nodes whose first-candidate QDWH ran in a level's batched solve
  int zolo_calls = 0;     // nodes whose first candidate's polar factor came from Zolo-PD
  int64_t reallocs = 0;   // workspace buffers replaced by larger ones during the call
  // device ms (CUDA events on the calling stream): each top-down level's splits, the
  // Jacobi leaves, the bottom-up back-transformation, the whole call
  int levels = 0;
  double ms_level[16] = {0};
  double ms_leaves = 0.0, ms_back = 0.0, ms_total = 0.0;
  // host wall ms summed over the levels: diagonals read back, the batched QDWH solves, the
  // concurrent splits, freeing the split nodes' matrices
  double wall_diag = 0.0, wall_batch = 0.0, wall_split = 0.0, wall_free = 0.0;
};

// H = Z diag(w) Z^T for symmetric H (n x n); w ascending.  Returns 0 or > 0 on failure.
int syev_dc(Context& c, int n, const double* dH, int64_t ldh, double* dW, double* dZ, int64_t ldz, EigStats* es);

// ZoloEig (ZoloEig.f90:78-102 with PQDWHSUBIT, pqdwhsubit.f90:227-312): from the polar
// factor Q of A - sigma I, the Rk = round(||(Q - I)/2||_F^2) eigenpairs of A below sigma:
// eigenvalues dW (Rk), eigenvectors dZ (n x Rk); optionally the subspace basis V (n x n)
// and V^T A V.
int zoloeig(Context& c, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, int* rk,
            double* dW, double* dZ, int64_t ldz, double* dVfull, int64_t ldv, double* dE, int64_t lde);

// A = U diag(s) V^T (m >= n) by a polar decomposition (algo 0 = QDWH, 1 = Zolo-PD with rk
// terms) followed by syev_dc of H; s ascending (the order ZoloCHK1 gets from ELPA).
int svd(Context& c, int m, int n, const double* dA, int64_t lda, int algo, int rk, double* dU, int64_t ldu,
        double* dS, double* dV, int64_t ldv, EigStats* es);

}  // namespace zolo
