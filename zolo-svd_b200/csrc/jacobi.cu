// Batched two-sided cyclic Jacobi eigensolver for the leaves of the spectral
// divide-and-conquer (symmetric, n <= 64), one CTA per leaf, everything in
// shared memory.  Parallel round-robin ordering: each step rotates n/2
// disjoint index pairs simultaneously (rows, then columns), n-1 steps per
// sweep, until the off-diagonal mass is below (n * eps)^2 of the diagonal
// mass.  Rotation: Golub & Van Loan, Matrix Computations, Alg. 8.5.1
// (symmetric Schur decomposition), applied as A <- J^T A J, V <- V J.
// The leaf eigensolver replaces the reference's ELPA / PDSYEVD call on the
// final blocks (elpa_pdsyevd2.F90:199-200, ZoloEig.f90:98-99).
#include "common.cuh"
#include "kernels.h"

namespace zolo {

namespace {

constexpr int JN = 64;
constexpr int JLD = JN + 1;
constexpr int JT = 256;

__global__ void __launch_bounds__(JT) jacobi_kernel(const JacobiLeaf* leaves, int max_sweeps, int* sweeps_out) {
  extern __shared__ double sm[];
  double* a = sm;
  double* v = sm + JN * JLD;
  __shared__ double cs[JN / 2][2];
  __shared__ int pp[JN / 2], qq[JN / 2];
  __shared__ double red[JT / 32][2];
  __shared__ int stop;
  const JacobiLeaf L = leaves[blockIdx.x];
  const int n = L.n;
  const int tid = threadIdx.x;
  const int N = (n + 1) / 2 * 2;  // players (one dummy when n is odd)
  const int np = N / 2;
  for (int e = tid; e < n * n; e += JT) {
    const int i = e % n, j = e / n;
    a[i + j * JLD] = L.A[i + static_cast<int64_t>(j) * L.lda];
    v[i + j * JLD] = (i == j) ? 1.0 : 0.0;
  }
  __syncthreads();
  const double eps = 1.1102230246251565e-16;
  int sweep = 0;
  for (; sweep < max_sweeps; ++sweep) {
    // convergence test: off-diagonal vs diagonal mass
    double off = 0.0, dg = 0.0;
    for (int e = tid; e < n * n; e += JT) {
      const int i = e % n, j = e / n;
      const double x = a[i + j * JLD];
      if (i == j) dg += x * x;
      else off += x * x;
    }
    off = warp_sum(off);
    dg = warp_sum(dg);
    if ((tid & 31) == 0) {
      red[tid >> 5][0] = off;
      red[tid >> 5][1] = dg;
    }
    __syncthreads();
    if (tid == 0) {
      double o = 0.0, d = 0.0;
      for (int q = 0; q < JT / 32; ++q) {
        o += red[q][0];
        d += red[q][1];
      }
      const double tol = static_cast<double>(n) * eps;
      stop = (o <= tol * tol * d) || (o == 0.0);
    }
    __syncthreads();
    if (stop) break;
    for (int step = 0; step < N - 1; ++step) {
      // round-robin pairing: position 0 fixed, positions 1..N-1 rotate by `step`
      if (tid < np) {
        auto player = [&](int pos) { return pos == 0 ? 0 : ((pos - 1 + step) % (N - 1)) + 1; };
        int p = player(tid), q = player(N - 1 - tid);
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        pp[tid] = p;
        qq[tid] = q;
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = a[p + q * JLD];
          const double app = a[p + p * JLD], aqq = a[q + q * JLD];
          if (apq != 0.0 && fabs(apq) > 1e-300) {
            const double tau = (aqq - app) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        cs[tid][0] = c;
        cs[tid][1] = s;
      }
      __syncthreads();
      // rows p, q of A for every column
      for (int e = tid; e < np * n; e += JT) {
        const int pi = e / n, k = e - pi * n;
        const int p = pp[pi], q = qq[pi];
        if (q >= n) continue;
        const double c = cs[pi][0], s = cs[pi][1];
        const double ap = a[p + k * JLD], aq = a[q + k * JLD];
        a[p + k * JLD] = c * ap - s * aq;
        a[q + k * JLD] = s * ap + c * aq;
      }
      __syncthreads();
      // columns p, q of A and V for every row
      for (int e = tid; e < np * n; e += JT) {
        const int pi = e / n, k = e - pi * n;
        const int p = pp[pi], q = qq[pi];
        if (q >= n) continue;
        const double c = cs[pi][0], s = cs[pi][1];
        const double ap = a[k + p * JLD], aq = a[k + q * JLD];
        a[k + p * JLD] = c * ap - s * aq;
        a[k + q * JLD] = s * ap + c * aq;
        const double vp = v[k + p * JLD], vq = v[k + q * JLD];
        v[k + p * JLD] = c * vp - s * vq;
        v[k + q * JLD] = s * vp + c * vq;
      }
      __syncthreads();
    }
  }
  for (int i = tid; i < n; i += JT) L.w[i] = a[i + i * JLD];
  for (int e = tid; e < n * n; e += JT) {
    const int i = e % n, j = e / n;
    L.V[i + static_cast<int64_t>(j) * L.ldv] = v[i + j * JLD];
  }
  if (tid == 0 && sweeps_out) sweeps_out[blockIdx.x] = sweep;
}

}  // namespace

cudaError_t jacobi_leaves(const JacobiLeaf* d_leaves, int count, int max_sweeps, int* d_sweeps, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  constexpr int smem = 2 * JN * JLD * 8;
  static std::atomic<int> attr_set[kMaxDevices];
  const cudaError_t attr = once_per_device(
      attr_set, [] { return cudaFuncSetAttribute(jacobi_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem); });
  if (attr != cudaSuccess) return attr;
  jacobi_kernel<<<count, JT, smem, st>>>(d_leaves, max_sweeps, d_sweeps);
  return cudaGetLastError();
}

}  // namespace zolo
