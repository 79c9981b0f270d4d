// Leaf kernels of the recursive Cholesky / triangular solves (FP64).
// The recursion itself (host side, linalg.cpp) turns all O(n^3) work into DMMA
// GEMMs; these kernels factor / invert the nb x nb diagonal blocks (nb <= 64)
// in shared memory, one CTA per batch entry.
#include "common.cuh"
#include "kernels.h"

namespace zolo {

namespace {

constexpr int LEAF = 64;
constexpr int LDS = LEAF + 1;

__global__ void __launch_bounds__(256) potrf_leaf_kernel(int nb, double* A, int64_t lda, int64_t strideA,
                                                         int* info, int info_offset) {
  __shared__ double a[LEAF * LDS];
  __shared__ int bad;
  double* Ab = A + blockIdx.x * strideA;
  const int tid = threadIdx.x;
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    a[i + j * LDS] = (i >= j) ? Ab[i + j * lda] : 0.0;
  }
  if (tid == 0) bad = 0;
  __syncthreads();
  for (int k = 0; k < nb; ++k) {
    if (tid == 0) {
      const double d = a[k + k * LDS];
      if (!(d > 0.0)) {  // not positive definite (or NaN): LAPACK's INFO = k+1
        if (!bad && info) atomicCAS(info + blockIdx.x, 0, info_offset + k + 1);
        bad = 1;
        a[k + k * LDS] = 1.0;
      } else {
        a[k + k * LDS] = sqrt(d);
      }
    }
    __syncthreads();
    const double piv = a[k + k * LDS];
    for (int i = k + 1 + tid; i < nb; i += blockDim.x) a[i + k * LDS] /= piv;
    __syncthreads();
    const int rem = nb - k - 1;
    for (int e = tid; e < rem * rem; e += blockDim.x) {
      const int i = k + 1 + e % rem, j = k + 1 + e / rem;
      if (i >= j) a[i + j * LDS] -= a[i + k * LDS] * a[j + k * LDS];
    }
    __syncthreads();
  }
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    if (i >= j) Ab[i + j * lda] = a[i + j * LDS];
  }
}

// Linv = L^{-1} for lower-triangular L (nb <= 64); zeros above the diagonal.
// Thread j forward-substitutes column j of the inverse directly in global memory.
__global__ void __launch_bounds__(LEAF) trtri_leaf_kernel(int nb, const double* L, int64_t ldl, int64_t strideL,
                                                         double* Linv, int64_t ldi, int64_t strideI) {
  __shared__ double l[LEAF * LDS];
  const double* Lb = L + blockIdx.x * strideL;
  double* Ib = Linv + blockIdx.x * strideI;
  const int tid = threadIdx.x;
  for (int e = tid; e < nb * nb; e += blockDim.x) {
    const int i = e % nb, j = e / nb;
    l[i + j * LDS] = (i >= j) ? Lb[i + j * ldl] : 0.0;
  }
  __syncthreads();
  const int j = tid;
  if (j < nb) {
    double* x = Ib + j * ldi;
    for (int i = 0; i < j; ++i) x[i] = 0.0;
    x[j] = 1.0 / l[j + j * LDS];
    for (int i = j + 1; i < nb; ++i) {
      double s = 0.0;
      for (int k = j; k < i; ++k) s += l[i + k * LDS] * x[k];
      x[i] = -s / l[i + i * LDS];
    }
  }
}

}  // namespace

cudaError_t potrf_leaf(int nb, double* A, int64_t lda, int64_t strideA, int batch, int* info, int info_offset,
                       cudaStream_t st) {
  if (nb <= 0 || batch <= 0) return cudaSuccess;
  if (nb > LEAF) return cudaErrorInvalidValue;
  potrf_leaf_kernel<<<batch, 256, 0, st>>>(nb, A, lda, strideA, info, info_offset);
  return cudaGetLastError();
}

cudaError_t trtri_leaf(int nb, const double* L, int64_t ldl, int64_t strideL, double* Linv, int64_t ldi,
                       int64_t strideI, int batch, cudaStream_t st) {
  if (nb <= 0 || batch <= 0) return cudaSuccess;
  if (nb > LEAF) return cudaErrorInvalidValue;
  trtri_leaf_kernel<<<batch, LEAF, 0, st>>>(nb, L, ldl, strideL, Linv, ldi, strideI);
  return cudaGetLastError();
}

}  // namespace zolo
