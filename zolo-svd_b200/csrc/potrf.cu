// Leaf kernels of the recursive Cholesky / triangular solves (FP64).
// The recursion (linalg.cpp) turns all O(n^3) work into DMMA GEMMs; these
// kernels factor the nb x nb diagonal blocks (nb <= 64) in shared memory and
// also return each block's inverse, which the triangular solves use at their
// leaves (so no separate inversion pass is needed).
#include "common.cuh"
#include "kernels.h"

namespace zolo {

namespace {

constexpr int LEAF = 64;
constexpr int LDS = LEAF + 1;
constexpr int PT = 256;
constexpr int MAXE = (LEAF * (LEAF + 1) / 2 + PT - 1) / PT;  // lower-triangle elements per thread

// x = l^{-1} for lower-triangular l (nb x nb in shared memory, ld LDS).
// Column j of the inverse is owned by a group of 4 lanes; lane q of the group keeps rows
// q, q+4, ... of the column in registers and the substitution runs right-looking: at row i
// the owning lane forms x_i = b_i / l_ii (one multiply by a reciprocal computed up front),
// the group shares it by a shuffle and every lane updates its rows below i.  Columns are
// independent, so only the 4-lane groups exchange data; the per-row work is independent
// FMAs, not a dependent dot product.
__device__ void tri_inverse_smem(int nb, const double* l, double* x) {
  __shared__ double rdiag[LEAF];
  for (int i = threadIdx.x; i < nb; i += blockDim.x) rdiag[i] = 1.0 / l[i + i * LDS];
  __syncthreads();
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int j = warp * 8 + (lane >> 2);
  const int q = lane & 3;
  const int base = lane & ~3;
  double b[LEAF / 4];
#pragma unroll
  for (int u = 0; u < LEAF / 4; ++u) b[u] = (q + 4 * u == j) ? 1.0 : 0.0;  // e_j
#pragma unroll
  for (int t = 0; t < LEAF / 4; ++t) {
#pragma unroll
    for (int qi = 0; qi < 4; ++qi) {
      const int i = 4 * t + qi;
      if (i < nb) {
        double xi = (q == qi) ? b[t] * rdiag[i] : 0.0;
        xi = __shfl_sync(0xffffffffu, xi, base | qi);
        if (q == qi) b[t] = xi;
#pragma unroll
        for (int u = 0; u < LEAF / 4; ++u)
          if (q + 4 * u > i && q + 4 * u < nb) b[u] -= l[q + 4 * u + i * LDS] * xi;
      }
    }
  }
  if (j < nb) {
#pragma unroll
    for (int u = 0; u < LEAF / 4; ++u)
      if (q + 4 * u < nb) x[q + 4 * u + j * LDS] = b[u];
  }
}

__global__ void __launch_bounds__(PT) potrf_leaf_kernel(int nb, double* A, int64_t lda, int64_t strideA, int* info,
                                                        int info_offset, double* Dinv, int64_t strideD) {
  extern __shared__ double sm[];
  double* a = sm;
  double* x = sm + LEAF * LDS;
  double* Ab = A + blockIdx.x * strideA;
  const int tid = threadIdx.x;
  // this thread's lower-triangle elements (packed column by column)
  int ei[MAXE], ej[MAXE];
  const int ne = nb * (nb + 1) / 2;
#pragma unroll
  for (int q = 0; q < MAXE; ++q) {
    int e = tid + q * PT;
    ei[q] = -1;
    ej[q] = 0;
    if (e < ne) {
      int j = 0;
      while (e >= nb - j) {
        e -= nb - j;
        ++j;
      }
      ei[q] = j + e;
      ej[q] = j;
    }
  }
#pragma unroll
  for (int q = 0; q < MAXE; ++q)
    if (ei[q] >= 0) a[ei[q] + ej[q] * LDS] = Ab[ei[q] + ej[q] * lda];
  __syncthreads();
  // right-looking elimination on unscaled columns: one barrier per step
  for (int k = 0; k < nb; ++k) {
    const double d = a[k + k * LDS];
    const double inv = (d > 0.0) ? 1.0 / d : 0.0;
#pragma unroll
    for (int q = 0; q < MAXE; ++q)
      if (ei[q] >= 0 && ej[q] > k) a[ei[q] + ej[q] * LDS] -= a[ei[q] + k * LDS] * a[ej[q] + k * LDS] * inv;
    __syncthreads();
  }
  if (tid == 0 && info) {
    for (int k = 0; k < nb; ++k)
      if (!(a[k + k * LDS] > 0.0)) {  // LAPACK INFO = first non-positive pivot
        atomicCAS(info + blockIdx.x, 0, info_offset + k + 1);
        break;
      }
  }
  // L(i,j) = a(i,j) / sqrt(d_j), L(j,j) = sqrt(d_j)
  double lv[MAXE];
#pragma unroll
  for (int q = 0; q < MAXE; ++q) {
    lv[q] = 0.0;
    if (ei[q] >= 0) {
      const double dj = a[ej[q] + ej[q] * LDS];
      const double sj = dj > 0.0 ? sqrt(dj) : 1.0;
      lv[q] = (ei[q] == ej[q]) ? sj : a[ei[q] + ej[q] * LDS] / sj;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < MAXE; ++q)
    if (ei[q] >= 0) {
      a[ei[q] + ej[q] * LDS] = lv[q];
      Ab[ei[q] + ej[q] * lda] = lv[q];
    }
  for (int e = tid; e < nb * nb; e += PT) {
    const int i = e % nb, j = e / nb;
    if (i < j) a[i + j * LDS] = 0.0;
  }
  __syncthreads();
  if (Dinv) {
    tri_inverse_smem(nb, a, x);
    __syncthreads();
    double* Db = Dinv + blockIdx.x * strideD;
    for (int e = tid; e < nb * nb; e += PT) {
      const int i = e % nb, j = e / nb;
      Db[i + j * LEAF] = x[i + j * LDS];
    }
  }
}

// Inverses of the diagonal blocks of a lower-triangular n x n matrix:
// block kb (rows/cols kb*64 ..) of batch entry b goes to Dinv + (b*nblk + kb)*64*64.
__global__ void __launch_bounds__(PT) trtri_blocks_kernel(int n, const double* L, int64_t ldl, int64_t strideL,
                                                          double* Dinv, int nblk) {
  extern __shared__ double sm[];
  double* l = sm;
  double* x = sm + LEAF * LDS;
  const int kb = blockIdx.x, b = blockIdx.y;
  const int o = kb * LEAF;
  const int nb = min(LEAF, n - o);
  const double* Lb = L + b * strideL + o + static_cast<int64_t>(o) * ldl;
  for (int e = threadIdx.x; e < nb * nb; e += PT) {
    const int i = e % nb, j = e / nb;
    l[i + j * LDS] = (i >= j) ? Lb[i + static_cast<int64_t>(j) * ldl] : 0.0;
  }
  __syncthreads();
  tri_inverse_smem(nb, l, x);
  __syncthreads();
  double* Db = Dinv + (static_cast<int64_t>(b) * nblk + kb) * LEAF * LEAF;
  for (int e = threadIdx.x; e < nb * nb; e += PT) {
    const int i = e % nb, j = e / nb;
    Db[i + j * LEAF] = x[i + j * LDS];
  }
}

constexpr int SMEM_BYTES = 2 * LEAF * LDS * 8;

}  // namespace

cudaError_t potrf_leaf(int nb, double* A, int64_t lda, int64_t strideA, int batch, int* info, int info_offset,
                       double* Dinv, int64_t strideD, cudaStream_t st) {
  if (nb <= 0 || batch <= 0) return cudaSuccess;
  if (nb > LEAF) return cudaErrorInvalidValue;
  static std::atomic<int> attr_set[kMaxDevices];
  const cudaError_t attr = once_per_device(attr_set, [] {
    return cudaFuncSetAttribute(potrf_leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  });
  if (attr != cudaSuccess) return attr;
  potrf_leaf_kernel<<<batch, PT, SMEM_BYTES, st>>>(nb, A, lda, strideA, info, info_offset, Dinv, strideD);
  return cudaGetLastError();
}

cudaError_t trtri_blocks(int n, const double* L, int64_t ldl, int64_t strideL, double* Dinv, int batch,
                         cudaStream_t st) {
  if (n <= 0 || batch <= 0) return cudaSuccess;
  static std::atomic<int> attr_set[kMaxDevices];
  const cudaError_t attr = once_per_device(attr_set, [] {
    return cudaFuncSetAttribute(trtri_blocks_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_BYTES);
  });
  if (attr != cudaSuccess) return attr;
  const int nblk = (n + LEAF - 1) / LEAF;
  trtri_blocks_kernel<<<dim3(nblk, batch), PT, SMEM_BYTES, st>>>(n, L, ldl, strideL, Dinv, nblk);
  return cudaGetLastError();
}

}  // namespace zolo
