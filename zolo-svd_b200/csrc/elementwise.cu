// HBM-bound FP64 kernels: scaling/copies, the stacked [X; sqrt(c) I] form, the
// shifted Gram copy, norms, and the fused FormX2 / QDWH combine with the
// ||X_{k+1} - X_k||_F reduction.  Reductions are deterministic: per-block
// partials followed by one fixed-order block sum.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace zolo {

namespace {

constexpr int TPB = 256;

inline int grid_for(int64_t work, int per_block = TPB) {
  int64_t b = (work + per_block - 1) / per_block;
  b = std::min<int64_t>(b, static_cast<int64_t>(num_sms()) * 8);
  return static_cast<int>(std::max<int64_t>(b, 1));
}

__global__ void scale_copy_kernel(int m, int n, double s, const double* __restrict__ src, int64_t lds,
                                  int64_t strideS, double* dst, int64_t ldd, int64_t strideD,
                                  double diag_add) {
  const int b = blockIdx.y;
  const double* S = src + b * strideS;
  double* D = dst + b * strideD;
  const int64_t total = static_cast<int64_t>(m) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    double v = s * S[i + j * lds];
    if (i == j) v += diag_add;
    D[i + j * ldd] = v;
  }
}

__global__ void form_stack_kernel(int m, int mpad, int n, const double* __restrict__ X, int64_t ldx, double* W,
                                  int64_t ldw, int64_t strideW, const double* s_vec, double s_scalar,
                                  int x_upper, int64_t strideX) {
  const int b = blockIdx.y;
  X += b * strideX;
  double* Wb = W + b * strideW;
  const double s = s_vec ? s_vec[b] : s_scalar;
  const int rows = mpad + n;
  const int64_t total = static_cast<int64_t>(rows) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % rows), j = static_cast<int>(e / rows);
    double v;
    if (i < m) v = (x_upper && i > j) ? 0.0 : X[i + j * ldx];
    else v = (i - mpad == j) ? s : 0.0;
    Wb[i + j * ldw] = v;
  }
}

__global__ void shift_lower_kernel(int n, const double* __restrict__ G, int64_t ldg, double* W,
                                   int64_t ldw, int64_t strideW, const double* c_vec) {
  const int b = blockIdx.y;
  double* Wb = W + b * strideW;
  const double c = c_vec[b];
  const int64_t total = static_cast<int64_t>(n) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (i < j) continue;
    double v = G[i + j * ldg];
    if (i == j) v += c;
    Wb[i + j * ldw] = v;
  }
}

template <int BS>
__device__ double block_sum(double v, double* sh) {
  v = warp_sum(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    for (int i = 0; i < BS / 32; ++i) r += sh[i];
  }
  __syncthreads();
  return r;
}

__global__ void frob2_kernel(int m, int n, const double* __restrict__ X, int64_t ldx, double* partial) {
  __shared__ double sh[TPB / 32];
  const int64_t total = static_cast<int64_t>(m) * n;
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    const double v = X[i + j * ldx];
    s += v * v;
  }
  s = block_sum<TPB>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void reduce_sum_kernel(const double* partial, int count, double* out) {
  __shared__ double sh[TPB / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s += partial[i];
  s = block_sum<TPB>(s, sh);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void colsum_abs_kernel(int m, int n, const double* __restrict__ X, int64_t ldx, double* colsum) {
  __shared__ double sh[TPB / 32];
  for (int j = blockIdx.x; j < n; j += gridDim.x) {
    double s = 0.0;
    for (int i = threadIdx.x; i < m; i += blockDim.x) s += fabs(X[i + j * ldx]);
    s = block_sum<TPB>(s, sh);
    if (threadIdx.x == 0) colsum[j] = s;
  }
}

__global__ void max_kernel(const double* v, int count, double* out) {
  __shared__ double sh[TPB];
  double s = 0.0;
  for (int i = threadIdx.x; i < count; i += blockDim.x) s = fmax(s, v[i]);
  sh[threadIdx.x] = s;
  __syncthreads();
  for (int o = TPB / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sh[threadIdx.x] = fmax(sh[threadIdx.x], sh[threadIdx.x + o]);
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = sh[0];
}

// X_new = cx*X + cz*sum_q Z_q ; partial = ||X_new - X||^2 per block.  In place on X.
__global__ void combine_kernel(int m, int n, double* X, int64_t ldx, const double* __restrict__ Z,
                               int64_t ldz, int64_t strideZ, int nz, double cx, double cz,
                               const double* __restrict__ cz_vec, double* partial) {
  __shared__ double sh[TPB / 32];
  const int64_t total = static_cast<int64_t>(m) * n;
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    const double x = X[i + j * ldx];
    double z = 0.0;
    if (cz_vec) {
      for (int q = 0; q < nz; ++q) z += cz_vec[q] * Z[q * strideZ + i + j * ldz];
    } else {
      for (int q = 0; q < nz; ++q) z += Z[q * strideZ + i + j * ldz];
      z *= cz;
    }
    const double xn = cx * x + z;
    const double d = x - xn;
    s += d * d;
    X[i + j * ldx] = xn;
  }
  s = block_sum<TPB>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void symmetrize_kernel(int n, double* B, int64_t ldb) {
  const int64_t total = static_cast<int64_t>(n) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (i <= j) continue;  // each pair once, by the lower element
    const double a = B[i + j * ldb], b = B[j + i * ldb];
    const double h = 0.5 * b + 0.5 * a;
    B[i + j * ldb] = h;
    B[j + i * ldb] = h;
  }
}

__global__ void transpose_kernel(int m, int n, const double* __restrict__ A, int64_t lda, double* B,
                                 int64_t ldb) {
  __shared__ double tile[32][33];
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int jj = threadIdx.y; jj < 32; jj += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + jj;
    if (i < m && j < n) tile[jj][threadIdx.x] = A[i + static_cast<int64_t>(j) * lda];
  }
  __syncthreads();
  for (int ii = threadIdx.y; ii < 32; ii += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + ii;
    if (i < m && j < n) B[j + static_cast<int64_t>(i) * ldb] = tile[threadIdx.x][ii];
  }
}

// Newton-Schulz step matrix from the lower triangle of G = X^T X: G <- (3I - G)/2
// (both triangles written; only when `write`) and partial[block] = sum of (G - I)^2
// over all entries.
__global__ void ns_prepare_kernel(int n, double* G, int64_t ldg, int write, double* partial) {
  __shared__ double sh[TPB / 32];
  const int64_t total = static_cast<int64_t>(n) * n;
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (i < j) continue;
    const double g = G[i + j * ldg];
    const double d = (i == j) ? g - 1.0 : g;
    s += (i == j) ? d * d : 2.0 * d * d;
    if (!write) continue;
    const double v = (i == j) ? 1.5 - 0.5 * g : -0.5 * g;
    G[i + j * ldg] = v;
    if (i != j) G[j + i * ldg] = v;
  }
  s = block_sum<TPB>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

// B(j, i) = B(i, j) for i > j: the lower triangle copied to the upper one
__global__ void mirror_lower_kernel(int n, double* B, int64_t ldb) {
  const int64_t total = static_cast<int64_t>(n) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (i > j) B[j + static_cast<int64_t>(i) * ldb] = B[i + static_cast<int64_t>(j) * ldb];
  }
}

__global__ void copy_upper_kernel(int n, const double* __restrict__ A, int64_t lda, double scale, double* B,
                                  int64_t ldb) {
  const int64_t total = static_cast<int64_t>(n) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    B[i + static_cast<int64_t>(j) * ldb] = (i <= j) ? scale * A[i + static_cast<int64_t>(j) * lda] : 0.0;
  }
}

__global__ void set_identity_kernel(int m, int n, double* Q, int64_t ldq, int64_t strideQ, double diag) {
  double* Qb = Q + blockIdx.y * strideQ;
  const int64_t total = static_cast<int64_t>(m) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    Qb[i + j * ldq] = (i == j) ? diag : 0.0;
  }
}

__global__ void add_diag_kernel(int n, double* A, int64_t lda, double d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    A[i + i * lda] += d;
}

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  // SplitMix64 finaliser (Steele, Lea, Flood 2014)
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__global__ void fill_random_kernel(int m, int n, double* X, int64_t ldx, uint64_t seed) {
  const int64_t total = static_cast<int64_t>(m) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    const uint64_t r = mix64(seed * 0x100000001B3ull + static_cast<uint64_t>(e));
    X[i + j * ldx] = 2.0 * (static_cast<double>(r >> 11) * (1.0 / 9007199254740992.0)) - 1.0;
  }
}

__global__ void trace_kernel(int n, const double* A, int64_t lda, double* out) {
  __shared__ double sh[TPB / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += A[i + i * lda];
  s = block_sum<TPB>(s, sh);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void gather_columns_kernel(int m, int n, const double* __restrict__ A, int64_t lda, const int* perm,
                                      double* B, int64_t ldb) {
  const int64_t total = static_cast<int64_t>(m) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    B[i + j * ldb] = A[i + static_cast<int64_t>(perm[j]) * lda];
  }
}

__global__ void get_diag_kernel(int n, const double* A, int64_t lda, double* d) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) d[i] = A[i + i * lda];
}

}  // namespace

cudaError_t fill_random(int m, int n, double* X, int64_t ldx, uint64_t seed, cudaStream_t st) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  fill_random_kernel<<<grid_for(static_cast<int64_t>(m) * n), TPB, 0, st>>>(m, n, X, ldx, seed);
  return cudaGetLastError();
}

cudaError_t trace(int n, const double* A, int64_t lda, double* out, cudaStream_t st) {
  trace_kernel<<<1, TPB, 0, st>>>(n, A, lda, out);
  return cudaGetLastError();
}

cudaError_t gather_columns(int m, int n, const double* A, int64_t lda, const int* perm, double* B, int64_t ldb,
                           cudaStream_t st) {
  if (m <= 0 || n <= 0) return cudaSuccess;
  gather_columns_kernel<<<grid_for(static_cast<int64_t>(m) * n), TPB, 0, st>>>(m, n, A, lda, perm, B, ldb);
  return cudaGetLastError();
}

cudaError_t get_diag(int n, const double* A, int64_t lda, double* d, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  get_diag_kernel<<<(n + TPB - 1) / TPB, TPB, 0, st>>>(n, A, lda, d);
  return cudaGetLastError();
}

cudaError_t scale_copy(int m, int n, double s, const double* src, int64_t lds, int64_t strideS, double* dst,
                       int64_t ldd, int64_t strideD, int batch, double diag_add, cudaStream_t st) {
  if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
  scale_copy_kernel<<<dim3(grid_for(static_cast<int64_t>(m) * n), batch), TPB, 0, st>>>(
      m, n, s, src, lds, strideS, dst, ldd, strideD, diag_add);
  return cudaGetLastError();
}

cudaError_t form_stack(int m, int mpad, int n, const double* X, int64_t ldx, double* W, int64_t ldw,
                       int64_t strideW, const double* s_vec, double s_scalar, int batch, cudaStream_t st,
                       int x_upper, int64_t strideX) {
  if (n <= 0 || batch <= 0) return cudaSuccess;
  if (mpad < m) return cudaErrorInvalidValue;
  form_stack_kernel<<<dim3(grid_for(static_cast<int64_t>(mpad + n) * n), batch), TPB, 0, st>>>(
      m, mpad, n, X, ldx, W, ldw, strideW, s_vec, s_scalar, x_upper, strideX);
  return cudaGetLastError();
}

cudaError_t shift_lower(int n, const double* G, int64_t ldg, double* W, int64_t ldw, int64_t strideW,
                        const double* c_vec, int batch, cudaStream_t st) {
  if (n <= 0 || batch <= 0) return cudaSuccess;
  shift_lower_kernel<<<dim3(grid_for(static_cast<int64_t>(n) * n), batch), TPB, 0, st>>>(n, G, ldg, W, ldw,
                                                                                         strideW, c_vec);
  return cudaGetLastError();
}

cudaError_t reduce_sum(const double* partial, int count, double* out, cudaStream_t st) {
  reduce_sum_kernel<<<1, TPB, 0, st>>>(partial, count, out);
  return cudaGetLastError();
}

cudaError_t frob2(int m, int n, const double* X, int64_t ldx, double* partial, double* out, cudaStream_t st) {
  const int blocks = std::min(grid_for(static_cast<int64_t>(m) * n), 1024);
  frob2_kernel<<<blocks, TPB, 0, st>>>(m, n, X, ldx, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return reduce_sum(partial, blocks, out, st);
}

cudaError_t norm1(int m, int n, const double* X, int64_t ldx, double* colsum, double* out, cudaStream_t st) {
  colsum_abs_kernel<<<std::min(n, 4096), TPB, 0, st>>>(m, n, X, ldx, colsum);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  max_kernel<<<1, TPB, 0, st>>>(colsum, n, out);
  return cudaGetLastError();
}

cudaError_t combine_update(int m, int n, double* X, int64_t ldx, const double* Z, int64_t ldz, int64_t strideZ,
                           int nz, double cx, double cz, const double* cz_vec, double* partial, double* err2,
                           cudaStream_t st) {
  const int blocks = std::min(grid_for(static_cast<int64_t>(m) * n), 1024);
  combine_kernel<<<blocks, TPB, 0, st>>>(m, n, X, ldx, Z, ldz, strideZ, nz, cx, cz, cz_vec, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return reduce_sum(partial, blocks, err2, st);
}

cudaError_t symmetrize(int n, double* B, int64_t ldb, cudaStream_t st) {
  symmetrize_kernel<<<grid_for(static_cast<int64_t>(n) * n), TPB, 0, st>>>(n, B, ldb);
  return cudaGetLastError();
}

cudaError_t transpose(int m, int n, const double* A, int64_t lda, double* B, int64_t ldb, cudaStream_t st) {
  dim3 grid((m + 31) / 32, (n + 31) / 32);
  transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(m, n, A, lda, B, ldb);
  return cudaGetLastError();
}

cudaError_t ns_prepare(int n, double* G, int64_t ldg, double* partial, double* err2, int write, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  const int blocks = static_cast<int>(std::min<int64_t>(grid_for(static_cast<int64_t>(n) * n), 1024));
  ns_prepare_kernel<<<blocks, TPB, 0, st>>>(n, G, ldg, write, partial);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  return reduce_sum(partial, blocks, err2, st);
}

cudaError_t copy_upper(int n, const double* A, int64_t lda, double scale, double* B, int64_t ldb, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  copy_upper_kernel<<<grid_for(static_cast<int64_t>(n) * n), TPB, 0, st>>>(n, A, lda, scale, B, ldb);
  return cudaGetLastError();
}

cudaError_t mirror_lower(int n, double* B, int64_t ldb, cudaStream_t st) {
  if (n <= 0) return cudaSuccess;
  mirror_lower_kernel<<<grid_for(static_cast<int64_t>(n) * n), TPB, 0, st>>>(n, B, ldb);
  return cudaGetLastError();
}

cudaError_t set_identity(int m, int n, double* Q, int64_t ldq, int64_t strideQ, int batch, double diag,
                         cudaStream_t st) {
  if (m <= 0 || n <= 0 || batch <= 0) return cudaSuccess;
  set_identity_kernel<<<dim3(grid_for(static_cast<int64_t>(m) * n), batch), TPB, 0, st>>>(m, n, Q, ldq,
                                                                                          strideQ, diag);
  return cudaGetLastError();
}

cudaError_t add_diag(int n, double* A, int64_t lda, double d, cudaStream_t st) {
  add_diag_kernel<<<std::max(1, (n + TPB - 1) / TPB), TPB, 0, st>>>(n, A, lda, d);
  return cudaGetLastError();
}

}  // namespace zolo
