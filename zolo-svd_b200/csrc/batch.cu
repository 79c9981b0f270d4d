// Kernels of the batched polar decomposition (many matrices of different sizes,
// grouped into buckets of one padded size; the driver is qdwh_batch in polar.cpp).  Every kernel takes a
// batch of equally shaped, equally strided matrices (blockIdx.y = member) and
// per-member scalars in device arrays.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace zolo {

namespace {

constexpr int TPB = 256;

int blocks_for(int64_t work, int cap = 1024) {
  int64_t b = (work + TPB - 1) / TPB;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return static_cast<int>(b);
}

template <int NT>
__device__ double block_sum_b(double v, double* sh) {
  v = warp_sum(v);
  if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < NT / 32; ++w) s += sh[w];
  __syncthreads();
  return s;
}

// A'(b) = [[A_b, 0], [0, tau_b I], [0, 0]]  (MB x NB, ld ldp, stride sp)
__global__ void pack_kernel(const BatchMember* mem, int MB, int NB, double* P, int64_t ldp, int64_t sp) {
  const BatchMember d = mem[blockIdx.y];
  double* Pb = P + blockIdx.y * sp;
  const int64_t total = static_cast<int64_t>(MB) * NB;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % MB), j = static_cast<int>(e / MB);
    double v;
    if (j < d.n) v = (i < d.m) ? d.A[i + static_cast<int64_t>(j) * d.lda] : 0.0;
    else v = (i == d.m + (j - d.n)) ? d.tau : 0.0;
    Pb[i + static_cast<int64_t>(j) * ldp] = v;
  }
}

// Q_b = Q'(b)[0:m, 0:n], H_b = H'(b)[0:n, 0:n]
__global__ void unpack_kernel(const BatchMember* mem, const double* Q, int64_t ldq, int64_t sq, const double* H,
                              int64_t ldh, int64_t sh) {
  const BatchMember d = mem[blockIdx.y];
  const double* Qb = Q + blockIdx.y * sq;
  const double* Hb = H ? H + blockIdx.y * sh : nullptr;
  const int64_t tq = static_cast<int64_t>(d.m) * d.n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < tq;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % d.m), j = static_cast<int>(e / d.m);
    d.Q[i + static_cast<int64_t>(j) * d.ldq] = Qb[i + static_cast<int64_t>(j) * ldq];
  }
  if (Hb && d.H) {
    const int64_t th = static_cast<int64_t>(d.n) * d.n;
    for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < th;
         e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int i = static_cast<int>(e % d.n), j = static_cast<int>(e / d.n);
      d.H[i + static_cast<int64_t>(j) * d.ldh] = Hb[i + static_cast<int64_t>(j) * ldh];
    }
  }
}

// partial[b * nb + block] = sum over this block's share of member b of f(x)
__global__ void frob2_batch_kernel(int m, int n, const double* X, int64_t ldx, int64_t sx, double* partial) {
  __shared__ double sh[TPB / 32];
  const double* Xb = X + blockIdx.y * sx;
  const int64_t total = static_cast<int64_t>(m) * n;
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    const double x = Xb[i + static_cast<int64_t>(j) * ldx];
    s += x * x;
  }
  s = block_sum_b<TPB>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// out[b] = sum of partial[b * nb .. b * nb + nb) in a fixed order
__global__ void reduce_rows_kernel(const double* partial, int nb, double* out) {
  __shared__ double sh[TPB / 32];
  double s = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) s += partial[blockIdx.x * nb + i];
  s = block_sum_b<TPB>(s, sh);
  if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// out[b] = max_j sum_i |X_b(i, j)|  (one CTA per member, a warp per column)
__global__ void norm1_batch_kernel(int m, int n, const double* X, int64_t ldx, int64_t sx, double* out) {
  __shared__ double sh[TPB / 32];
  const double* Xb = X + blockIdx.x * sx;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double best = 0.0;
  for (int j = warp; j < n; j += TPB / 32) {
    double s = 0.0;
    for (int i = lane; i < m; i += 32) s += fabs(Xb[i + static_cast<int64_t>(j) * ldx]);
    s = warp_sum(s);
    best = fmax(best, s);
  }
  if (lane == 0) sh[warp] = best;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < TPB / 32; ++w) b = fmax(b, sh[w]);
    out[blockIdx.x] = b;
  }
}

// X_b <- s_b * X_b
__global__ void scale_batch_kernel(int m, int n, double* X, int64_t ldx, int64_t sx, const double* s) {
  double* Xb = X + blockIdx.y * sx;
  const double f = s[blockIdx.y];
  const int64_t total = static_cast<int64_t>(m) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    Xb[i + static_cast<int64_t>(j) * ldx] *= f;
  }
}

// X_b <- cx_b X_b + cz_b Z_b, partial[b * nb + block] = sum (X_new - X_old)^2
__global__ void combine_batch_kernel(int m, int n, double* X, int64_t ldx, int64_t sx, const double* Z, int64_t ldz,
                                     int64_t sz, const double* cx, const double* cz, double* partial) {
  __shared__ double sh[TPB / 32];
  double* Xb = X + blockIdx.y * sx;
  const double* Zb = Z + blockIdx.y * sz;
  const double a = cx[blockIdx.y], c = cz[blockIdx.y];
  const int64_t total = static_cast<int64_t>(m) * n;
  double s = 0.0;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    const double x = Xb[i + static_cast<int64_t>(j) * ldx];
    const double xn = (c == 0.0) ? x : a * x + c * Zb[i + static_cast<int64_t>(j) * ldz];
    const double d = xn - x;
    s += d * d;
    Xb[i + static_cast<int64_t>(j) * ldx] = xn;
  }
  s = block_sum_b<TPB>(s, sh);
  if (threadIdx.x == 0) partial[blockIdx.y * gridDim.x + blockIdx.x] = s;
}

// A member whose step in this row is conditional (cond[b] != 0) takes it only when the previous
// step's error sqrt(err2_prev[b]) is above tol; otherwise its coefficients become neutral
// (Cholesky form: c = 0, so that the shifted Gram is I; QR form: scale 1; cx = 1, cz = 0,
// which leaves X_b unchanged and its error 0).
__global__ void gate_batch_kernel(int batch, const double* err2_prev, const double* cond, double* row, int qr,
                                  double tol) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  if (cond[b] != 0.0 && !(sqrt(err2_prev[b]) > tol)) {
    row[b] = qr ? 1.0 : 0.0;
    row[batch + b] = 1.0;
    row[2 * batch + b] = 0.0;
  }
}

// G_b += d I
__global__ void add_diag_batch_kernel(int n, double* G, int64_t ldg, int64_t sg, double d) {
  double* Gb = G + blockIdx.y * sg;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    Gb[i + static_cast<int64_t>(i) * ldg] += d;
}

// B_b <- (B_b + B_b^T)/2
__global__ void symmetrize_batch_kernel(int n, double* B, int64_t ldb, int64_t sb) {
  double* Bb = B + blockIdx.y * sb;
  const int64_t total = static_cast<int64_t>(n) * n;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % n), j = static_cast<int>(e / n);
    if (i <= j) continue;
    const double x = Bb[i + static_cast<int64_t>(j) * ldb], y = Bb[j + static_cast<int64_t>(i) * ldb];
    const double h = 0.5 * y + 0.5 * x;
    Bb[i + static_cast<int64_t>(j) * ldb] = h;
    Bb[j + static_cast<int64_t>(i) * ldb] = h;
  }
}

// B_b = A_b^T  (A m x n)
__global__ void transpose_batch_kernel(int m, int n, const double* A, int64_t lda, int64_t sa, double* B,
                                       int64_t ldb, int64_t sb) {
  __shared__ double tile[32][33];
  const double* Ab = A + blockIdx.z * sa;
  double* Bb = B + blockIdx.z * sb;
  const int i0 = blockIdx.x * 32, j0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int i = i0 + threadIdx.x, j = j0 + r;
    if (i < m && j < n) tile[r][threadIdx.x] = Ab[i + static_cast<int64_t>(j) * lda];
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    const int j = j0 + threadIdx.x, i = i0 + r;
    if (i < m && j < n) Bb[j + static_cast<int64_t>(i) * ldb] = tile[threadIdx.x][r];
  }
}

}  // namespace

cudaError_t batch_pack(const BatchMember* d_mem, int count, int MB, int NB, double* P, int64_t ldp, int64_t sp,
                       cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  pack_kernel<<<dim3(blocks_for(static_cast<int64_t>(MB) * NB, 256), count), TPB, 0, st>>>(d_mem, MB, NB, P, ldp,
                                                                                          sp);
  return cudaGetLastError();
}

cudaError_t batch_unpack(const BatchMember* d_mem, int count, int MB, int NB, const double* Q, int64_t ldq,
                         int64_t sq, const double* H, int64_t ldh, int64_t sh, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  unpack_kernel<<<dim3(blocks_for(static_cast<int64_t>(MB) * NB, 256), count), TPB, 0, st>>>(d_mem, Q, ldq, sq, H,
                                                                                            ldh, sh);
  return cudaGetLastError();
}

cudaError_t batch_frob2(int m, int n, const double* X, int64_t ldx, int64_t sx, int batch, double* partial,
                        int partial_cap, double* out, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  int nb = blocks_for(static_cast<int64_t>(m) * n, 64);
  if (static_cast<int64_t>(nb) * batch > partial_cap) nb = std::max(1, partial_cap / batch);
  frob2_batch_kernel<<<dim3(nb, batch), TPB, 0, st>>>(m, n, X, ldx, sx, partial);
  reduce_rows_kernel<<<batch, TPB, 0, st>>>(partial, nb, out);
  return cudaGetLastError();
}

cudaError_t batch_norm1(int m, int n, const double* X, int64_t ldx, int64_t sx, int batch, double* out,
                        cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  norm1_batch_kernel<<<batch, TPB, 0, st>>>(m, n, X, ldx, sx, out);
  return cudaGetLastError();
}

cudaError_t batch_scale(int m, int n, double* X, int64_t ldx, int64_t sx, int batch, const double* s,
                        cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  scale_batch_kernel<<<dim3(blocks_for(static_cast<int64_t>(m) * n, 128), batch), TPB, 0, st>>>(m, n, X, ldx, sx, s);
  return cudaGetLastError();
}

cudaError_t batch_combine(int m, int n, double* X, int64_t ldx, int64_t sx, const double* Z, int64_t ldz, int64_t sz,
                          int batch, const double* cx, const double* cz, double* partial, int partial_cap,
                          double* err2, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  int nb = blocks_for(static_cast<int64_t>(m) * n, 64);
  if (static_cast<int64_t>(nb) * batch > partial_cap) nb = std::max(1, partial_cap / batch);
  combine_batch_kernel<<<dim3(nb, batch), TPB, 0, st>>>(m, n, X, ldx, sx, Z, ldz, sz, cx, cz, partial);
  reduce_rows_kernel<<<batch, TPB, 0, st>>>(partial, nb, err2);
  return cudaGetLastError();
}

cudaError_t batch_gate(int batch, const double* err2_prev, const double* cond, double* row, int qr, double tol,
                       cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  gate_batch_kernel<<<(batch + TPB - 1) / TPB, TPB, 0, st>>>(batch, err2_prev, cond, row, qr, tol);
  return cudaGetLastError();
}

cudaError_t batch_add_diag(int n, double* G, int64_t ldg, int64_t sg, int batch, double d, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  add_diag_batch_kernel<<<dim3(blocks_for(n, 8), batch), TPB, 0, st>>>(n, G, ldg, sg, d);
  return cudaGetLastError();
}

cudaError_t batch_symmetrize(int n, double* B, int64_t ldb, int64_t sb, int batch, cudaStream_t st) {
  if (batch <= 0) return cudaSuccess;
  symmetrize_batch_kernel<<<dim3(blocks_for(static_cast<int64_t>(n) * n, 128), batch), TPB, 0, st>>>(n, B, ldb, sb);
  return cudaGetLastError();
}

cudaError_t batch_transpose(int m, int n, const double* A, int64_t lda, int64_t sa, double* B, int64_t ldb,
                            int64_t sb, int batch, cudaStream_t st) {
  if (batch <= 0 || m <= 0 || n <= 0) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
  dim3 grid((m + 31) / 32, (n + 31) / 32, batch);
  transpose_batch_kernel<<<grid, dim3(32, 8), 0, st>>>(m, n, A, lda, sa, B, ldb, sb);
  return cudaGetLastError();
}

}  // namespace zolo
