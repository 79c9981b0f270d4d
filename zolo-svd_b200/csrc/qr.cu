// Householder panel factorisation for the blocked QR of the stacked matrix
// [X; sqrt(c) I] (mpdgeqrf.f:252-313 / PDGEQR2 semantics, LAPACK dlarfg
// conventions) on one thread-block cluster per panel.
//
// The m x w panel (w <= 32) is split by rows over the CL CTAs of a cluster.
// Column k costs ONE pass over the CTA's rows and ONE cluster barrier:
//   * the pass applies reflector k-1 to the remaining columns and, on the
//     fly, accumulates the partial sums needed by reflector k
//     (||x_below||^2 and x_below . a_c for every later column c);
//   * the partials are block-reduced into this CTA's shared memory; after the
//     barrier every CTA sums all CTAs' partials through distributed shared
//     memory in the same fixed order, so all CTAs derive bit-identical
//     beta / tau / w = v^T A and no second barrier is needed (partials are
//     double-buffered by column parity).
// After the last column the CTAs reduce V^T V the same way and rank 0 forms
// the triangular factor T of I - V T V^T (dlarft, forward, columnwise).
#include "common.cuh"
#include "kernels.h"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace zolo {

namespace {

constexpr int QW = 32;    // max panel width
constexpr int QT = 256;   // threads per CTA
constexpr int NWARP = QT / 32;
constexpr int SLOT = 1 + QW + QW;  // s0, d[QW], rowk[QW]

struct PanelArgs {
  int m, w, rows_per;
  double* A;
  int64_t lda, strideA;
  double* tau;
  int64_t strideTau;
  double* T;
  int64_t strideT;
  double* V;
  int64_t ldv, strideV;
};

__device__ void block_reduce_vec(double (&acc)[QW + 1], double* red, double* out, int nvals) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < QW + 1; ++c) {
    if (c < nvals) {
      double v = warp_sum(acc[c]);
      if (lane == 0) red[warp * (QW + 1) + c] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < nvals) {
    double s = 0.0;
    for (int q = 0; q < NWARP; ++q) s += red[q * (QW + 1) + threadIdx.x];
    out[threadIdx.x] = s;
  }
  __syncthreads();
}

__global__ void __launch_bounds__(QT) qr_panel_kernel(PanelArgs p) {
  cg::cluster_group cluster = cg::this_cluster();
  __shared__ double part[2][SLOT];
  __shared__ double red[NWARP * (QW + 1)];
  __shared__ double vtv[QW * QW];
  __shared__ double colk[QW];  // scratch: wv[c]
  __shared__ double tvec[QW];
  __shared__ double gram[QW * QW];
  __shared__ double vt[32 * (QW + 1)];

  const int rank = static_cast<int>(cluster.block_rank());
  const int CL = static_cast<int>(cluster.num_blocks());
  const int b = blockIdx.y;
  const int m = p.m, w = p.w;
  double* A = p.A + b * p.strideA;
  double* V = p.V + b * p.strideV;
  const int64_t lda = p.lda, ldv = p.ldv;
  const int r0 = rank * p.rows_per;
  const int r1 = min(m, r0 + p.rows_per);
  const int tid = threadIdx.x;

  double acc[QW + 1];

  // ---- partials for column 0 ----
#pragma unroll
  for (int c = 0; c < QW + 1; ++c) acc[c] = 0.0;
  for (int r = r0 + tid; r < r1; r += QT) {
    const double x = A[r];
    if (r > 0) {
      acc[0] += x * x;
#pragma unroll
      for (int c = 1; c < QW; ++c)
        if (c < w) acc[1 + c] += x * A[r + c * lda];
    } else {
#pragma unroll
      for (int c = 0; c < QW; ++c)
        if (c < w) part[0][1 + QW + c] = A[c * lda];
    }
  }
  block_reduce_vec(acc, red, part[0], 1 + w);
  cluster.sync();

  for (int k = 0; k < w; ++k) {
    const int buf = k & 1;
    const int owner = k / p.rows_per;
    // gather partials (fixed order -> identical on every CTA)
    double s0 = 0.0;
    for (int q = 0; q < CL; ++q) s0 += cluster.map_shared_rank(&part[buf][0], q)[0];
    if (tid < w) {
      double d = 0.0;
      for (int q = 0; q < CL; ++q) d += cluster.map_shared_rank(&part[buf][0], q)[1 + tid];
      colk[tid] = d;  // x_below . a_c
      tvec[tid] = cluster.map_shared_rank(&part[buf][0], owner)[1 + QW + tid];  // row k
    }
    __syncthreads();
    const double alpha = tvec[k];
    double beta, tau, scal;
    if (s0 == 0.0) {
      tau = 0.0;
      beta = alpha;
      scal = 0.0;
    } else {
      beta = -copysign(sqrt(alpha * alpha + s0), alpha);
      tau = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    }
    __syncthreads();
    if (tid < w) colk[tid] = (tid > k) ? tvec[tid] + scal * colk[tid] : 0.0;  // w_c = v^T a_c
    __syncthreads();
    if (rank == 0 && tid == 0) p.tau[b * p.strideTau + k] = tau;

    // apply reflector k, accumulate partials for column k+1
#pragma unroll
    for (int c = 0; c < QW + 1; ++c) acc[c] = 0.0;
    const int nk = k + 1;
    for (int r = r0 + tid; r < r1; r += QT) {
      if (r < k) {
        V[r + k * ldv] = 0.0;
        continue;
      }
      if (r == k) {
        A[r + k * lda] = beta;
        V[r + k * ldv] = 1.0;
#pragma unroll
        for (int c = 0; c < QW; ++c)
          if (c > k && c < w) A[r + c * lda] -= tau * colk[c];
        continue;
      }
      const double v = A[r + k * lda] * scal;
      A[r + k * lda] = v;
      V[r + k * ldv] = v;
      double xn = 0.0;
#pragma unroll
      for (int c = 0; c < QW; ++c) {
        if (c > k && c < w) {
          const double a = A[r + c * lda] - tau * v * colk[c];
          A[r + c * lda] = a;
          if (c == nk) {
            xn = a;
            if (r > nk) acc[0] += a * a;
          } else if (r > nk) {
            acc[1 + c] += xn * a;
          }
        }
      }
      if (r == nk && nk < w) {
        // pivot row of the next column: publish its entries
        double* dst = &part[buf ^ 1][1 + QW];
#pragma unroll
        for (int c = 0; c < QW; ++c)
          if (c >= nk && c < w) dst[c] = A[r + c * lda];
      }
    }
    if (nk < w) block_reduce_vec(acc, red, part[buf ^ 1], 1 + w);
    cluster.sync();
  }

  // ---- T factor: reduce V^T V, rank 0 runs the dlarft recurrence ----
  {
    // partial V^T V over this CTA's rows, staged through shared memory in 32-row tiles
    double s[(QW * QW + QT - 1) / QT];
#pragma unroll
    for (int q = 0; q < (QW * QW + QT - 1) / QT; ++q) s[q] = 0.0;
    for (int rb = r0; rb < r1; rb += 32) {
      __syncthreads();
      for (int e = tid; e < 32 * QW; e += QT) {
        const int rr = e % 32, c = e / 32;
        const int r = rb + rr;
        vt[rr * (QW + 1) + c] = (r < r1 && c < w) ? V[r + c * ldv] : 0.0;
      }
      __syncthreads();
#pragma unroll
      for (int q = 0; q < (QW * QW + QT - 1) / QT; ++q) {
        const int e = tid + q * QT;
        const int i = e % QW, j = e / QW;
        if (i <= j && j < w) {
          double acc2 = 0.0;
#pragma unroll 8
          for (int rr = 0; rr < 32; ++rr) acc2 += vt[rr * (QW + 1) + i] * vt[rr * (QW + 1) + j];
          s[q] += acc2;
        }
      }
    }
#pragma unroll
    for (int q = 0; q < (QW * QW + QT - 1) / QT; ++q) vtv[tid + q * QT] = s[q];
  }
  cluster.sync();
  if (rank == 0) {
    for (int e = tid; e < w * w; e += QT) {
      const int i = e % w, j = e / w;
      double s = 0.0;
      if (i <= j)
        for (int q = 0; q < CL; ++q) s += cluster.map_shared_rank(vtv, q)[i + j * QW];
      gram[i + j * QW] = s;
    }
    __syncthreads();
    double* T = p.T + b * p.strideT;
    const double* tau = p.tau + b * p.strideTau;
    // T(k,k) = tau_k ; T(0:k,k) = -tau_k * T(0:k,0:k) * gram(0:k,k)
    for (int k = 0; k < w; ++k) {
      if (tid < k) {
        double s = 0.0;
        for (int j = tid; j < k; ++j) s += T[tid + j * QW] * gram[j + k * QW];
        tvec[tid] = -tau[k] * s;
      }
      __syncthreads();
      if (tid < QW) {
        double v;
        if (tid < k) v = tvec[tid];
        else if (tid == k) v = tau[k];
        else v = 0.0;
        T[tid + k * QW] = v;
      }
      __syncthreads();
    }
  }
  cluster.sync();  // keep every CTA's shared memory alive until rank 0 has read it
}

__global__ void extract_v_kernel(int m, int w, const double* __restrict__ A, int64_t lda, int64_t strideA,
                                 double* V, int64_t ldv, int64_t strideV) {
  const double* Ab = A + blockIdx.y * strideA;
  double* Vb = V + blockIdx.y * strideV;
  const int64_t total = static_cast<int64_t>(m) * w;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    double v = (i > j) ? Ab[i + j * lda] : (i == j ? 1.0 : 0.0);
    Vb[i + j * ldv] = v;
  }
}

// P(:,col) <- T^T P(:,col)  or  T P(:,col), T upper triangular w x w (ld QW)
__global__ void apply_t_kernel(int w, int n, const double* __restrict__ T, int64_t strideT, double* P,
                               int64_t ldp, int64_t strideP, int trans) {
  __shared__ double t[QW * QW];
  const double* Tb = T + blockIdx.y * strideT;
  double* Pb = P + blockIdx.y * strideP;
  for (int e = threadIdx.x; e < QW * QW; e += blockDim.x) t[e] = Tb[e];
  __syncthreads();
  for (int col = blockIdx.x * blockDim.x + threadIdx.x; col < n; col += gridDim.x * blockDim.x) {
    double x[QW];
#pragma unroll
    for (int i = 0; i < QW; ++i) x[i] = (i < w) ? Pb[i + col * ldp] : 0.0;
    for (int i = 0; i < w; ++i) {
      double s = 0.0;
      if (trans) {
        // (T^T x)_i = sum_{j<=i} T(j,i) x_j
#pragma unroll
        for (int j = 0; j < QW; ++j)
          if (j <= i) s += t[j + i * QW] * x[j];
      } else {
        // (T x)_i = sum_{i<=j<w} T(i,j) x_j
#pragma unroll
        for (int j = 0; j < QW; ++j)
          if (j >= i && j < w) s += t[i + j * QW] * x[j];
      }
      Pb[i + col * ldp] = s;
    }
  }
}

}  // namespace

cudaError_t qr_panel(int m, int w, double* A, int64_t lda, int64_t strideA, double* tau, int64_t strideTau,
                     double* T, int64_t strideT, double* Vexp, int64_t ldv, int64_t strideV, int batch,
                     cudaStream_t st) {
  if (m <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  if (w > QW || m < w) return cudaErrorInvalidValue;
  int cl = (m + 511) / 512;
  cl = std::max(1, std::min(cl, 8));
  PanelArgs pa;
  pa.m = m;
  pa.w = w;
  pa.rows_per = (m + cl - 1) / cl;
  pa.A = A;
  pa.lda = lda;
  pa.strideA = strideA;
  pa.tau = tau;
  pa.strideTau = strideTau;
  pa.T = T;
  pa.strideT = strideT;
  pa.V = Vexp;
  pa.ldv = ldv;
  pa.strideV = strideV;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, batch, 1);
  cfg.blockDim = dim3(QT, 1, 1);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = cl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, qr_panel_kernel, pa);
}

cudaError_t extract_v(int m, int w, const double* A, int64_t lda, int64_t strideA, double* V, int64_t ldv,
                      int64_t strideV, int batch, cudaStream_t st) {
  if (m <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  int blocks = static_cast<int>(std::min<int64_t>((static_cast<int64_t>(m) * w + 255) / 256, 2048));
  extract_v_kernel<<<dim3(blocks, batch), 256, 0, st>>>(m, w, A, lda, strideA, V, ldv, strideV);
  return cudaGetLastError();
}

cudaError_t apply_t(int w, int n, const double* T, int64_t strideT, double* P, int64_t ldp, int64_t strideP,
                    int trans, int batch, cudaStream_t st) {
  if (n <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  if (w > QW) return cudaErrorInvalidValue;
  int blocks = std::max(1, std::min((n + 127) / 128, 1024));
  apply_t_kernel<<<dim3(blocks, batch), 128, 0, st>>>(w, n, T, strideT, P, ldp, strideP, trans);
  return cudaGetLastError();
}

}  // namespace zolo
