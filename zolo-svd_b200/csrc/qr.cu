// Householder panel factorisation for the blocked QR of the stacked matrix
// [X; sqrt(c) I] (mpdgeqrf.f:252-313 / PDGEQR2 semantics, LAPACK dlarfg and
// dlarft conventions) on one thread-block cluster per panel.
//
// The m x w panel (w <= 32) is split by rows over the CL CTAs of a cluster;
// each CTA keeps its rows in shared memory when they fit.  Column k costs ONE
// pass over the CTA's rows and ONE cluster barrier:
//   * the pass applies reflector k to the remaining columns and accumulates,
//     in the same sweep, everything the next step needs: ||x_below||^2 and
//     x_below . a_c of column k+1, and the Gram column V(:,0:k)^T v_k that
//     the compact-WY factor T needs;
//   * the 65 partial sums are block-reduced (warp reduce-scatter) into this
//     CTA's shared memory; after the barrier every CTA gathers all CTAs'
//     partials through distributed shared memory and sums them in the same
//     fixed order, so all CTAs derive bit-identical beta / tau / v^T A and the
//     same T column; partials are double-buffered by column parity.
#include "common.cuh"
#include "kernels.h"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace zolo {

namespace {

constexpr int QW = 32;   // max panel width
constexpr int QT = 256;  // threads per CTA
constexpr int NWARP = QT / 32;
constexpr int SLOT = 1 + 2 * QW;  // s0, d[QW], g[QW]
constexpr int ROWK = SLOT;        // pivot row of the next column follows the partials
constexpr int SLOT_ALL = SLOT + QW;
constexpr int MAX_CL = 16;
constexpr size_t SMEM_CHUNK_CAP = 190 * 1024;

struct PanelArgs {
  int m, w, rows_per, rp_ld;  // rp_ld: leading dimension of the shared-memory chunk
  double* A;
  int64_t lda, strideA;
  double* tau;
  int64_t strideTau;
  double* T;
  int64_t strideT;
  double* V;
  int64_t ldv, strideV;
};

// after the call lane l holds in v[0] the warp sum of value index l
ZDEV void warp_reduce_scatter32(double (&v)[QW], int lane) {
#pragma unroll
  for (int o = 16; o >= 1; o >>= 1) {
    const bool up = lane & o;
#pragma unroll
    for (int i = 0; i < o; ++i) {
      const double send = up ? v[i] : v[i + o];
      const double keep = up ? v[i + o] : v[i];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, o);
    }
  }
}

struct PanelShared {
  double part[2][SLOT_ALL];
  double red[NWARP][SLOT];
  double gat[MAX_CL][SLOT];
  double sum[SLOT];
  double rowk[QW];
  double colk[QW];
  double tauv[QW];
  double T[QW * QW];
};

template <bool SMEM>
__global__ void __launch_bounds__(QT) qr_panel_kernel(PanelArgs p) {
  cg::cluster_group cluster = cg::this_cluster();
  extern __shared__ __align__(16) unsigned char smem_raw[];
  PanelShared& S = *reinterpret_cast<PanelShared*>(smem_raw);
  double* chunk = reinterpret_cast<double*>(smem_raw + ((sizeof(PanelShared) + 15) / 16) * 16);

  const int rank = static_cast<int>(cluster.block_rank());
  const int CL = static_cast<int>(cluster.num_blocks());
  const int b = blockIdx.y;
  const int m = p.m, w = p.w;
  double* A = p.A + b * p.strideA;
  double* V = p.V + b * p.strideV;
  const int64_t lda = p.lda, ldv = p.ldv;
  const int r0 = rank * p.rows_per;
  const int r1 = min(m, r0 + p.rows_per);
  const int nloc = max(r1 - r0, 0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int rp = p.rp_ld;

  // element (local row rl of this CTA, column c) of the panel
  auto at = [&](int rl, int c) -> double& {
    if (SMEM) return chunk[c * rp + rl];
    return A[(r0 + rl) + c * lda];
  };

  if (SMEM) {
    for (int c = 0; c < w; ++c)
      for (int rl = tid; rl < nloc; rl += QT) chunk[c * rp + rl] = A[(r0 + rl) + c * lda];
  }
  for (int e = tid; e < QW * QW; e += QT) S.T[e] = 0.0;

  double acc_s0;
  double accd[QW], accg[QW];

  auto reduce_and_publish = [&](double* out) {
    const double s0w = warp_sum(acc_s0);
    warp_reduce_scatter32(accd, lane);
    warp_reduce_scatter32(accg, lane);
    if (lane == 0) S.red[warp][0] = s0w;
    S.red[warp][1 + lane] = accd[0];
    S.red[warp][1 + QW + lane] = accg[0];
    __syncthreads();
    if (tid < SLOT) {
      double s = 0.0;
#pragma unroll
      for (int q = 0; q < NWARP; ++q) s += S.red[q][tid];
      out[tid] = s;
    }
  };

  // ---- partials for column 0 ----
  acc_s0 = 0.0;
#pragma unroll
  for (int c = 0; c < QW; ++c) accd[c] = accg[c] = 0.0;
  __syncthreads();
  for (int rl = tid; rl < nloc; rl += QT) {
    const int r = r0 + rl;
    const double x = at(rl, 0);
    if (r > 0) {
      acc_s0 += x * x;
#pragma unroll
      for (int c = 1; c < QW; ++c)
        if (c < w) accd[c] += x * at(rl, c);
    } else {
#pragma unroll
      for (int c = 0; c < QW; ++c)
        if (c < w) S.part[0][ROWK + c] = at(rl, c);
    }
  }
  reduce_and_publish(S.part[0]);
  cluster.sync();

  for (int k = 0; k <= w; ++k) {
    const int buf = k & 1;
    // ---- gather the partials of all CTAs (one remote load per element) ----
    for (int e = tid; e < CL * SLOT; e += QT) {
      const int q = e / SLOT, i = e - q * SLOT;
      S.gat[q][i] = cluster.map_shared_rank(&S.part[buf][0], q)[i];
    }
    if (k < w) {
      const int owner = k / p.rows_per;
      if (tid < w) S.rowk[tid] = cluster.map_shared_rank(&S.part[buf][0], owner)[ROWK + tid];
    }
    __syncthreads();
    if (tid < SLOT) {
      double s = 0.0;
      for (int q = 0; q < CL; ++q) s += S.gat[q][tid];
      S.sum[tid] = s;
    }
    __syncthreads();
    // ---- T column k-1 from the Gram column g = V(:,0:k-1)^T v_{k-1} (dlarft) ----
    if (k > 0) {
      const int kc = k - 1;
      const double tk = S.tauv[kc];
      double tv = 0.0;
      if (tid < kc) {
        for (int j = tid; j < kc; ++j) tv += S.T[tid + j * QW] * S.sum[1 + QW + j];
        tv = -tk * tv;
      }
      __syncthreads();
      if (tid < kc) S.T[tid + kc * QW] = tv;
      if (tid == 0) S.T[kc + kc * QW] = tk;
      __syncthreads();
    }
    if (k == w) break;

    // ---- reflector k (dlarfg) ----
    const double s0 = S.sum[0];
    const double alpha = S.rowk[k];
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
    if (tid < w) S.colk[tid] = (tid > k) ? S.rowk[tid] + scal * S.sum[1 + tid] : 0.0;  // v^T a_c
    if (tid == 0) {
      S.tauv[k] = tau;
      if (rank == 0) p.tau[b * p.strideTau + k] = tau;
    }
    __syncthreads();

    // ---- apply reflector k; accumulate partials of column k+1 and the Gram column of v_k ----
    acc_s0 = 0.0;
#pragma unroll
    for (int c = 0; c < QW; ++c) accd[c] = accg[c] = 0.0;
    const int nk = k + 1;
    for (int rl = tid; rl < nloc; rl += QT) {
      const int r = r0 + rl;
      if (r < k) {
        V[r + k * ldv] = 0.0;
        continue;
      }
      if (r == k) {
        at(rl, k) = beta;
        V[r + k * ldv] = 1.0;
#pragma unroll
        for (int c = 0; c < QW; ++c) {
          if (c > k && c < w) at(rl, c) -= tau * S.colk[c];
          if (c < k) accg[c] += at(rl, c);  // V(k, c) * 1
        }
        if (nk < w) {
#pragma unroll
          for (int c = 0; c < QW; ++c)
            if (c >= nk && c < w) S.part[buf ^ 1][ROWK + c] = at(rl, c);
        }
        continue;
      }
      const double v = at(rl, k) * scal;
      at(rl, k) = v;
      V[r + k * ldv] = v;
      double xn = 0.0;
#pragma unroll
      for (int c = 0; c < QW; ++c) {
        if (c < k) {
          accg[c] += at(rl, c) * v;
        } else if (c > k && c < w) {
          const double a = at(rl, c) - tau * v * S.colk[c];
          at(rl, c) = a;
          if (c == nk) {
            xn = a;
            if (r > nk) acc_s0 += a * a;
          } else if (r > nk) {
            accd[c] += xn * a;
          }
        }
      }
      if (r == nk && nk < w) {
#pragma unroll
        for (int c = 0; c < QW; ++c)
          if (c >= nk && c < w) S.part[buf ^ 1][ROWK + c] = at(rl, c);
      }
    }
    reduce_and_publish(S.part[buf ^ 1]);
    cluster.sync();
  }

  if (SMEM) {
    for (int c = 0; c < w; ++c)
      for (int rl = tid; rl < nloc; rl += QT) A[(r0 + rl) + c * lda] = chunk[c * rp + rl];
  }
  if (rank == 0) {
    double* T = p.T + b * p.strideT;
    for (int e = tid; e < QW * QW; e += QT) T[e] = S.T[e];
  }
  cluster.sync();  // no CTA leaves while others may still read its shared memory
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

constexpr size_t shared_base() { return ((sizeof(PanelShared) + 15) / 16) * 16; }

template <bool SMEM>
cudaError_t set_attrs() {
  static cudaError_t done = cudaErrorNotReady;
  if (done == cudaErrorNotReady) {
    done = cudaFuncSetAttribute(qr_panel_kernel<SMEM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                static_cast<int>(shared_base() + SMEM_CHUNK_CAP + 64));
    if (done == cudaSuccess)
      done = cudaFuncSetAttribute(qr_panel_kernel<SMEM>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  }
  return done;
}

template <bool SMEM>
cudaError_t launch_panel(const PanelArgs& pa, int cl, int batch, size_t smem, cudaStream_t st) {
  cudaError_t e = set_attrs<SMEM>();
  if (e != cudaSuccess) return e;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(cl, batch, 1);
  cfg.blockDim = dim3(QT, 1, 1);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr_l[1];
  attr_l[0].id = cudaLaunchAttributeClusterDimension;
  attr_l[0].val.clusterDim.x = cl;
  attr_l[0].val.clusterDim.y = 1;
  attr_l[0].val.clusterDim.z = 1;
  cfg.attrs = attr_l;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, qr_panel_kernel<SMEM>, pa);
}

// 16-CTA clusters are non-portable: use them only if the device can place one
// with the largest shared-memory footprint; otherwise the portable 8.
int max_cluster() {
  static int mc = 0;
  if (!mc) {
    mc = 8;
    if (set_attrs<true>() == cudaSuccess) {
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(16, 1, 1);
      cfg.blockDim = dim3(QT, 1, 1);
      cfg.dynamicSmemBytes = shared_base() + SMEM_CHUNK_CAP;
      cudaLaunchAttribute a[1];
      a[0].id = cudaLaunchAttributeClusterDimension;
      a[0].val.clusterDim.x = 16;
      a[0].val.clusterDim.y = 1;
      a[0].val.clusterDim.z = 1;
      cfg.attrs = a;
      cfg.numAttrs = 1;
      int n = 0;
      if (cudaOccupancyMaxActiveClusters(&n, qr_panel_kernel<true>, &cfg) == cudaSuccess && n > 0) mc = 16;
    }
    cudaGetLastError();
  }
  return mc;
}

}  // namespace

cudaError_t qr_panel(int m, int w, double* A, int64_t lda, int64_t strideA, double* tau, int64_t strideTau,
                     double* T, int64_t strideT, double* Vexp, int64_t ldv, int64_t strideV, int batch,
                     cudaStream_t st) {
  if (m <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  if (w > QW || m < w) return cudaErrorInvalidValue;
  const int maxcl = max_cluster();
  // smallest cluster whose per-CTA row chunk fits in shared memory, with at most ~512 rows per CTA
  int cl = 1;
  while (cl < maxcl && (static_cast<size_t>(((m + cl - 1) / cl) | 1) * w * 8 > SMEM_CHUNK_CAP ||
                        (m + cl - 1) / cl > 512))
    cl *= 2;
  PanelArgs pa;
  pa.m = m;
  pa.w = w;
  pa.rows_per = (m + cl - 1) / cl;
  pa.rp_ld = pa.rows_per | 1;  // odd stride
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
  const size_t chunk = static_cast<size_t>(pa.rp_ld) * w * 8;
  if (chunk <= SMEM_CHUNK_CAP) return launch_panel<true>(pa, cl, batch, shared_base() + chunk, st);
  return launch_panel<false>(pa, cl, batch, shared_base(), st);
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
