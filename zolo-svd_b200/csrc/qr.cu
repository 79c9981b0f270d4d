// Householder panel factorisation for the blocked QR of the stacked matrix
// [X; sqrt(c) I] (mpdgeqrf.f:252-313 / PDGEQR2 semantics, LAPACK dlarfg and
// dlarft conventions) on one thread-block cluster per panel.
//
// The m x w panel (w <= 32) is split by rows over the CL CTAs of a cluster;
// each CTA keeps its rows in shared memory when they fit.  Inside a CTA the
// work is column-parallel: thread (c, g) owns column c of the rows
// r = g, g+8, g+16, ... of its chunk, so every phase is a short scalar loop
// over independent rows and the row sums are 3 warp shuffles.  Column k costs
// three CTA barriers and ONE cluster barrier:
//   * gather: every CTA sums all CTAs' partials (||x_below||^2 and
//     x_below . a_c) in the same fixed order, so all CTAs derive bit-identical
//     beta / tau / v^T A; the partials were pushed into every CTA's receive
//     slots (distributed shared memory stores) before the cluster barrier, so
//     the sum reads local shared memory and the remote latency overlaps the
//     barrier;
//   * update: columns c > k apply reflector k;
//   * scale + dots: column k is scaled into v_k and the partials of column
//     k+1 are formed and published (double-buffered by column parity).
// The compact-WY factor T (dlarft) is formed once, after the last column, from
// the cluster-wide V^T V.
#include "common.cuh"
#include "kernels.h"

#include <cooperative_groups.h>

#include <algorithm>

namespace cg = cooperative_groups;

namespace zolo {

namespace {

constexpr int QW = 32;   // max panel width
constexpr int QT = 256;  // threads per CTA: 32 columns x 8 row groups
constexpr int NG = 8;    // row groups
constexpr int UB = 8;    // rows per load batch
constexpr int UC = 16;   // columns per load batch in the update
constexpr int SLOT = 1 + QW;  // s0, d[QW]
constexpr int QCL = 16;       // largest cluster
constexpr size_t SMEM_CHUNK_CAP = 190 * 1024;

struct PanelArgs {
  int m, w, rows_per, rp_ld;  // rp_ld: leading dimension of the shared-memory chunk
  double* A;
  int64_t lda, strideA;
  int split;    // logical rows >= split live `gap` rows further down in A
  int64_t gap;
  double* tau;
  int64_t strideTau;
  double* T;
  int64_t strideT;
  double* V;
  int64_t ldv, strideV;
};

ZDEV double group_sum8(double v) {
  v += __shfl_xor_sync(0xffffffffu, v, 1);
  v += __shfl_xor_sync(0xffffffffu, v, 2);
  v += __shfl_xor_sync(0xffffffffu, v, 4);
  return v;
}

struct PanelShared {
  double recv[2][QCL][SLOT];  // partials of every CTA (by rank), double-buffered by column parity
  double rowkr[2][QW];        // the pivot row of the next column, from the CTA holding it
  double sum[SLOT];
  double rowk[QW];
  double colk[QW];
  double tauv[QW];
  double G[QW * QW];   // this CTA's partial V^T V (upper triangle)
  double Gs[QW * QW];  // rank 0: cluster sum of G
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
  const int tid = threadIdx.x, lane = tid & 31;
  const int col = (tid >> 5) * 4 + (lane >> 3);  // column owned by this thread
  const int grp = lane & 7;                      // row group: local rows grp, grp+8, ...
  const int rp = p.rp_ld;

  // physical row of A holding logical row r
  auto prow = [&](int r) -> int64_t { return r + (r >= p.split ? p.gap : 0); };
  auto at = [&](int rl, int c) -> double& {
    if (SMEM) return chunk[c * rp + rl];
    return A[prow(r0 + rl) + c * lda];
  };
  // first local row >= global row `from` that belongs to this thread's group
  auto first_row = [&](int from) {
    int rl = max(from - r0, 0);
    rl += (grp - rl % NG + NG) % NG;
    return rl;
  };
  // sum over this thread's rows (from rl0) of a(r, x) * a(r, col): batches of UB rows whose
  // loads are all issued first, four independent partial sums
  auto dot_rows = [&](int rl0, int x) {
    double s4[4] = {0.0, 0.0, 0.0, 0.0};
    for (int rl = rl0; rl < nloc; rl += NG * UB) {
      double xa[UB], xb[UB];
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        const int r = rl + u * NG;
        xa[u] = (r < nloc) ? at(r, x) : 0.0;
        xb[u] = (r < nloc) ? at(r, col) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < UB; ++u) s4[u & 3] += xa[u] * xb[u];
    }
    return (s4[0] + s4[1]) + (s4[2] + s4[3]);
  };

  if (SMEM) {
    const int tot = w * nloc;
    for (int e = tid; e < tot; e += QT) {
      const int c = e / nloc, rl = e - c * nloc;
      chunk[c * rp + rl] = A[prow(r0 + rl) + c * lda];
    }
  }
  __syncthreads();

  // partials into slot `slot` of receive buffer `bf` of every CTA of the cluster, the pivot
  // row entry c likewise (stores to distributed shared memory, visible after the barrier)
  auto publish = [&](int bf, int slot, double v) {
    for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(&S.recv[bf][rank][slot], q) = v;
  };
  auto publish_pivot = [&](int bf, int c, double v) {
    for (int q = 0; q < CL; ++q) *cluster.map_shared_rank(&S.rowkr[bf][c], q) = v;
  };

  // ---- partials of column 0 ----
  {
    double acc = 0.0, pv = 0.0;
    bool has_pv = false;
    if (col < w) {
      acc = dot_rows(first_row(1), 0);  // col 0: ||x_below||^2
      if (r0 == 0 && grp == 0 && nloc > 0) {  // pivot row 0
        pv = at(0, col);
        has_pv = true;
      }
    }
    acc = group_sum8(acc);
    if (grp == 0 && col < w) publish(0, col == 0 ? 0 : 1 + col, acc);
    if (has_pv) publish_pivot(0, col, pv);
  }
  cluster.sync();

  for (int k = 0; k < w; ++k) {
    const int buf = k & 1;
    // ---- gather: thread i < SLOT sums entry i over all CTAs in rank order (the same order
    // everywhere) from this CTA's receive slots ----
    if (tid < SLOT) {
      double s = 0.0;
      for (int q = 0; q < CL; ++q) s += S.recv[buf][q][tid];
      S.sum[tid] = s;
    } else if (tid < SLOT + w) {
      const int c = tid - SLOT;
      S.rowk[c] = S.rowkr[buf][c];
    }
    __syncthreads();

    // ---- reflector k (dlarfg), computed redundantly and identically by every thread ----
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

    // ---- update: a(r,c) -= tau * v_r * (v^T a_c) for c > k, rows r >= k ----
    // each thread owns whole rows and loads a batch of UC columns before storing any
    // (a store may alias the next loads of the same array, so batching is explicit)
    for (int rl = max(k - r0, 0) + tid; rl < nloc; rl += QT) {
      const double tv = tau * ((r0 + rl == k) ? 1.0 : at(rl, k) * scal);
      for (int c0 = k + 1; c0 < w; c0 += UC) {
        double xc[UC];
#pragma unroll
        for (int u = 0; u < UC; ++u)
          if (c0 + u < w) xc[u] = at(rl, c0 + u);
#pragma unroll
        for (int u = 0; u < UC; ++u)
          if (c0 + u < w) at(rl, c0 + u) = xc[u] - tv * S.colk[c0 + u];
      }
    }
    __syncthreads();

    // ---- scale column k into v_k (all threads); partials of column k+1 (column threads) ----
    const int nk = k + 1;
    for (int base = tid; base < nloc; base += QT * UB) {
      double x[UB];
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        const int rl = base + u * QT;
        if (rl < nloc && r0 + rl > k) x[u] = at(rl, k);
      }
#pragma unroll
      for (int u = 0; u < UB; ++u) {
        const int rl = base + u * QT;
        if (rl >= nloc) continue;
        const int r = r0 + rl;
        double v;
        if (r < k) {
          v = 0.0;
        } else if (r == k) {
          at(rl, k) = beta;
          v = 1.0;
        } else {
          v = x[u] * scal;
          at(rl, k) = v;
        }
        V[r + k * ldv] = v;
      }
    }
    double acc = 0.0, pv = 0.0;
    bool has_pv = false;
    if (nk < w && col >= nk && col < w) {
      acc = dot_rows(first_row(nk + 1), nk);
      const int lr = nk - r0;  // pivot row of column k+1, if this CTA holds it
      if (lr >= 0 && lr < nloc && grp == lr % NG) {
        pv = at(lr, col);
        has_pv = true;
      }
    }
    acc = group_sum8(acc);
    // the other buffer: no CTA reads it before every CTA has passed this column's barrier
    if (nk < w && grp == 0 && col >= nk && col < w) publish(buf ^ 1, col == nk ? 0 : 1 + col, acc);
    if (has_pv) publish_pivot(buf ^ 1, col, pv);
    cluster.sync();
  }

  // ---- V^T V of this CTA's rows on the FP64 tensor path: warp q takes rows q, q+8k8 ...
  // V(r,i) = a(r,i) below the diagonal, 1 on it, 0 above; the 32 x 32 partials of the 8
  // warps are summed through shared memory into G ----
  {
    const int warp = tid >> 5;
    const int gq = lane >> 2, tq = lane & 3;
    auto vval = [&](int rl, int i) -> double {
      const int r = r0 + rl;
      if (rl >= nloc || i >= w || r < i) return 0.0;
      return (r == i) ? 1.0 : at(rl, i);
    };
    double accg[2][4][4];
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int bb = 0; bb < 4; ++bb)
#pragma unroll
        for (int r = 0; r < 4; ++r) accg[a][bb][r] = 0.0;
    // k8 steps of rows: step s covers local rows 8s .. 8s+7; warp q does steps q, q+8, ...
    for (int st = warp; st * 8 < nloc; st += QT / 32) {
      const int rb = st * 8;
      double af[2][4], bf[4][2];
#pragma unroll
      for (int a = 0; a < 2; ++a) {  // A = V^T: rows i, k = local row
        const int i0 = a * 16 + gq;
        af[a][0] = vval(rb + tq, i0);
        af[a][1] = vval(rb + tq, i0 + 8);
        af[a][2] = vval(rb + tq + 4, i0);
        af[a][3] = vval(rb + tq + 4, i0 + 8);
      }
#pragma unroll
      for (int bb = 0; bb < 4; ++bb) {  // B = V: k = local row, n = j
        const int j0 = bb * 8 + gq;
        bf[bb][0] = vval(rb + tq, j0);
        bf[bb][1] = vval(rb + tq + 4, j0);
      }
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int bb = 0; bb < 4; ++bb) dmma_16x8x8(accg[a][bb], af[a], bf[bb]);
    }
    for (int e = tid; e < QW * QW; e += QT) S.G[e] = 0.0;
    __syncthreads();
    // warps add their partials one after another: a fixed summation order, so the
    // panel (and everything downstream) is bitwise reproducible run to run
    for (int wq = 0; wq < QT / 32; ++wq) {
      if (warp == wq) {
#pragma unroll
        for (int a = 0; a < 2; ++a)
#pragma unroll
          for (int bb = 0; bb < 4; ++bb) {
            const int i = a * 16 + gq, j = bb * 8 + 2 * tq;
            S.G[i + j * QW] += accg[a][bb][0];
            S.G[i + (j + 1) * QW] += accg[a][bb][1];
            S.G[i + 8 + j * QW] += accg[a][bb][2];
            S.G[i + 8 + (j + 1) * QW] += accg[a][bb][3];
          }
      }
      __syncthreads();
    }
  }
  if (SMEM) {
    const int tot = w * nloc;
    for (int e = tid; e < tot; e += QT) {
      const int c = e / nloc, rl = e - c * nloc;
      A[prow(r0 + rl) + c * lda] = chunk[c * rp + rl];
    }
  }
  cluster.sync();
  if (rank == 0) {
    // T(k,k) = tau_k, T(0:k,k) = -tau_k T(0:k,0:k) V(:,0:k)^T v_k  (dlarft, forward, columnwise)
    for (int e = tid; e < QW * QW; e += QT) {
      double gq[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) gq[q] = (q < CL) ? cluster.map_shared_rank(S.G, q)[e] : 0.0;
      double g = 0.0;
#pragma unroll
      for (int q = 0; q < 16; ++q) g += gq[q];
      S.Gs[e] = g;
      S.T[e] = 0.0;
    }
    __syncthreads();
    for (int k = 0; k < w; ++k) {
      const double tk = S.tauv[k];
      if (tid < k) {
        double tv = 0.0;
        for (int j = tid; j < k; ++j) tv += S.T[tid + j * QW] * S.Gs[j + k * QW];
        S.T[tid + k * QW] = -tk * tv;
      } else if (tid == k) {
        S.T[k + k * QW] = tk;
      }
      __syncthreads();
    }
    double* T = p.T + b * p.strideT;
    for (int e = tid; e < QW * QW; e += QT) T[e] = S.T[e];
  }
  cluster.sync();  // no CTA leaves while others may still read its shared memory
}

__global__ void extract_v_kernel(int m, int w, const double* __restrict__ A, int64_t lda, int64_t strideA,
                                 double* V, int64_t ldv, int64_t strideV, int split, int64_t gap) {
  const double* Ab = A + blockIdx.y * strideA;
  double* Vb = V + blockIdx.y * strideV;
  const int64_t total = static_cast<int64_t>(m) * w;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % m), j = static_cast<int>(e / m);
    double v = (i > j) ? Ab[i + (i >= split ? gap : 0) + j * lda] : (i == j ? 1.0 : 0.0);
    Vb[i + j * ldv] = v;
  }
}

// TB (jb x jb) <- the block diagonal of consecutive panels' T factors (QW x QW each, ld QW,
// QW*QW apart), zero elsewhere: the diagonal of the block reflector's T.
__global__ void block_t_init_kernel(int jb, const double* __restrict__ T, int64_t strideT, double* TB,
                                    int64_t ldtb, int64_t strideTB) {
  const double* Tb = T + blockIdx.y * strideT;
  double* Bb = TB + blockIdx.y * strideTB;
  const int total = jb * jb;
  for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < total; e += gridDim.x * blockDim.x) {
    const int i = e % jb, j = e / jb;
    const int q = i / QW;
    const double v = (q == j / QW && i <= j) ? Tb[q * QW * QW + (i % QW) + (j % QW) * QW] : 0.0;
    Bb[i + static_cast<int64_t>(j) * ldtb] = v;
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
  static std::atomic<int> attr_set[kMaxDevices];
  return once_per_device(attr_set, [] {
    const cudaError_t e = cudaFuncSetAttribute(qr_panel_kernel<SMEM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(shared_base() + SMEM_CHUNK_CAP + 64));
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(qr_panel_kernel<SMEM>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  });
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
  static std::atomic<int> cache[kMaxDevices];
  return per_device_value(cache, [] {
    int mc = 8;
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
    return mc;
  });
}

}  // namespace

int qr_panel_config(int m, int w) {
  const int maxcl = max_cluster();
  int cl = 1;
  while (cl < maxcl && (static_cast<size_t>(((m + cl - 1) / cl + 7) / 16 * 16 + 8) * w * 8 > SMEM_CHUNK_CAP ||
                        (m + cl - 1) / cl > 512))
    cl *= 2;
  const size_t chunk = static_cast<size_t>(((m + cl - 1) / cl + 7) / 16 * 16 + 8) * w * 8;
  return chunk <= SMEM_CHUNK_CAP ? cl : -cl;
}

cudaError_t qr_panel(int m, int w, double* A, int64_t lda, int64_t strideA, double* tau, int64_t strideTau,
                     double* T, int64_t strideT, double* Vexp, int64_t ldv, int64_t strideV, int batch,
                     cudaStream_t st, int split, int64_t gap) {
  if (m <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  if (w > QW || m < w || gap < 0 || (gap > 0 && split < w)) return cudaErrorInvalidValue;
  const int maxcl = max_cluster();
  // smallest cluster whose per-CTA row chunk fits in shared memory, with at most ~512 rows per CTA
  int cl = 1;
  while (cl < maxcl && (static_cast<size_t>(((m + cl - 1) / cl + 7) / 16 * 16 + 8) * w * 8 > SMEM_CHUNK_CAP ||
                        (m + cl - 1) / cl > 512))
    cl *= 2;
  PanelArgs pa;
  pa.m = m;
  pa.w = w;
  pa.rows_per = (m + cl - 1) / cl;
  pa.rp_ld = (pa.rows_per + 7) / 16 * 16 + 8;  // = 8 mod 16: conflict-free half-warp access
  pa.A = A;
  pa.lda = lda;
  pa.strideA = strideA;
  pa.split = (split > 0 && gap > 0) ? split : m;
  pa.gap = gap;
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
                      int64_t strideV, int batch, cudaStream_t st, int split, int64_t gap) {
  if (m <= 0 || w <= 0 || batch <= 0) return cudaSuccess;
  if (gap < 0 || (gap > 0 && split < w)) return cudaErrorInvalidValue;
  if (!(split > 0 && gap > 0)) split = m;
  int blocks = static_cast<int>(std::min<int64_t>((static_cast<int64_t>(m) * w + 255) / 256, 2048));
  extract_v_kernel<<<dim3(blocks, batch), 256, 0, st>>>(m, w, A, lda, strideA, V, ldv, strideV, split, gap);
  return cudaGetLastError();
}

cudaError_t block_t_init(int jb, const double* T, int64_t strideT, double* TB, int64_t ldtb, int64_t strideTB,
                         int batch, cudaStream_t st) {
  if (jb <= 0 || batch <= 0) return cudaSuccess;
  const int blocks = (jb * jb + 255) / 256;
  block_t_init_kernel<<<dim3(blocks, batch), 256, 0, st>>>(jb, T, strideT, TB, ldtb, strideTB);
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
