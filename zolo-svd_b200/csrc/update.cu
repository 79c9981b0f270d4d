// Streaming rank-k update C = beta*C + alpha*A*B for K <= 32 (FP64, DMMA).
//
// This is the trailing-matrix update of the blocked Householder QR and of the
// explicit-Q accumulation (W -= V P with K = the panel width): 4 flops per byte
// at K = 32, just below the FP64-DMMA ridge (~5.4 flop/byte), so the tensor work
// (~1.9k cycles per tile) and the HBM stream must overlap.  CTAs (two per SM,
// 8 warps each) walk contiguous ranges of at most 8 tiles of 128 x 32 of C.  The C
// tile and the K x 32 block of B of the next tile are in flight through shared
// memory (cp.async, zero-filled outside the matrix) while the current tile is
// computed, and the other CTA on the SM fills the gaps; the A row block
// (128 x K) lives in registers as DMMA fragments and is reloaded only when the
// row block changes.  Each warp owns 16 rows x 32 columns of the tile.  With
// 16-byte alignment the results go back through the stage as 512-byte column
// runs per warp.  Measured at 8192^2, K = 32: 0.28 ms (3.9 TB/s of algorithmic
// bytes, 15.6 TF/s); one CTA per SM with four stages ran 0.35 ms, and a
// warp-specialised bulk-copy (cp.async.bulk + mbarrier) form 0.37-0.41 ms.
#include "common.cuh"
#include "kernels.h"

namespace zolo {

namespace {

constexpr int UM = 128;         // tile rows
constexpr int UN = 32;          // tile columns
constexpr int UK = 32;          // max K
constexpr int UT = 256;         // threads (8 warps x 16 rows)
constexpr int CSTAGES = 2;      // two CTAs per SM, two stages each
constexpr int LDC_S = UM + 2;   // = 2 mod 8: conflict-free C fragment reads
constexpr int LDB_S = UK + 4;   // = 4 mod 16: conflict-free B fragment reads
constexpr int C_STAGE = UN * LDC_S;
constexpr int B_STAGE = UN * LDB_S;
constexpr int STAGE = C_STAGE + B_STAGE;

struct UpdParams {
  int M, N, K;
  const double* A;
  int64_t lda, strideA;
  const double* B;
  int64_t ldb, strideB;
  double* C;
  int64_t ldc, strideC;
  double alpha, beta;
  int row_blocks, col_tiles;
  int64_t total;  // batch * row_blocks * col_tiles
};

// V16: C and B are 16-byte aligned with even leading dimensions and strides, so
// element pairs (rows r, r+1 with r even) move as one 16-byte cp.async (the last
// pair of an odd extent moves 8 bytes and zero-fills the rest); otherwise 8-byte copies.
template <bool V16>
__global__ void __launch_bounds__(UT, 2) rank_update_kernel(UpdParams p) {
  extern __shared__ __align__(16) double sm[];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int64_t per_batch = static_cast<int64_t>(p.row_blocks) * p.col_tiles;
  const int64_t t0 = p.total * blockIdx.x / gridDim.x;
  const int64_t t1 = p.total * (blockIdx.x + 1) / gridDim.x;
  const bool load_c = p.beta != 0.0;

  auto decode = [&](int64_t tau, int& b, int& rb, int& ct) {
    b = static_cast<int>(tau / per_batch);
    const int64_t r = tau - b * per_batch;
    rb = static_cast<int>(r / p.col_tiles);
    ct = static_cast<int>(r - static_cast<int64_t>(rb) * p.col_tiles);
  };
  // issue the copies of tile tau into stage s (C tile, if used, and the K x 32 block of B)
  auto issue = [&](int64_t tau, int s) {
    int b, rb, ct;
    decode(tau, b, rb, ct);
    double* cs = sm + s * STAGE;
    double* bs = cs + C_STAGE;
    const int r0 = rb * UM, c0 = ct * UN;
    const double* Bb = p.B + b * p.strideB;
    if (V16) {
      if (load_c) {
        const double* Cb = p.C + b * p.strideC;
        for (int e = tid; e < UM * UN / 2; e += UT) {
          const int r = (e & (UM / 2 - 1)) * 2, c = e >> 6;
          const int rows = (c0 + c < p.N) ? min(max(p.M - (r0 + r), 0), 2) : 0;
          const double* src = rows ? Cb + (r0 + r) + static_cast<int64_t>(c0 + c) * p.ldc : Cb;
          cp_async16(cs + r + c * LDC_S, src, rows * 8);
        }
      }
      for (int e = tid; e < UK * UN / 2; e += UT) {
        const int k = (e & (UK / 2 - 1)) * 2, c = e >> 4;
        const int rows = (c0 + c < p.N) ? min(max(p.K - k, 0), 2) : 0;
        const double* src = rows ? Bb + k + static_cast<int64_t>(c0 + c) * p.ldb : Bb;
        cp_async16(bs + k + c * LDB_S, src, rows * 8);
      }
      return;
    }
    if (load_c) {
      const double* Cb = p.C + b * p.strideC;
      for (int e = tid; e < UM * UN; e += UT) {
        const int r = e & (UM - 1), c = e >> 7;
        const bool ok = (r0 + r < p.M) && (c0 + c < p.N);
        const double* src = ok ? Cb + (r0 + r) + static_cast<int64_t>(c0 + c) * p.ldc : Cb;
        cp_async8(cs + r + c * LDC_S, src, ok ? 8 : 0);
      }
    }
    for (int e = tid; e < UK * UN; e += UT) {
      const int k = e & (UK - 1), c = e >> 5;
      const bool ok = (k < p.K) && (c0 + c < p.N);
      const double* src = ok ? Bb + k + static_cast<int64_t>(c0 + c) * p.ldb : Bb;
      cp_async8(bs + k + c * LDB_S, src, ok ? 8 : 0);
    }
  };

  // prologue: CSTAGES - 1 tiles in flight (empty groups keep the group count uniform)
#pragma unroll
  for (int s = 0; s < CSTAGES - 1; ++s) {
    if (t0 + s < t1) issue(t0 + s, s);
    cp_async_commit();
  }

  double af[4][4];  // A fragments of this warp's 16 rows, k-steps 0..3
  int cur_b = -1, cur_rb = -1;
  for (int64_t tau = t0; tau < t1; ++tau) {
    const int s = static_cast<int>((tau - t0) % CSTAGES);
    {
      const int64_t nx = tau + CSTAGES - 1;
      if (nx < t1) issue(nx, static_cast<int>((nx - t0) % CSTAGES));
      cp_async_commit();
    }
    int b, rb, ct;
    decode(tau, b, rb, ct);
    const int r0 = rb * UM, c0 = ct * UN;
    if (b != cur_b || rb != cur_rb) {
      cur_b = b;
      cur_rb = rb;
      const double* Ab = p.A + b * p.strideA;
      const int ra = r0 + warp * 16 + g;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        const int k0 = kk * 8 + t;
        af[kk][0] = (ra < p.M && k0 < p.K) ? Ab[ra + static_cast<int64_t>(k0) * p.lda] : 0.0;
        af[kk][1] = (ra + 8 < p.M && k0 < p.K) ? Ab[ra + 8 + static_cast<int64_t>(k0) * p.lda] : 0.0;
        af[kk][2] = (ra < p.M && k0 + 4 < p.K) ? Ab[ra + static_cast<int64_t>(k0 + 4) * p.lda] : 0.0;
        af[kk][3] = (ra + 8 < p.M && k0 + 4 < p.K) ? Ab[ra + 8 + static_cast<int64_t>(k0 + 4) * p.lda] : 0.0;
      }
    }
    cp_async_wait<CSTAGES - 1>();
    __syncthreads();
    const double* cs = sm + s * STAGE;
    const double* bs = cs + C_STAGE;
    double d[4][4];
#pragma unroll
    for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
      for (int q = 0; q < 4; ++q) d[nt][q] = 0.0;
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        double bf[2];
        bf[0] = bs[(kk * 8 + t) + (nt * 8 + g) * LDB_S];
        bf[1] = bs[(kk * 8 + t + 4) + (nt * 8 + g) * LDB_S];
        dmma_16x8x8(d[nt], af[kk], bf);
      }
    }
    double* Cb = p.C + b * p.strideC;
    const int rl = warp * 16 + g;
    if (V16) {
      // results into the stage (each thread rewrites what it read), then whole
      // 16-byte row pairs per thread: a warp stores 512 contiguous bytes of a column
      double* cw = sm + s * STAGE;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = rl + ((q & 2) ? 8 : 0);
          const int c = nt * 8 + 2 * t + (q & 1);
          double v = p.alpha * d[nt][q];
          if (load_c) v += p.beta * cw[r + c * LDC_S];
          cw[r + c * LDC_S] = v;
        }
      }
      __syncthreads();
      for (int e = tid; e < UM * UN / 2; e += UT) {
        const int r = (e & (UM / 2 - 1)) * 2, c = e >> 6;
        if (c0 + c >= p.N || r0 + r >= p.M) continue;
        double* dst = Cb + (r0 + r) + static_cast<int64_t>(c0 + c) * p.ldc;
        if (r0 + r + 1 < p.M) {
          *reinterpret_cast<double2*>(dst) = *reinterpret_cast<const double2*>(cw + r + c * LDC_S);
        } else {
          *dst = cw[r + c * LDC_S];
        }
      }
    } else {
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int r = rl + ((q & 2) ? 8 : 0);
          const int c = nt * 8 + 2 * t + (q & 1);
          if (r0 + r < p.M && c0 + c < p.N) {
            double v = p.alpha * d[nt][q];
            if (load_c) v += p.beta * cs[r + c * LDC_S];
            Cb[(r0 + r) + static_cast<int64_t>(c0 + c) * p.ldc] = v;
          }
        }
      }
    }
    __syncthreads();  // stage s is refilled by the next iteration's issue
  }
  cp_async_wait<0>();
}

}  // namespace

bool rank_update_applies(const GemmArgs& a) {
  return !a.transA && !a.transB && a.K >= 1 && a.K <= UK && !a.tri && !a.kfrom_n && !a.kto_m && !a.alpha_vec &&
         static_cast<int64_t>(a.M) * a.N >= static_cast<int64_t>(UM) * UN * 16;
}

cudaError_t rank_update(const GemmArgs& a, cudaStream_t st) {
  if (a.M <= 0 || a.N <= 0 || a.batch <= 0) return cudaSuccess;
  if (a.K < 1 || a.K > UK) return cudaErrorInvalidValue;
  UpdParams p;
  p.M = a.M;
  p.N = a.N;
  p.K = a.K;
  p.A = a.A;
  p.lda = a.lda;
  p.strideA = a.strideA;
  p.B = a.B;
  p.ldb = a.ldb;
  p.strideB = a.strideB;
  p.C = a.C;
  p.ldc = a.ldc;
  p.strideC = a.strideC;
  p.alpha = a.alpha;
  p.beta = a.beta;
  p.row_blocks = (a.M + UM - 1) / UM;
  p.col_tiles = (a.N + UN - 1) / UN;
  p.total = static_cast<int64_t>(a.batch) * p.row_blocks * p.col_tiles;
  constexpr int csmem = CSTAGES * STAGE * static_cast<int>(sizeof(double));
  static std::atomic<int> attr_set[kMaxDevices];
  const cudaError_t attr = once_per_device(attr_set, [] {
    const cudaError_t e =
        cudaFuncSetAttribute(rank_update_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, csmem);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(rank_update_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, csmem);
  });
  if (attr != cudaSuccess) return attr;
  auto al16 = [](const void* ptr, int64_t ld) {
    return reinterpret_cast<uintptr_t>(ptr) % 16 == 0 && ld % 2 == 0;
  };
  const bool v16 = al16(a.B, a.ldb) && al16(a.C, a.ldc) && (a.batch <= 1 || ((a.strideB | a.strideC) & 1) == 0);
  // at most kChunk tiles per CTA: CTAs retire every few tiles, so a Householder panel
  // launched on the high-priority side stream (look-ahead) finds SMs within ~tens of us
  constexpr int64_t kChunk = 8;
  const int64_t grid = std::max<int64_t>(std::min<int64_t>(p.total, 2 * static_cast<int64_t>(num_sms())),
                                         (p.total + kChunk - 1) / kChunk);
  if (v16)
    rank_update_kernel<true><<<static_cast<unsigned>(grid), UT, csmem, st>>>(p);
  else
    rank_update_kernel<false><<<static_cast<unsigned>(grid), UT, csmem, st>>>(p);
  return cudaGetLastError();
}

}  // namespace zolo
