// FP64 GEMM on the sm_100a FP64 tensor path (DMMA mma.sync.m16n8k8.f64).
//
// tcgen05.mma has no FP64 kind, so the FP64 contractions of the polar
// iterations (Gram matrix, TRSM updates, Householder trailing updates,
// Q1*Q2^T) run on DMMA.  General shapes: CTA tile 64x128x16, 8 warps (2 x 4),
// warp tile 32x32, 3-stage cp.async pipeline, two CTAs per SM (measured 33.1
// TF/s on a 4096^3 main-loop probe against 30.3 for 128x128 tiles with one CTA
// per SM; the FP64 tensor pipe saturates at 37.0).  Padded shared-memory
// layouts make every fragment load a conflict-free LDS.128 (or LDS.64 for
// op(B)=B^T).
//
// Index permutations (free because they are applied consistently):
//   * inside each 16-row MMA tile, logical row g <-> physical row 2g and
//     logical row g+8 <-> physical row 2g+1, so a thread's two A rows are
//     adjacent in memory;
//   * inside each 8-wide k step, logical k slot t <-> physical k 2t and slot
//     t+4 <-> 2t+1 for both operands, so a thread's two k values are adjacent.
#include "common.cuh"
#include "kernels.h"

#include <algorithm>

namespace zolo {

namespace {

constexpr int BK = 16, NT = 256;
constexpr int LDA_T = BK + 4;  // sA[m][k]  (op(A) = A^T)
constexpr int LDB_N = BK + 8;  // sB[n][k]  (op(B) = B)

// CTA tile BM x BN, WM x WN warps, each warp owns (BM/WM) x (BN/WN) = MI m16 x NJ n8 MMA tiles.
template <int BM_, int BN_, int WM_, int WN_, int ST_ = 4, int MINB_ = 1>
struct Cfg {
  static constexpr int BM = BM_, BN = BN_, WM = WM_, WN = WN_, STAGES = ST_, MINB = MINB_;
  static constexpr int MI = BM / WM / 16, NJ = BN / WN / 8;
  static constexpr int LDA_N = BM + 2;  // sA[k][m]  (op(A) = A)
  static constexpr int LDB_T = BN + 2;  // sB[k][n]  (op(B) = B^T)
  static_assert(WM * WN * 32 == NT, "8 warps");
  __host__ __device__ static constexpr int a_elems(bool ta) { return ta ? BM * LDA_T : BK * LDA_N; }
  __host__ __device__ static constexpr int b_elems(bool tb) { return tb ? BK * LDB_T : BN * LDB_N; }
  static constexpr int smem(bool ta, bool tb) { return ST_ * (a_elems(ta) + b_elems(tb)) * 8; }
};
using CfgWide = Cfg<64, 128, 2, 4, 3, 2>;     // general: 2 CTAs / SM, warp tile 32x32
using CfgSkinnyM = Cfg<32, 64, 1, 8, 4, 3>;    // M <= 32 (V^T W products of the QR updates)
using CfgSmall = Cfg<64, 64, 2, 4, 2, 3>;      // K <= 64 rank-k updates and N <= 64: 3 CTAs / SM
using CfgTri = Cfg<64, 64, 2, 4, 3, 3>;        // lower-triangle output (square tiles): 3 CTAs / SM

struct KParams {
  GemmArgs g;
  int tiles_m, tiles_n;
  int splitk;
  int preload;  // C loaded into the accumulators up front (rank-k updates)
  double* P;  // split-K partials
  int64_t ldp;
};

template <class C, bool TA, bool TB, bool V16>
__global__ void __launch_bounds__(NT, C::MINB) dgemm_kernel(KParams kp) {
  constexpr int BM = C::BM, BN = C::BN, MI = C::MI, NJ = C::NJ;
  constexpr int LDA_N = C::LDA_N, LDB_T = C::LDB_T;
  constexpr int AE = C::a_elems(TA), BE = C::b_elems(TB);
  constexpr int STAGES = C::STAGES;
  extern __shared__ __align__(16) double smem[];
  const GemmArgs& p = kp.g;
  double* sAb = smem;
  double* sBb = smem + STAGES * AE;

  const int bz = blockIdx.z;
  const int split = blockIdx.y;
  int tm, tn;
  if (p.tri) {
    const int t = blockIdx.x;
    int r = static_cast<int>((sqrtf(8.0f * t + 1.0f) - 1.0f) * 0.5f);
    while ((r + 1) * (r + 2) / 2 <= t) ++r;
    while (r * (r + 1) / 2 > t) --r;
    tm = r;
    tn = t - r * (r + 1) / 2;
  } else {
    const int G = 8;
    const int t = blockIdx.x;
    const int group = t / (G * kp.tiles_n);
    const int first = group * G;
    const int gsz = min(kp.tiles_m - first, G);
    const int in = t - group * G * kp.tiles_n;
    tm = first + in % gsz;
    tn = in / gsz;
  }
  const int m0 = tm * BM, n0 = tn * BN;
  const int M = p.M, N = p.N;

  int kb = 0, ke = p.K;
  if (p.kfrom_n) kb = min((p.kfrom_n == 1 ? n0 : (p.kfrom_n == 2 ? m0 : max(m0, n0))) / BK * BK, ke);
  if (p.kto_m) ke = max(kb, min(ke, p.kto_m == 2 ? n0 + BN : m0 + BM));
  if (kp.splitk > 1) {
    const int span = ke - kb;
    int len = (span + kp.splitk - 1) / kp.splitk;
    len = (len + BK - 1) / BK * BK;
    const int nb = kb + split * len;
    kb = min(nb, ke);
    ke = min(nb + len, ke);
  }

  const double* A = p.A + static_cast<int64_t>(bz) * p.strideA;
  const double* B = p.B + static_cast<int64_t>(bz) * p.strideB;
  const int64_t lda = p.lda, ldb = p.ldb;
  const int tid = threadIdx.x;

  // 16-byte chunks (two FP64 values along the contiguous dimension).  V16: one
  // cp.async of 16 bytes with zero fill; otherwise two 8-byte copies.
  auto chunk = [&](double* dst, const double* base, int64_t off0, bool in0, bool in1) {
    if (V16) {
      const int bytes = in0 ? (in1 ? 16 : 8) : 0;
      cp_async16(dst, bytes ? base + off0 : base, bytes);
    } else {
      cp_async8(dst, in0 ? base + off0 : base, in0 ? 8 : 0);
      cp_async8(dst + 1, in1 ? base + off0 + 1 : base, in1 ? 8 : 0);
    }
  };
  auto load_stage = [&](int stage, int k0) {
    double* sa = sAb + stage * AE;
    double* sb = sBb + stage * BE;
    for (int c = tid; c < BM * BK / 2; c += NT) {
      if (!TA) {
        const int k = c / (BM / 2), m = (c % (BM / 2)) * 2;
        const int gm = m0 + m, gk = k0 + k;
        const bool kin = gk < ke;
        chunk(sa + k * LDA_N + m, A, gm + static_cast<int64_t>(gk) * lda, kin && gm < M, kin && gm + 1 < M);
      } else {
        const int m = c / (BK / 2), k = (c % (BK / 2)) * 2;
        const int gm = m0 + m, gk = k0 + k;
        const bool mi = gm < M;
        chunk(sa + m * LDA_T + k, A, gk + static_cast<int64_t>(gm) * lda, mi && gk < ke, mi && gk + 1 < ke);
      }
    }
    for (int c = tid; c < BN * BK / 2; c += NT) {
      if (!TB) {
        const int n = c / (BK / 2), k = (c % (BK / 2)) * 2;
        const int gn = n0 + n, gk = k0 + k;
        const bool ni = gn < N;
        chunk(sb + n * LDB_N + k, B, gk + static_cast<int64_t>(gn) * ldb, ni && gk < ke, ni && gk + 1 < ke);
      } else {
        const int k = c / (BN / 2), n = (c % (BN / 2)) * 2;
        const int gn = n0 + n, gk = k0 + k;
        const bool kin = gk < ke;
        chunk(sb + k * LDB_T + n, B, gn + static_cast<int64_t>(gk) * ldb, kin && gn < N, kin && gn + 1 < N);
      }
    }
  };

  const int warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = (warp % C::WM) * (BM / C::WM);
  const int wn = (warp / C::WM) * (BN / C::WN);

  double acc[MI][NJ][4];
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j)
#pragma unroll
      for (int r = 0; r < 4; ++r) acc[i][j][r] = 0.0;

  const int ktiles = (ke > kb) ? (ke - kb + BK - 1) / BK : 0;
  // Rank-k updates C += alpha A B with |alpha| = 1 (the Householder and TRSM updates) are
  // bound by streaming C: its tile is loaded into the accumulators before the MMAs, so the
  // C reads overlap the A/B copies instead of following them.  C is pre-scaled by
  // beta/alpha (exact for alpha = +-1) and the epilogue then writes alpha * acc.
  const bool preload = kp.preload;
  if (preload) {
    const double* Cb = p.C + static_cast<int64_t>(bz) * p.strideC;
    const double sc = p.beta / p.alpha;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int r = m0 + wm + i * 16 + 2 * g;
        const int c = n0 + wn + j * 8 + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int cc = c + h;
          if (cc >= N || r >= M) continue;
          const double* src = Cb + r + static_cast<int64_t>(cc) * p.ldc;
          if (V16 && r + 1 < M) {
            const double2 o = *reinterpret_cast<const double2*>(src);
            acc[i][j][h] = sc * o.x;
            acc[i][j][2 + h] = sc * o.y;
          } else {
            acc[i][j][h] = sc * src[0];
            if (r + 1 < M) acc[i][j][2 + h] = sc * src[1];
          }
        }
      }
  }
#pragma unroll
  for (int s = 0; s < STAGES - 1; ++s) {
    if (s < ktiles) load_stage(s, kb + s * BK);
    cp_async_commit();
  }

  for (int kt = 0; kt < ktiles; ++kt) {
    cp_async_wait<STAGES - 2>();
    __syncthreads();
    {
      const int nk = kt + STAGES - 1;
      if (nk < ktiles) load_stage(nk % STAGES, kb + nk * BK);
      cp_async_commit();
    }
    const double* sa = sAb + (kt % STAGES) * AE;
    const double* sb = sBb + (kt % STAGES) * BE;
#pragma unroll
    for (int kk = 0; kk < BK / 8; ++kk) {
      double af[MI][4];
      double bf[NJ][2];
#pragma unroll
      for (int i = 0; i < MI; ++i) {
        const int m = wm + i * 16 + 2 * g;
        if (!TA) {
          const double2 v0 = *reinterpret_cast<const double2*>(sa + (kk * 8 + 2 * t) * LDA_N + m);
          const double2 v1 = *reinterpret_cast<const double2*>(sa + (kk * 8 + 2 * t + 1) * LDA_N + m);
          af[i][0] = v0.x;
          af[i][1] = v0.y;
          af[i][2] = v1.x;
          af[i][3] = v1.y;
        } else {
          const double2 v0 = *reinterpret_cast<const double2*>(sa + m * LDA_T + kk * 8 + 2 * t);
          const double2 v1 = *reinterpret_cast<const double2*>(sa + (m + 1) * LDA_T + kk * 8 + 2 * t);
          af[i][0] = v0.x;
          af[i][2] = v0.y;
          af[i][1] = v1.x;
          af[i][3] = v1.y;
        }
      }
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int n = wn + j * 8 + g;
        if (!TB) {
          const double2 v = *reinterpret_cast<const double2*>(sb + n * LDB_N + kk * 8 + 2 * t);
          bf[j][0] = v.x;
          bf[j][1] = v.y;
        } else {
          bf[j][0] = sb[(kk * 8 + 2 * t) * LDB_T + n];
          bf[j][1] = sb[(kk * 8 + 2 * t + 1) * LDB_T + n];
        }
      }
#pragma unroll
      for (int i = 0; i < MI; ++i)
#pragma unroll
        for (int j = 0; j < NJ; ++j) dmma_16x8x8(acc[i][j], af[i], bf[j]);
    }
  }
  cp_async_wait<0>();

  // ---- epilogue ----
  if (kp.splitk > 1) {
    double* P = kp.P + (static_cast<int64_t>(split) * p.batch + bz) * kp.ldp * N;
#pragma unroll
    for (int i = 0; i < MI; ++i)
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const int r = m0 + wm + i * 16 + 2 * g;
        const int c = n0 + wn + j * 8 + 2 * t;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int cc = c + h;
          if (cc >= N) continue;
          double* dst = P + r + static_cast<int64_t>(cc) * kp.ldp;
          if (r < M) dst[0] = acc[i][j][h];
          if (r + 1 < M) dst[1] = acc[i][j][2 + h];
        }
      }
    return;
  }
  double* C_ = p.C + static_cast<int64_t>(bz) * p.strideC;
  const int64_t ldc = p.ldc;
  const double alpha = p.alpha * (p.alpha_vec ? p.alpha_vec[bz] : 1.0);
  const double beta = preload ? 0.0 : p.beta;
#pragma unroll
  for (int i = 0; i < MI; ++i)
#pragma unroll
    for (int j = 0; j < NJ; ++j) {
      const int r = m0 + wm + i * 16 + 2 * g;
      const int c = n0 + wn + j * 8 + 2 * t;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int cc = c + h;
        if (cc >= N || r >= M) continue;
        double* dst = C_ + r + static_cast<int64_t>(cc) * ldc;
        double v0 = alpha * acc[i][j][h];
        double v1 = alpha * acc[i][j][2 + h];
        const bool ok0 = !p.tri || r >= cc;
        const bool ok1 = (r + 1 < M) && (!p.tri || r + 1 >= cc);
        if (V16 && ok0 && ok1) {
          if (beta != 0.0) {
            const double2 o = *reinterpret_cast<const double2*>(dst);
            v0 += beta * o.x;
            v1 += beta * o.y;
          }
          *reinterpret_cast<double2*>(dst) = make_double2(v0, v1);
        } else {
          if (ok0) dst[0] = (beta != 0.0) ? v0 + beta * dst[0] : v0;
          if (ok1) dst[1] = (beta != 0.0) ? v1 + beta * dst[1] : v1;
        }
      }
    }
}

__global__ void splitk_reduce_kernel(GemmArgs p, int splitk, const double* P, int64_t ldp) {
  const int64_t total = static_cast<int64_t>(p.M) * p.N;
  const int bz = blockIdx.y;
  const double alpha = p.alpha * (p.alpha_vec ? p.alpha_vec[bz] : 1.0);
  double* C = p.C + static_cast<int64_t>(bz) * p.strideC;
  for (int64_t e = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; e < total;
       e += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    const int i = static_cast<int>(e % p.M);
    const int j = static_cast<int>(e / p.M);
    if (p.tri && i < j) continue;
    double s = 0.0;
    for (int q = 0; q < splitk; ++q)
      s += P[(static_cast<int64_t>(q) * p.batch + bz) * ldp * p.N + i + static_cast<int64_t>(j) * ldp];
    double* dst = C + i + static_cast<int64_t>(j) * p.ldc;
    double v = alpha * s;
    if (p.beta != 0.0) v += p.beta * *dst;
    *dst = v;
  }
}

template <class C, bool TA, bool TB, bool V16>
cudaError_t launch_t(const KParams& kp, dim3 grid, cudaStream_t st) {
  static std::atomic<int> attr_set[kMaxDevices];
  const cudaError_t attr = once_per_device(attr_set, [] {
    return cudaFuncSetAttribute(dgemm_kernel<C, TA, TB, V16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                C::smem(TA, TB));
  });
  if (attr != cudaSuccess) return attr;
  dgemm_kernel<C, TA, TB, V16><<<grid, NT, C::smem(TA, TB), st>>>(kp);
  return cudaGetLastError();
}

template <class C, bool V16>
cudaError_t launch_v(const KParams& kp, dim3 grid, cudaStream_t st) {
  const GemmArgs& a = kp.g;
  if (!a.transA && !a.transB) return launch_t<C, false, false, V16>(kp, grid, st);
  if (!a.transA && a.transB) return launch_t<C, false, true, V16>(kp, grid, st);
  if (a.transA && !a.transB) return launch_t<C, true, false, V16>(kp, grid, st);
  return launch_t<C, true, true, V16>(kp, grid, st);
}

template <class C>
cudaError_t launch_c(const KParams& kp, dim3 grid, bool v16, cudaStream_t st) {
  return v16 ? launch_v<C, true>(kp, grid, st) : launch_v<C, false>(kp, grid, st);
}

// tile shape: 0 = 64x128 (general), 1 = 32x64 (M <= 32), 2 = 64x64 (K <= 64 or N <= 64),
// 3 = 64x64 with 3 stages (lower-triangle output)
int pick_cfg(const GemmArgs& a) {
  if (a.tri) return 3;
  if (a.M <= 32) return 1;
  if (a.K <= 64 || a.N <= 64) return 2;
  // C += A B updates with K <= 256 (the 128-column block reflector updates of the QR):
  // 64 x 64 tiles, three CTAs per SM, C loaded up front (21.7 TF/s against 18.7 for
  // 64 x 128 tiles at M = 16384, N = 4096, K = 128)
  if (a.K <= 256 && !a.transA && a.beta != 0.0) return 2;
  return 0;
}

void tile_dims(int cfg, int* bm, int* bn, int* per_sm) {
  if (cfg == 1) {
    *bm = CfgSkinnyM::BM;
    *bn = CfgSkinnyM::BN;
    *per_sm = CfgSkinnyM::MINB;
  } else if (cfg == 2) {
    *bm = CfgSmall::BM;
    *bn = CfgSmall::BN;
    *per_sm = CfgSmall::MINB;
  } else if (cfg == 3) {
    *bm = CfgTri::BM;
    *bn = CfgTri::BN;
    *per_sm = CfgTri::MINB;
  } else {
    *bm = CfgWide::BM;
    *bn = CfgWide::BN;
    *per_sm = CfgWide::MINB;
  }
}

// Split K only when the tile grid cannot fill the GPU; pick the split that fills whole
// waves (sms * resident CTAs per SM) best, with at least 8 K tiles per split.
int choose_splitk(const GemmArgs& a, int sms) {
  if (a.splitk >= 1) return a.splitk;
  int BM, BN, per_sm;
  tile_dims(pick_cfg(a), &BM, &BN, &per_sm);
  const int tm = (a.M + BM - 1) / BM, tn = (a.N + BN - 1) / BN;
  const int64_t tiles = a.tri ? static_cast<int64_t>(tm) * (tm + 1) / 2 : static_cast<int64_t>(tm) * tn;
  const int64_t ctas = tiles * a.batch;
  const int64_t wave = static_cast<int64_t>(sms) * per_sm;
  if (ctas >= wave) return 1;
  const int kt = (a.K + BK - 1) / BK;
  const int smax = std::min(32, kt / 8);
  if (smax < 2) return 1;
  int best = 1;
  double best_eff = static_cast<double>(ctas) / wave;  // fraction of one wave used unsplit
  for (int s = 2; s <= smax; ++s) {
    const int64_t c = ctas * s;
    const int64_t waves = (c + wave - 1) / wave;
    const double eff = static_cast<double>(c) / (waves * wave);  // wave fill
    // prefer more parallelism until the first full wave, then fill
    const double score = (c < wave ? static_cast<double>(c) / wave : eff) * (waves <= 3 ? 1.0 : 0.9);
    if (score > best_eff + 1e-9) {
      best_eff = score;
      best = s;
    }
  }
  return best;
}

}  // namespace

int num_sms() {
  static std::atomic<int> cache[kMaxDevices];
  return per_device_value(cache, [] {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    return sms > 0 ? sms : 148;
  });
}

size_t dgemm_splitk_bytes(const GemmArgs& a, int sms) {
  const int s = choose_splitk(a, sms);
  if (s <= 1) return 0;
  const int64_t ldp = (a.M + 1) / 2 * 2;
  return static_cast<size_t>(s) * a.batch * ldp * a.N * sizeof(double);
}

cudaError_t dgemm(GemmArgs a, const Scratch& ws, cudaStream_t st) {
  if (a.M <= 0 || a.N <= 0 || a.batch <= 0) return cudaSuccess;
  if (a.tri && a.M != a.N) return cudaErrorInvalidValue;
  // 16-byte cp.async path when every tile chunk is 16-byte aligned, else 8-byte copies
  auto al = [](const void* ptr, int64_t ld) {
    return (reinterpret_cast<uintptr_t>(ptr) % 16 == 0) && (ld % 2 == 0);
  };
  auto al8 = [](const void* ptr) { return reinterpret_cast<uintptr_t>(ptr) % 8 == 0; };
  if (!al8(a.A) || !al8(a.B) || !al8(a.C)) return cudaErrorMisalignedAddress;
  const bool v16 = al(a.A, a.lda) && al(a.B, a.ldb) && al(a.C, a.ldc) &&
                   (a.batch <= 1 || ((a.strideA | a.strideB | a.strideC) & 1) == 0);
  if (rank_update_applies(a)) return rank_update(a, st);
  const int sms = num_sms();
  if (a.K <= 0) {
    // C = beta*C
    return scale_copy(a.M, a.N, a.beta, a.C, a.ldc, a.strideC, a.C, a.ldc, a.strideC, a.batch, 0.0, st);
  }
  KParams kp;
  kp.g = a;
  const int cfg = pick_cfg(a);
  int BM, BN, per_sm;
  tile_dims(cfg, &BM, &BN, &per_sm);
  kp.tiles_m = (a.M + BM - 1) / BM;
  kp.tiles_n = (a.N + BN - 1) / BN;
  kp.splitk = choose_splitk(a, sms);
  kp.ldp = (a.M + 1) / 2 * 2;
  kp.P = nullptr;
  if (kp.splitk > 1) {
    const size_t need = static_cast<size_t>(kp.splitk) * a.batch * kp.ldp * a.N * sizeof(double);
    if (ws.ptr == nullptr || ws.bytes < need) {
      kp.splitk = 1;  // not enough scratch: run unsplit
    } else {
      kp.P = ws.ptr;
    }
  }
  kp.preload = (kp.splitk <= 1 && a.beta != 0.0 && !a.tri && !a.kto_m && !a.alpha_vec &&
                 (a.alpha == 1.0 || a.alpha == -1.0) && (a.K <= 64 || (cfg == 2 && a.K <= 256)))
                   ? 1
                   : 0;
  const int64_t tiles = a.tri ? static_cast<int64_t>(kp.tiles_m) * (kp.tiles_m + 1) / 2
                              : static_cast<int64_t>(kp.tiles_m) * kp.tiles_n;
  if (tiles > 0x7fffffff || a.batch > 65535) return cudaErrorInvalidValue;
  dim3 grid(static_cast<unsigned>(tiles), kp.splitk, a.batch);
  const cudaError_t e = cfg == 1   ? launch_c<CfgSkinnyM>(kp, grid, v16, st)
                        : cfg == 2 ? launch_c<CfgSmall>(kp, grid, v16, st)
                        : cfg == 3 ? launch_c<CfgTri>(kp, grid, v16, st)
                                   : launch_c<CfgWide>(kp, grid, v16, st);
  if (e != cudaSuccess || kp.splitk <= 1) return e;
  const int64_t total = static_cast<int64_t>(a.M) * a.N;
  int blocks = static_cast<int>(std::min<int64_t>((total + 255) / 256, 4 * sms));
  splitk_reduce_kernel<<<dim3(blocks, a.batch), 256, 0, st>>>(a, kp.splitk, kp.P, kp.ldp);
  return cudaGetLastError();
}

}  // namespace zolo
