// FP64 matrix products emulated on the INT8 tensor cores of sm_100a
// (tcgen05.mma kind::i8, exact INT32 accumulation in tensor memory) by the
// Ozaki splitting (Ozaki, Ogita, Oishi, Rump, "Error-free transformations of
// matrix multiplication by using fast routines of matrix multiplication and its
// applications", Numer. Algorithms 59, 2012), in its integer form.
//
// Splitting.  Row r of op(A) is scaled by 2^-e_r, e_r the exponent with
// max_k |op(A)(r,k)| < 2^e_r, and cut into S signed 7-bit digits by
// round-to-nearest:  op(A)(r,k) = 2^e_r sum_t a_t(r,k) 2^-7(t+1) + O(2^(e_r-7S)),
// a_t in [-127, 127] (int8).  Columns of op(B) likewise (exponents f_c).  Then
//   op(A) op(B) ~= 2^(e_r + f_c) sum_{d < S} 2^-7(d+2) D_d,
//   D_d = sum_{t+u=d} A_t B_u  (integer products, exact in INT32 for K <= 16384).
// The digit products with t + u >= S are below the splitting error and dropped:
// S(S+1)/2 INT8 products in all.  S = 8 gives FP64-level normwise accuracy.
//
// Kernel (persistent, one CTA per SM, 192 threads): warp 0 issues the TMA loads
// of one 32-byte K step of all S digit planes of a 128-row A tile and a 64-row B
// tile (one 4D box each, 32-byte swizzle) into a STAGES-deep ring; warp 1 issues,
// per K step and per A digit t, one MMA A_t x [B_0 | ... | B_{S-1-t}] whose
// accumulator is the contiguous TMEM column range of D_t .. D_{S-1} (64 columns
// per diagonal, S * 64 <= 512), so every digit plane is loaded once per K step;
// warps 2-5 drain the S diagonals from TMEM (tcgen05.ld), combine them in FP64
// by Horner's rule, scale by 2^(e_r + f_c), apply alpha/beta and store the tile.
// Every wait on an mbarrier is bounded: on a timeout the kernel records an error
// in a status word, drains what it issued and returns.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstdint>

#include "common.cuh"
#include "kernels.h"

namespace zolo {
namespace oz {

constexpr int BM = 128;  // rows of an A tile (UMMA M)
constexpr int BN = 64;   // rows of a B tile = columns of one diagonal accumulator
constexpr int BK = 32;   // bytes (= int8 elements) of K per pipeline stage (one UMMA K)
constexpr int kThreads = 192;
constexpr long long kTimeoutCycles = 2000000000LL;  // about a second at 1.9 GHz

template <int S>
struct Cfg {
  static constexpr int A_BYTES = S * BM * BK;
  static constexpr int B_BYTES = S * BN * BK;
  static constexpr int STAGE = A_BYTES + B_BYTES;
  static constexpr int STAGES = S >= 8 ? 4 : (S == 7 ? 5 : 6);
  static constexpr int SMEM = STAGES * STAGE + 1024 + 256;
  static_assert(S * BN <= 512, "diagonal accumulators exceed tensor memory");
};

struct Params {
  int M, N, K;
  int tiles_m, tiles_n, batch;
  int tri, kfrom_n, kto_m;
  double alpha, beta;
  double* C;
  int64_t ldc, strideC;
  const int* expA;  // e_r per batch entry: expA[b * rpadA + r]
  const int* expB;
  int rpadA, rpadB;
  int* status;
};

ZDEV uint32_t smem_u32(const void* p) { return static_cast<uint32_t>(__cvta_generic_to_shared(p)); }

ZDEV void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
ZDEV void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
ZDEV void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
ZDEV bool mbar_try_wait(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
// Bounded wait: false (and the CTA's abort flag set, the status word written) on a timeout
// or when another role of the CTA has aborted.
ZDEV bool mbar_wait(uint32_t bar, uint32_t parity, volatile int* abort_flag, int* status, int code) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (*abort_flag) return false;
    if (clock64() - t0 > kTimeoutCycles) {
      *abort_flag = 1;
      set_status(status, code);
      return false;
    }
  }
  return true;
}

ZDEV void tma_load_4d(uint32_t dst, const CUtensorMap* map, uint32_t bar, int c0, int c1, int c2, int c3) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, "
      "%5}], [%6];" ::"r"(dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(bar)
      : "memory");
}

// Shared-memory matrix descriptor of a K-major operand in the 32-byte swizzle layout the
// TMA writes: rows of 32 bytes, 8-row core groups 256 bytes apart (stride byte offset),
// leading byte offset unused (1), descriptor version 1, layout type 6 (SWIZZLE_32B).
ZDEV uint64_t sw32_desc(uint32_t addr) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFF) | (1ull << 16) | (16ull << 32) | (1ull << 46) |
         (6ull << 61);
}
// Instruction descriptor: D = S32 (bits 4-5 = 2), A and B signed 8-bit (bits 7-9, 10-12 = 1),
// both K-major, N >> 3 at bit 17, M >> 4 at bit 24 (M = 128).
ZDEV uint32_t i8_idesc(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (static_cast<uint32_t>(n >> 3) << 17) | (8u << 24);
}
ZDEV void umma_i8(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate)
      : "memory");
}
ZDEV void umma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar)
               : "memory");
}
ZDEV void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
ZDEV void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// 32 lanes x 16 columns of 32-bit TMEM words; the registers are valid after tmem_wait.
ZDEV void tmem_ld16(uint32_t taddr, uint32_t (&r)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
}
// Waits for this thread's TMEM loads; naming the registers orders their uses after the wait.
ZDEV void tmem_wait(uint32_t (&r)[16]) {
  asm volatile("tcgen05.wait::ld.sync.aligned;"
               : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                 "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                 "+r"(r[15])
               :
               : "memory");
}

// 2^k, exact (built from the IEEE-754 exponent field in the normal range)
ZDEV double pow2(int k) {
  if (k >= -1022 && k <= 1023) return __longlong_as_double(static_cast<long long>(k + 1023) << 52);
  return ldexp(1.0, k);
}

// Output tile t of the launch: batch entry, tile row and column, K-step range [kb0, kb1).
struct Tile {
  int b, mt, nt, kb0, kb1;
};
// tiles per batch entry; with `tri` only those meeting the lower triangle: tile row mt
// has min(tiles_n, 2 mt + 2) of them (BM = 2 BN)
ZDEV int tiles_per_entry(const Params& p) {
  if (!p.tri) return p.tiles_m * p.tiles_n;
  int per = 0;
  for (int i = 0; i < p.tiles_m; ++i) per += min(p.tiles_n, 2 * i + 2);
  return per;
}
ZDEV Tile tile_at(const Params& p, int t, int per) {
  Tile x;
  x.b = t / per;
  const int r = t - x.b * per;
  if (p.tri) {
    int rr = r, mt = 0;
    while (rr >= min(p.tiles_n, 2 * mt + 2)) {
      rr -= min(p.tiles_n, 2 * mt + 2);
      ++mt;
    }
    x.mt = mt;
    x.nt = rr;
  } else {
    // groups of 16 tile rows, rows fastest: concurrent CTAs share A and B tiles in L2
    const int group = r / (16 * p.tiles_n);
    const int first = group * 16;
    const int gm = min(16, p.tiles_m - first);
    const int in = r - group * 16 * p.tiles_n;
    x.mt = first + in % gm;
    x.nt = in / gm;
  }
  const int m0 = x.mt * BM, n0 = x.nt * BN;
  int k0 = 0, k1 = p.K;
  if (p.kfrom_n) k0 = p.kfrom_n == 1 ? n0 : (p.kfrom_n == 2 ? m0 : max(m0, n0));
  if (p.kto_m) k1 = min(k1, p.kto_m == 2 ? n0 + BN : m0 + BM);
  x.kb0 = k0 / BK;
  x.kb1 = (k1 + BK - 1) / BK;
  if (x.kb1 < x.kb0) x.kb1 = x.kb0;
  return x;
}

template <int S>
__global__ void __launch_bounds__(kThreads, 1)
    ozgemm_kernel(const __grid_constant__ CUtensorMap mapA, const __grid_constant__ CUtensorMap mapB, Params p) {
  using C = Cfg<S>;
  extern __shared__ __align__(1024) uint8_t smem_raw[];
  uint8_t* smem = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* bars = reinterpret_cast<uint64_t*>(smem + C::STAGES * C::STAGE);
  // bars: full[STAGES], empty[STAGES], acc_full, acc_empty, done; then the TMEM address and abort flag
  const uint32_t full0 = smem_u32(bars), empty0 = smem_u32(bars + C::STAGES);
  const uint32_t acc_full = smem_u32(bars + 2 * C::STAGES), acc_empty = smem_u32(bars + 2 * C::STAGES + 1);
  const uint32_t done_bar = smem_u32(bars + 2 * C::STAGES + 2);
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(bars + 2 * C::STAGES + 3);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < C::STAGES; ++s) {
      mbar_init(full0 + 8 * s, 1);
      mbar_init(empty0 + 8 * s, 1);
    }
    mbar_init(acc_full, 1);
    mbar_init(acc_empty, 4);
    mbar_init(done_bar, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapA)) : "memory");
    asm volatile("prefetch.tensormap [%0];" ::"l"(reinterpret_cast<uint64_t>(&mapB)) : "memory");
  }
  if (warp == 1) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" ::"r"(smem_u32(tmem_holder))
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_holder;
  const int per = tiles_per_entry(p);
  const int ntiles = per * p.batch;

  if (warp == 0) {
    if (lane == 0) {
      // TMA producer
      int stage = 0;
      uint32_t phase = 0;
      uint32_t armed = 0, last_parity = 0;  // per-stage bit masks, for the drain at the end
      bool ok = true;
      for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x) {
        const Tile x = tile_at(p, t, per);
        for (int kb = x.kb0; kb < x.kb1; ++kb) {
          if (!mbar_wait(empty0 + 8 * stage, phase ^ 1, abort_flag, p.status, 901)) {
            ok = false;
            break;
          }
          const uint32_t fb = full0 + 8 * stage;
          mbar_expect_tx(fb, C::STAGE);
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          tma_load_4d(sa, &mapA, fb, kb * BK, x.mt * BM, 0, x.b);
          tma_load_4d(sa + C::A_BYTES, &mapB, fb, kb * BK, x.nt * BN, 0, x.b);
          armed |= 1u << stage;
          last_parity = (last_parity & ~(1u << stage)) | (phase << stage);
          if (++stage == C::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
      }
      // every load this thread issued has landed before the CTA may exit (bounded)
      for (int s = 0; s < C::STAGES; ++s) {
        if (!(armed & (1u << s))) continue;
        const long long t0 = clock64();
        while (!mbar_try_wait(full0 + 8 * s, (last_parity >> s) & 1)) {
          if (clock64() - t0 > kTimeoutCycles) {
            set_status(p.status, 904);
            break;
          }
        }
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issuer
      int stage = 0;
      uint32_t phase = 0, acc_phase = 0;
      bool issued = false;
      for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const Tile x = tile_at(p, t, per);
        if (!mbar_wait(acc_empty, acc_phase ^ 1, abort_flag, p.status, 902)) break;
        acc_phase ^= 1;
        tc_fence_after();
        bool ok = true;
        for (int kb = x.kb0; kb < x.kb1; ++kb) {
          if (!mbar_wait(full0 + 8 * stage, phase, abort_flag, p.status, 903)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sa = smem_u32(smem + stage * C::STAGE);
          const uint32_t sb = sa + C::A_BYTES;
#pragma unroll
          for (int d = 0; d < S; ++d) {
            // A_d x [B_0 | ... | B_{S-1-d}] -> TMEM columns [64 d, 64 S), at most 256 per MMA
            const int ncols = (S - d) * BN;
#pragma unroll
            for (int part = 0; part * 256 < ncols; ++part) {
              const int nn = min(256, ncols - part * 256);
              const uint64_t adesc = sw32_desc(sa + d * BM * BK);
              const uint64_t bdesc = sw32_desc(sb + part * 256 * BK);
              const uint32_t acc = (kb > x.kb0 || d > 0) ? 1u : 0u;
              umma_i8(tmem + d * BN + part * 256, adesc, bdesc, i8_idesc(nn), acc);
            }
          }
          issued = true;
          umma_commit(empty0 + 8 * stage);
          if (++stage == C::STAGES) {
            stage = 0;
            phase ^= 1;
          }
        }
        if (!ok) break;
        if (x.kb1 > x.kb0) {
          umma_commit(acc_full);
        } else {
          mbar_arrive(acc_full);  // empty K range: the epilogue writes beta * C
        }
      }
      // all MMAs complete before the TMEM is released
      if (issued) {
        umma_commit(done_bar);
        const long long t0 = clock64();
        while (!mbar_try_wait(done_bar, 0)) {
          if (clock64() - t0 > kTimeoutCycles) {
            set_status(p.status, 905);
            break;
          }
        }
      }
    }
  } else {
    // epilogue: warps 2..5; warp w reads TMEM lanes 32 (w % 4) .. + 31
    const int q = warp & 3;
    uint32_t acc_phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const Tile x = tile_at(p, t, per);
      // warp-uniform outcome: the TMEM loads below are .sync.aligned
      const bool ok = __all_sync(0xffffffffu, mbar_wait(acc_full, acc_phase, abort_flag, p.status, 906));
      if (!ok) break;
      acc_phase ^= 1;
      tc_fence_after();
      const int r = x.mt * BM + q * 32 + lane;  // < rpadA
      const double srow = pow2(p.expA[static_cast<int64_t>(x.b) * p.rpadA + r] - 7) * p.alpha;
      double* Cb = p.C + static_cast<int64_t>(x.b) * p.strideC;
      const bool has_k = x.kb1 > x.kb0;
      const int* eb = p.expB + static_cast<int64_t>(x.b) * p.rpadB;
#pragma unroll 1
      for (int cc = 0; cc < BN / 16; ++cc) {
        double acc[16];
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[j] = 0.0;
        if (has_k) {
          uint32_t v[S][16];
#pragma unroll
          for (int d = 0; d < S; ++d)
            tmem_ld16(tmem + (static_cast<uint32_t>(q * 32) << 16) + d * BN + cc * 16, v[d]);
#pragma unroll
          for (int d = 0; d < S; ++d) tmem_wait(v[d]);
          // sum_d 2^-7d D_d by Horner's rule from the smallest diagonal
#pragma unroll
          for (int j = 0; j < 16; ++j) acc[j] = static_cast<double>(static_cast<int>(v[S - 1][j]));
#pragma unroll
          for (int d = S - 2; d >= 0; --d) {
#pragma unroll
            for (int j = 0; j < 16; ++j)
              acc[j] = fma(acc[j], 0.0078125, static_cast<double>(static_cast<int>(v[d][j])));
          }
        }
        if (r < p.M) {
#pragma unroll
          for (int j = 0; j < 16; ++j) {
            const int col = x.nt * BN + cc * 16 + j;
            if (col < p.N && (!p.tri || r >= col)) {
              double val = acc[j] * srow * pow2(eb[col] - 7);
              double* cp = Cb + r + static_cast<int64_t>(col) * p.ldc;
              if (p.beta != 0.0) val = fma(p.beta, *cp, val);
              *cp = val;
            }
          }
        }
      }
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(acc_empty);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 1) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" ::"r"(tmem) : "memory");
  }
}

// ---- splitting ----

// Row maxima of |op(X)| (op(X) is R x K; element (r, k) at X[k + r ld] when kmaj, else
// X[r + k ld]) as IEEE bit patterns, which order like the values for x >= 0.
__global__ void rowmax_kmaj_kernel(const double* X, int64_t ld, int64_t sx, int R, int K,
                                   unsigned long long* rowmax, int rpad) {
  const int b = blockIdx.y;
  const int row = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (row >= R) return;
  const double* p = X + b * sx + row * ld;
  double m = 0.0;
  for (int k = lane; k < K; k += 32) m = fmax(m, fabs(p[k]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0)
    rowmax[static_cast<int64_t>(b) * rpad + row] = static_cast<unsigned long long>(__double_as_longlong(m));
}

constexpr int kRowChunk = 64;
__global__ void rowmax_strided_kernel(const double* X, int64_t ld, int64_t sx, int R, int K,
                                      unsigned long long* rowmax, int rpad) {
  const int b = blockIdx.z;
  const int row = blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= R) return;
  const int k0 = blockIdx.y * kRowChunk, k1 = min(K, k0 + kRowChunk);
  const double* p = X + b * sx + row;
  double m = 0.0;
  for (int k = k0; k < k1; ++k) m = fmax(m, fabs(p[k * ld]));
  atomicMax(rowmax + static_cast<int64_t>(b) * rpad + row,
            static_cast<unsigned long long>(__double_as_longlong(m)));
}

// exponent e with max < 2^e (0 for a zero row)
ZDEV int row_exponent(unsigned long long bits) {
  if (bits == 0) return 0;
  int e;
  frexp(__longlong_as_double(static_cast<long long>(bits)), &e);
  return e;
}

// S digit planes of op(X) (R x K), K-major int8: plane t of batch entry b, row r at
// out[((b S + t) rpad + r) kpad + k]; zero in the padding r >= R or k >= K.  Tiles of
// 32 rows x 128 k staged through shared memory so both the FP64 reads and the int8
// writes are contiguous.  expo[b rpad + r] receives e_r.
template <int S>
__global__ void __launch_bounds__(256) slice_kernel(const double* X, int64_t ld, int64_t sx, int R, int K, int kmaj,
                                                    const unsigned long long* rowmax, int8_t* out, int* expo,
                                                    int rpad, int kpad) {
  __shared__ double tile[32][129];
  const int b = blockIdx.z, r0 = blockIdx.y * 32, k0 = blockIdx.x * 128, tid = threadIdx.x;
  const double* Xb = X + b * sx;
#pragma unroll 4
  for (int i = 0; i < 16; ++i) {
    const int idx = i * 256 + tid;
    const int rr = kmaj ? (idx >> 7) : (idx & 31);
    const int kk = kmaj ? (idx & 127) : (idx >> 5);
    const int r = r0 + rr, k = k0 + kk;
    tile[rr][kk] = (r < R && k < K)
                       ? Xb[kmaj ? k + static_cast<int64_t>(r) * ld : r + static_cast<int64_t>(k) * ld]
                       : 0.0;
  }
  __syncthreads();
  const int rr = tid >> 3, kg = (tid & 7) * 16, r = r0 + rr;
  const int e = r < R ? row_exponent(rowmax[static_cast<int64_t>(b) * rpad + r]) : 0;
  const double scale = pow2(7 - e);
  uint32_t w[S][4];
#pragma unroll
  for (int t = 0; t < S; ++t)
#pragma unroll
    for (int i = 0; i < 4; ++i) w[t][i] = 0;
#pragma unroll
  for (int j = 0; j < 16; ++j) {
    double y = tile[rr][kg + j] * scale;  // |y| < 128
#pragma unroll
    for (int t = 0; t < S; ++t) {
      const double a = fmin(127.0, fmax(-127.0, rint(y)));
      w[t][j >> 2] |= (static_cast<uint32_t>(static_cast<int>(a)) & 0xFFu) << (8 * (j & 3));
      y = (y - a) * 128.0;  // exact: the remainder of a rounding, scaled by a power of two
    }
  }
  if (k0 + kg < kpad) {
#pragma unroll
    for (int t = 0; t < S; ++t) {
      int8_t* dst = out + ((static_cast<int64_t>(b) * S + t) * rpad + r) * kpad + k0 + kg;
      *reinterpret_cast<uint4*>(dst) = make_uint4(w[t][0], w[t][1], w[t][2], w[t][3]);
    }
  }
  if (blockIdx.x == 0 && (tid & 7) == 0 && expo) expo[static_cast<int64_t>(b) * rpad + r] = e;
}

// ---- host side ----

// The driver's tensor-map encoder, looked up once (thread-safe static initialization).
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
    return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
  }();
  return fn;
}

// 4D map over the digit planes [batch][S][rpad][kpad] (int8) with a {32, rows, S, 1} box.
bool make_map(CUtensorMap* map, const int8_t* base, int S, int rpad, int kpad, int batch, int box_rows) {
  auto fn = encode_fn();
  if (!fn) return false;
  const cuuint64_t dims[4] = {static_cast<cuuint64_t>(kpad), static_cast<cuuint64_t>(rpad),
                              static_cast<cuuint64_t>(S), static_cast<cuuint64_t>(batch)};
  const cuuint64_t strides[3] = {static_cast<cuuint64_t>(kpad), static_cast<cuuint64_t>(kpad) * rpad,
                                 static_cast<cuuint64_t>(kpad) * rpad * S};
  const cuuint32_t box[4] = {static_cast<cuuint32_t>(BK), static_cast<cuuint32_t>(box_rows),
                             static_cast<cuuint32_t>(S), 1};
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, const_cast<int8_t*>(base), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_32B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

template <int S>
cudaError_t set_smem_attr() {
  static std::atomic<int> attr_set[kMaxDevices];
  return once_per_device(attr_set, [] {
    return cudaFuncSetAttribute(ozgemm_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg<S>::SMEM);
  });
}

template <int S>
cudaError_t slice_launch(const double* X, int64_t ld, int64_t sx, int R, int K, int kmaj, unsigned long long* rowmax,
                         int8_t* out, int* expo, int rpad, int kpad, int batch, cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(rowmax, 0, sizeof(unsigned long long) * rpad * batch, st);
  if (e != cudaSuccess) return e;
  if (kmaj) {
    rowmax_kmaj_kernel<<<dim3((R + 7) / 8, batch), 256, 0, st>>>(X, ld, sx, R, K, rowmax, rpad);
  } else {
    rowmax_strided_kernel<<<dim3((R + 255) / 256, (K + kRowChunk - 1) / kRowChunk, batch), 256, 0, st>>>(
        X, ld, sx, R, K, rowmax, rpad);
  }
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  slice_kernel<S><<<dim3((kpad + 127) / 128, rpad / 32, batch), 256, 0, st>>>(X, ld, sx, R, K, kmaj, rowmax, out,
                                                                              expo, rpad, kpad);
  return cudaGetLastError();
}

template <int S>
cudaError_t run(const GemmArgs& a, const OzWork& w, cudaStream_t st, int sms) {
  const int rpadA = (a.M + BM - 1) / BM * BM, rpadB = (a.N + BN - 1) / BN * BN;
  const int kpad = (a.K + BK - 1) / BK * BK;
  // op(A) row r, k: A[k + r lda] if transA else A[r + k lda]; op(B)^T row c, k: B[c + k ldb]
  // if transB else B[k + c ldb]
  const int kmajA = a.transA ? 1 : 0, kmajB = a.transB ? 0 : 1;
  cudaError_t e = slice_launch<S>(a.A, a.lda, a.strideA, a.M, a.K, kmajA, w.maxA, w.sliceA, w.expA, rpadA, kpad,
                                  a.batch, st);
  if (e != cudaSuccess) return e;
  // X^T X-type products (the same matrix on both sides, read the same way): one splitting
  const bool same = a.A == a.B && a.lda == a.ldb && a.strideA == a.strideB && kmajA == kmajB && a.M == a.N;
  const int8_t* sB = w.sliceA;
  const int* eB = w.expA;
  if (!same) {
    e = slice_launch<S>(a.B, a.ldb, a.strideB, a.N, a.K, kmajB, w.maxB, w.sliceB, w.expB, rpadB, kpad, a.batch,
                        st);
    if (e != cudaSuccess) return e;
    sB = w.sliceB;
    eB = w.expB;
  }
  // with the same splitting on both sides the B map reads the A planes (rows padded to BM)
  const int rpadBm = same ? rpadA : rpadB;
  CUtensorMap mapA, mapB;
  if (!make_map(&mapA, w.sliceA, S, rpadA, kpad, a.batch, BM) || !make_map(&mapB, sB, S, rpadBm, kpad, a.batch, BN))
    return cudaErrorInvalidValue;
  e = set_smem_attr<S>();
  if (e != cudaSuccess) return e;
  Params p;
  p.M = a.M;
  p.N = a.N;
  p.K = a.K;
  p.tiles_m = rpadA / BM;
  p.tiles_n = rpadB / BN;
  p.batch = a.batch;
  p.tri = a.tri;
  p.kfrom_n = a.kfrom_n;
  p.kto_m = a.kto_m;
  p.alpha = a.alpha;
  p.beta = a.beta;
  p.C = a.C;
  p.ldc = a.ldc;
  p.strideC = a.strideC;
  p.expA = w.expA;
  p.expB = eB;
  p.rpadA = rpadA;
  p.rpadB = rpadBm;
  p.status = w.status;
  int64_t tiles = 0;
  if (a.tri) {
    for (int i = 0; i < p.tiles_m; ++i) tiles += std::min(p.tiles_n, 2 * i + 2);
  } else {
    tiles = static_cast<int64_t>(p.tiles_m) * p.tiles_n;
  }
  tiles *= a.batch;
  if (tiles <= 0 || tiles > 0x7fffffff) return cudaErrorInvalidValue;
  const int grid = static_cast<int>(std::min<int64_t>(tiles, sms));
  if (w.before_kernel) {
    e = cudaEventRecord(w.before_kernel, st);
    if (e == cudaSuccess && w.before_kernel2) e = cudaEventRecord(w.before_kernel2, st);
    if (e != cudaSuccess) return e;
  }
  ozgemm_kernel<S><<<grid, kThreads, Cfg<S>::SMEM, st>>>(mapA, mapB, p);
  return cudaGetLastError();
}

}  // namespace oz

size_t ozgemm_work_bytes(const GemmArgs& a, int slices, OzWorkSizes* sz) {
  const size_t rpadA = (a.M + oz::BM - 1) / oz::BM * oz::BM, rpadB = (a.N + oz::BN - 1) / oz::BN * oz::BN;
  const size_t kpad = (a.K + oz::BK - 1) / oz::BK * oz::BK;
  const size_t b = a.batch;
  sz->slice_a = b * slices * rpadA * kpad;
  sz->slice_b = b * slices * rpadB * kpad;
  sz->rows_a = b * rpadA;
  sz->rows_b = b * rpadB;
  return sz->slice_a + sz->slice_b + 12 * (sz->rows_a + sz->rows_b);
}

bool ozgemm_k_ok(int slices, int K) { return static_cast<double>(slices) * 127.0 * 127.0 * K < 2147483647.0; }

cudaError_t ozgemm(const GemmArgs& a, int slices, const OzWork& w, cudaStream_t st, int sms) {
  if (a.M <= 0 || a.N <= 0 || a.batch <= 0) return cudaSuccess;
  if (a.tri && a.M != a.N) return cudaErrorInvalidValue;
  if (a.K <= 0)
    return scale_copy(a.M, a.N, a.beta, a.C, a.ldc, a.strideC, a.C, a.ldc, a.strideC, a.batch, 0.0, st);
  if (a.alpha_vec) return cudaErrorInvalidValue;
  // exact INT32 accumulation: S products of |digits| <= 127 over K terms stay below 2^31
  if (!ozgemm_k_ok(slices, a.K)) return cudaErrorInvalidValue;
  switch (slices) {
    case 6:
      return oz::run<6>(a, w, st, sms);
    case 7:
      return oz::run<7>(a, w, st, sms);
    case 8:
      return oz::run<8>(a, w, st, sms);
    default:
      return cudaErrorInvalidValue;
  }
}

}  // namespace zolo
