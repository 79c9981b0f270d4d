// Cholesky entry point that allocates nothing on the device.
//
// Some callers cannot let a library call cudaMalloc: a Fortran or C host whose
// device memory is owned entirely by another allocator (a framework's caching
// pool that has reserved the GPU, or an application-level arena), and
// latency-sensitive callers for whom cudaMalloc's implicit device-wide
// synchronisation is not acceptable.  zolo_dpotrf_noalloc serves them: it runs
// the same recursive blocked Cholesky as zolo_dpotrf_dev, but its scratch (the
// copy of the sub-diagonal panel, the inverses of the 64 x 64 diagonal blocks
// and the INFO word) lives in file-scope __device__ arrays of a fixed size,
// which limits n to ZOLO_NOALLOC_MAX_N = 1024.  Every GPU that loads the
// library holds these arrays (2.5 MiB) until the process exits.
//
// Host code must not pass the arrays' names to a kernel (in host code the name
// is a host-side stand-in, not a device address): the device address is looked
// up with cudaGetSymbolAddress once per device, on the first call made with
// that device current, and cached.  All calls share the arrays, which keep the
// last call's contents; the INFO word is cleared at the start of every call.
// Calls that overlap on the GPU (different streams, or different host threads)
// race on the shared scratch and must be serialised by the caller.
#include <mutex>

#include "../../include/zolo_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace zolo {
namespace {

constexpr int kMaxN = ZOLO_NOALLOC_MAX_N;
constexpr int kLeafN = 64;
constexpr size_t kTmpDoubles = static_cast<size_t>(kMaxN / 2) * (kMaxN / 2);             // largest A21 copy
constexpr size_t kDinvDoubles = static_cast<size_t>(kMaxN / kLeafN) * kLeafN * kLeafN;  // block inverses

static __device__ __align__(256) double g_potrf_scratch[kTmpDoubles + kDinvDoubles];
static __device__ __align__(256) int g_potrf_info[64];

struct DevicePtrs {
  double* scratch = nullptr;
  int* info = nullptr;
};
std::mutex g_mu;
DevicePtrs g_ptrs[128];

// device addresses of the static arrays for the current device (set up once per device)
cudaError_t device_ptrs(DevicePtrs* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 128) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_mu);
  DevicePtrs& p = g_ptrs[dev];
  if (!p.scratch) {
    void* s = nullptr;
    void* i = nullptr;
    e = cudaGetSymbolAddress(&s, g_potrf_scratch);
    if (e != cudaSuccess) return e;
    e = cudaGetSymbolAddress(&i, g_potrf_info);
    if (e != cudaSuccess) return e;
    p.scratch = static_cast<double*>(s);
    p.info = static_cast<int*>(i);
  }
  *out = p;
  return cudaSuccess;
}

int split_at(int n) {
  int n1 = ((n / 2) + kLeafN - 1) / kLeafN * kLeafN;
  if (n1 >= n) n1 = n - kLeafN;
  if (n1 <= 0) n1 = n / 2;
  return n1;
}

// C = alpha op(A) op(B) + beta C without split-K (the only GEMM scratch)
cudaError_t gemm_nosplit(int ta, int tb, int M, int N, int K, double alpha, const double* A, int64_t lda,
                         const double* B, int64_t ldb, double beta, double* C, int64_t ldc, int tri,
                         cudaStream_t st) {
  GemmArgs g;
  g.M = M;
  g.N = N;
  g.K = K;
  g.transA = ta;
  g.transB = tb;
  g.A = A;
  g.lda = lda;
  g.B = B;
  g.ldb = ldb;
  g.C = C;
  g.ldc = ldc;
  g.alpha = alpha;
  g.beta = beta;
  g.tri = tri;
  g.splitk = 1;
  return dgemm(g, Scratch{}, st);
}

// Y = X L^{-T}; the inverse of L's diagonal block k is at dinv + (k0 + k) * 4096
cudaError_t trsm_rlt_static(int m, int n, const double* L, int64_t ldl, double* X, int64_t ldx, double* Y,
                            int64_t ldy, const double* dinv, int k0, cudaStream_t st) {
  if (n <= kLeafN)
    return gemm_nosplit(0, 1, m, n, n, 1.0, X, ldx, dinv + static_cast<int64_t>(k0) * 4096, kLeafN, 0.0, Y, ldy, 0,
                        st);
  const int n1 = split_at(n), n2 = n - n1;
  cudaError_t e = trsm_rlt_static(m, n1, L, ldl, X, ldx, Y, ldy, dinv, k0, st);
  if (e != cudaSuccess) return e;
  e = gemm_nosplit(0, 1, m, n2, n1, -1.0, Y, ldy, L + n1, ldl, 1.0, X + static_cast<int64_t>(n1) * ldx, ldx, 0, st);
  if (e != cudaSuccess) return e;
  return trsm_rlt_static(m, n2, L + n1 + static_cast<int64_t>(n1) * ldl, ldl, X + static_cast<int64_t>(n1) * ldx,
                         ldx, Y + static_cast<int64_t>(n1) * ldy, ldy, dinv, k0 + n1 / kLeafN, st);
}

cudaError_t potrf_static(int n, double* A, int64_t lda, int off, double* tmp, double* dinv, int* info,
                         cudaStream_t st) {
  if (n <= kLeafN)
    return potrf_leaf(n, A, lda, 0, 1, info, off, dinv + static_cast<int64_t>(off / kLeafN) * 4096, 0, st);
  const int n1 = split_at(n), n2 = n - n1;
  cudaError_t e = potrf_static(n1, A, lda, off, tmp, dinv, info, st);
  if (e != cudaSuccess) return e;
  const int64_t ldt = (n2 + 1) / 2 * 2;
  double* a21 = A + n1;
  e = scale_copy(n2, n1, 1.0, a21, lda, 0, tmp, ldt, 0, 1, 0.0, st);
  if (e != cudaSuccess) return e;
  e = trsm_rlt_static(n2, n1, A, lda, tmp, ldt, a21, lda, dinv, off / kLeafN, st);
  if (e != cudaSuccess) return e;
  e = gemm_nosplit(0, 1, n2, n2, n1, -1.0, a21, lda, a21, lda, 1.0, A + n1 + static_cast<int64_t>(n1) * lda, lda, 1,
                   st);
  if (e != cudaSuccess) return e;
  return potrf_static(n2, A + n1 + static_cast<int64_t>(n1) * lda, lda, off + n1, tmp, dinv, info, st);
}

}  // namespace
}  // namespace zolo

extern "C" int zolo_dpotrf_noalloc(int n, double* dA, int64_t lda, void* stream) {
  if (n < 0 || n > ZOLO_NOALLOC_MAX_N) return -1;
  if (lda < (n > 1 ? n : 1)) return -3;
  if (n == 0) return 0;
  if (!dA) return -2;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  zolo::DevicePtrs p;
  cudaError_t e = zolo::device_ptrs(&p);
  if (e != cudaSuccess) return -1000 - static_cast<int>(e);
  double* tmp = p.scratch;
  double* dinv = p.scratch + zolo::kTmpDoubles;
  e = cudaMemsetAsync(p.info, 0, sizeof(int), st);  // INFO must start at zero on every call
  if (e == cudaSuccess) e = zolo::potrf_static(n, dA, lda, 0, tmp, dinv, p.info, st);
  int info = 0;
  if (e == cudaSuccess) e = cudaMemcpyAsync(&info, p.info, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return -1000 - static_cast<int>(e);
  return info;
}
