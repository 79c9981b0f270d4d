// Shared device helpers for the FP64 kernels (sm_100a).
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#define ZDEV __device__ __forceinline__

namespace zolo {

// 16-byte async global->shared copy; src_bytes in {0, 8, 16}, the rest is zero-filled.
ZDEV void cp_async16(void* smem, const void* gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
// 8-byte async global->shared copy; src_bytes in {0, 8}.
ZDEV void cp_async8(void* smem, const void* gmem, int src_bytes) {
  unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
ZDEV void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
ZDEV void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// D(16x8) += A(16x8) * B(8x8), FP64 tensor core (DMMA).
// Fragment layout (PTX ISA, mma.m16n8k8 .f64): g = lane/4, t = lane%4
//   a0=(g,t) a1=(g+8,t) a2=(g,t+4) a3=(g+8,t+4);  b0=(t,g) b1=(t+4,g)
//   c0=(g,2t) c1=(g,2t+1) c2=(g+8,2t) c3=(g+8,2t+1)
ZDEV void dmma_16x8x8(double (&d)[4], const double (&a)[4], const double (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+d"(d[0]), "+d"(d[1]), "+d"(d[2]), "+d"(d[3])
      : "d"(a[0]), "d"(a[1]), "d"(a[2]), "d"(a[3]), "d"(b[0]), "d"(b[1]));
}

ZDEV double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Kernel attributes (cudaFuncSetAttribute) and device properties are per device: these
// helpers apply / compute them once for each device the library launches on.
constexpr int kMaxDevices = 64;
template <class F>
inline cudaError_t once_per_device(std::atomic<int> (&state)[kMaxDevices], F&& set) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return set();
  if (state[dev].load(std::memory_order_acquire) == 1) return cudaSuccess;
  e = set();
  if (e == cudaSuccess) state[dev].store(1, std::memory_order_release);
  return e;
}
// cache[device] holds compute() (a positive value) after the first call on that device.
template <class F>
inline int per_device_value(std::atomic<int> (&cache)[kMaxDevices], F&& compute) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return compute();
  int v = cache[dev].load(std::memory_order_acquire);
  if (v <= 0) {
    v = compute();
    cache[dev].store(v, std::memory_order_release);
  }
  return v;
}

// Device status word: kernels record the first error code here (never trap).
ZDEV void set_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

}  // namespace zolo
