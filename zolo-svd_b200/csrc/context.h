// Per-handle state: device, stream, cached device workspace, statistics.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include <memory>

#include "batch_plan.h"
#include "kernels.h"

namespace zolo {

struct Stats {
  int iterations = 0;
  int qr_iterations = 0;
  int chol_iterations = 0;
  int info = 0;
  double alpha = 0.0, beta = 0.0, last_err = 0.0;
  double ms_total = 0.0, ms_bounds = 0.0, ms_iter = 0.0, ms_h = 0.0;
  double flops = 0.0;
  int64_t launches = 0;
  double con[16] = {0};
  double err[16] = {0};
  int branch[16] = {0};  // 1 = QR, 2 = Cholesky, 3 = Newton-Schulz
  double flops_exec_delta = 0.0;  // executed minus canonical flops (shared-QR form: < 0)
  int ns_steps = 0;
  int ns_finish = 0;  // 1 if Newton-Schulz steps ended the iteration
  double ms_step[16] = {0};  // device ms of each iteration
  double ms_finish = 0.0;    // device ms of the Newton-Schulz finish (check included)
  int terms[16] = {0};       // Zolotarev terms of each iteration
};

// Optional per-kernel-class timing with CUDA events recorded around launches on
// their own stream: 0 = DMMA GEMM (general shapes, K > 64), 1 = Householder panel,
// 2 = Cholesky leaf, 3 = GEMM with M <= 32, 4 = GEMM with N <= 64,
// 5 = GEMM rank-k update (K <= 64), 6 = GEMM lower-triangle output, 7 = FP64 product
// emulated on the INT8 tensor cores (the ozgemm kernel), 8 = GEMM with 64 < K <= 256 (the
// Householder block-reflector updates; class 0 is then K > 256), 9 = the emulated
// products' splitting into digit planes (row maxima and slices).
struct Profiler {
  static constexpr int kClasses = 10;
  bool on = false;
  // each launch timed alone: the device is synchronized before its first event, so that work
  // overlapping on other streams (the look-ahead panels) is not counted in its time
  bool serialize = false;
  struct Rec {
    cudaEvent_t a, b;
    int cls;
    double flops;
  };
  std::vector<Rec> recs;
  std::vector<cudaEvent_t> pool;
  double launches[kClasses] = {}, ms[kClasses] = {}, flops[kClasses] = {};
  cudaEvent_t take();
  void begin(int cls, double fl, cudaStream_t st, Rec* r);
  void end(Rec& r, cudaStream_t st);
  void collect();  // synchronizes the recorded events and folds them into the totals
  void reset();
  ~Profiler();
};

// Thrown inside the library on a CUDA error; converted to an INFO code at the C-ABI.
struct CudaFailure {
  cudaError_t err;
};

inline void ck(cudaError_t e) {
  if (e != cudaSuccess) throw CudaFailure{e};
}

class Context {
 public:
  explicit Context(int device);
  ~Context();

  int device() const { return device_; }
  cudaStream_t stream() const { return stream_; }
  void set_stream(cudaStream_t s) { stream_ = s ? s : own_stream_; }
  // high-priority stream for latency-bound work overlapped with the main stream
  cudaStream_t side_stream() const { return side_; }
  cudaEvent_t event(int i) const { return ev_[i]; }

  // Named cached device buffer of at least `elems` doubles (grow-only).
  double* buf(const std::string& name, size_t elems);
  int* ibuf(const std::string& name, size_t elems);
  // split-K partial sums; GEMMs on the side stream have their own
  Scratch& splitk(bool side = false) { return side ? splitk_side_ : splitk_; }
  void ensure_splitk(size_t bytes, bool side = false);
  void release_all();

  Stats stats;
  Profiler prof;
  std::mutex mu;
  // Zolo-PD QR iterations: 1 = one QR of X shared by the r terms (default),
  // 0 = one QR of the stacked [X; sqrt(c_j) I] per term (mpdgeqrf.f form).
  int zolo_shared_qr = 1;
  // Zolo-PD stopping: 0 = reference rule, 1 = Newton-Schulz finish once ||X^T X - I|| is small.
  int zolo_ns_finish = 0;
  // Zolo-PD Cholesky iterations: 0 = two triangular solves per term (zolochol.f90),
  // 1 = explicit inverses summed into S, then one Z = X S.
  int zolo_chol_inverse = 0;
  // zolo_polar's bounds: 0 = beta = 1/(sqrt(n) ||R^-1||_1) (test_zolodrv1.f90), 1 = 1/||R^-1||_F.
  int zolo_beta_frob = 0;
  // Zolo-PD term counts: 0 = rk in every iteration, 1 = planned per iteration (r <= rk) by cost.
  int zolo_term_plan = 0;
  // Mixed form: 0 = every product on the FP64 DMMA GEMM; 1 = the large products of the
  // Cholesky iterations, the Newton-Schulz finish and Q, H run on the INT8-emulated GEMM
  // (ozgemm, oz_slices digit planes); the bounds and the QR iterations stay on DMMA.
  int zolo_mixed = 0;
  // PZOLOPD1 entries: 1 = compute ALPHA, BETA from A (zolo_polar) instead of the caller's
  int zolo_own_bounds = 0;
  // zolo_polar's bounds: 1 = alpha lowered to a guaranteed bound of ||A||_2 (BOUNDS_NORM2)
  int zolo_norm2 = 0;
  // diagnostic: k + 1 = the Cholesky step of iteration k reports failure (0 = off)
  int inject_chol_fail = 0;
  // diagnostic: 1 = the batched solver's scheduled run sees its first member's last error
  // above the stopping tolerance (0 = off)
  int inject_batch_err = 0;
  // eigensolver: nodes of at least this size split with the Zolo-PD fast form (r = 8, every
  // cost option), smaller ones with QDWH (batched per level); 0 = QDWH for every node
  int eig_zolo_min = 4096;
  // batched solver: 1 = each bucket's iterations, H and unpacking run as one CUDA graph
  // launch from a host-computed schedule, 2 = the same launches issued eagerly, 0 = a
  // host-synchronized loop
  int batch_graph = 1;
  // batched solver: cost model of its bucket plan, and the worker contexts (own stream and
  // workspace each) its buckets run on concurrently
  BatchCostModel batch_model;
  std::vector<std::unique_ptr<Context>> workers;
  int oz_slices = 8;
  // digit planes of the products gemm() routes to ozgemm right now (0 = none); set by OzScope
  int oz_active = 0;

  // A buffer that must grow is replaced without a synchronization and the old block is kept
  // alive (retired) until free_retired(), called once the work that may use it has run (the
  // end of a bucket's solve, or sync_and_free_retired() after a library call, which also
  // covers the worker contexts).  alloc_gen changes whenever a block is replaced or freed,
  // which invalidates cached graphs; `capturing` marks a stream capture in progress.
  bool capturing = false;
  uint64_t alloc_gen() const { return alloc_gen_; }
  void free_retired();
  void sync_and_free_retired();
  // waits for this context's and its workers' streams (errors ignored: used on exit paths)
  void sync_all();
  // Pool of device blocks for call-scoped matrices (the eigensolver's nodes): pool_take returns
  // a free block of at least `bytes` (and at most twice that) or a new one, its size in *got;
  // pool_give puts it back.  Blocks are freed by release_all only.  Thread-safe.
  void* pool_take(size_t bytes, size_t* got);
  void pool_give(void* p, size_t bytes);
  int64_t reallocs = 0;  // buffers replaced by larger ones (diagnostic)
  // cached executable graphs of the batched solver, by bucket shape and schedule
  struct CachedGraph {
    cudaGraphExec_t exec = nullptr;
    uint64_t gen = 0;
    int64_t launches = 0;
    bool seen = false;  // the shape ran once eagerly (its workspace exists)
  };
  std::map<std::string, CachedGraph> graphs;
  void drop_graphs();

  // small device scalars / partial sums
  double* dscal();     // 64 doubles
  double* dpartial();  // 4096 doubles
  int* dinfo();        // 1024 ints
  int* oz_status_word();  // status of the INT8-emulated products (zeroed when allocated)

 private:
  int device_;
  cudaStream_t stream_ = nullptr, own_stream_ = nullptr, side_ = nullptr;
  cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
  std::map<std::string, std::pair<void*, size_t>> bufs_;
  Scratch splitk_, splitk_side_;
  std::vector<void*> retired_;
  std::multimap<size_t, void*> pool_;
  std::mutex pool_mu_;
  uint64_t alloc_gen_ = 0;
  void* grow(const std::string& name, size_t bytes);
};

// Device time between construction and stop() on one stream (CUDA events; stop() waits).
struct EventTimer {
  cudaEvent_t a = nullptr, b = nullptr;
  cudaStream_t s;
  explicit EventTimer(cudaStream_t st) : s(st) {
    ck(cudaEventCreate(&a));
    ck(cudaEventCreate(&b));
    ck(cudaEventRecord(a, s));
  }
  double stop() {
    ck(cudaEventRecord(b, s));
    ck(cudaEventSynchronize(b));
    float ms = 0.f;
    ck(cudaEventElapsedTime(&ms, a, b));
    return ms;
  }
  EventTimer(const EventTimer&) = delete;
  EventTimer& operator=(const EventTimer&) = delete;
  ~EventTimer() {
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
  }
};

// Routes the large products of gemm() to the INT8-emulated GEMM while in scope (when the
// handle's mixed form is on), and restores the previous routing on exit.
struct OzScope {
  Context& c;
  int saved;
  OzScope(Context& ctx, bool on) : c(ctx), saved(ctx.oz_active) { c.oz_active = on ? c.oz_slices : 0; }
  ~OzScope() { c.oz_active = saved; }
};

}  // namespace zolo
