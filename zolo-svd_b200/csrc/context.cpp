#include "context.h"

namespace zolo {

Context::Context(int device) : device_(device) {
  ck(cudaSetDevice(device));
  // Blocking streams: work on them is ordered after work already queued on the
  // legacy default stream (where a caller typically produced the inputs), as on a
  // cuBLAS handle's default stream.  A non-blocking stream would let a solve read
  // its input before the producing kernel on the default stream has finished.
  ck(cudaStreamCreateWithFlags(&own_stream_, cudaStreamDefault));
  stream_ = own_stream_;
  int lo = 0, hi = 0;
  ck(cudaDeviceGetStreamPriorityRange(&lo, &hi));
  ck(cudaStreamCreateWithPriority(&side_, cudaStreamDefault, hi));
  for (auto& e : ev_) ck(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
}

Context::~Context() {
  release_all();
  for (auto& e : ev_)
    if (e) cudaEventDestroy(e);
  if (side_) cudaStreamDestroy(side_);
  if (own_stream_) cudaStreamDestroy(own_stream_);
}

void Context::drop_graphs() {
  for (auto& kv : graphs)
    if (kv.second.exec) cudaGraphExecDestroy(kv.second.exec);
  graphs.clear();
}

void Context::free_retired() {
  for (void* p : retired_) cudaFree(p);
  retired_.clear();
}

void* Context::pool_take(size_t bytes, size_t* got) {
  {
    std::lock_guard<std::mutex> lk(pool_mu_);
    auto it = pool_.lower_bound(bytes);
    if (it != pool_.end() && it->first <= 2 * bytes) {
      void* p = it->second;
      *got = it->first;
      pool_.erase(it);
      return p;
    }
  }
  const size_t b = (bytes + 65535) / 65536 * 65536;
  void* p = nullptr;
  ck(cudaMalloc(&p, b));
  *got = b;
  return p;
}

void Context::pool_give(void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(pool_mu_);
  pool_.emplace(bytes, p);
}

void Context::sync_all() {
  cudaStreamSynchronize(stream_);
  cudaStreamSynchronize(side_);
  for (auto& w : workers) {
    cudaStreamSynchronize(w->stream_);
    cudaStreamSynchronize(w->side_);
  }
}

void Context::sync_and_free_retired() {
  bool any = !retired_.empty();
  for (auto& w : workers) any = any || !w->retired_.empty();
  if (!any) return;
  ck(cudaStreamSynchronize(stream_));
  ck(cudaStreamSynchronize(side_));
  for (auto& w : workers) {
    ck(cudaStreamSynchronize(w->stream_));
    ck(cudaStreamSynchronize(w->side_));
    w->free_retired();
  }
  free_retired();
}

void Context::release_all() {
  workers.clear();
  if (stream_) cudaStreamSynchronize(stream_);
  if (side_) cudaStreamSynchronize(side_);
  drop_graphs();
  free_retired();
  for (auto& kv : bufs_) cudaFree(kv.second.first);
  bufs_.clear();
  {
    std::lock_guard<std::mutex> lk(pool_mu_);
    for (auto& kv : pool_) cudaFree(kv.second);
    pool_.clear();
  }
  ++alloc_gen_;
  if (splitk_.ptr) cudaFree(splitk_.ptr);
  if (splitk_side_.ptr) cudaFree(splitk_side_.ptr);
  splitk_ = Scratch{};
  splitk_side_ = Scratch{};
}

void* Context::grow(const std::string& name, size_t bytes) {
  auto it = bufs_.find(name);
  if (it != bufs_.end() && it->second.second >= bytes) return it->second.first;
  if (it != bufs_.end()) {
    // kernels queued on this context's streams (or captured nodes) may still use the old
    // block: it is kept alive and freed once they have run (free_retired after a
    // synchronization), instead of a cudaFree here, which would wait for the whole device
    // while other worker contexts are running
    retired_.push_back(it->second.first);
    bufs_.erase(it);
    ++alloc_gen_;
    ++reallocs;
  }
  void* p = nullptr;
  const size_t b = bytes < 256 ? 256 : bytes;
  ck(cudaMalloc(&p, b));
  bufs_[name] = {p, b};
  return p;
}

double* Context::buf(const std::string& name, size_t elems) {
  return static_cast<double*>(grow(name, elems * sizeof(double)));
}

int* Context::ibuf(const std::string& name, size_t elems) {
  return static_cast<int*>(grow(name, elems * sizeof(int)));
}

void Context::ensure_splitk(size_t bytes, bool side) {
  Scratch& s = side ? splitk_side_ : splitk_;
  if (s.bytes >= bytes) return;
  if (s.ptr) {
    retired_.push_back(s.ptr);  // freed by free_retired, as in grow
    ++alloc_gen_;
    ++reallocs;
  }
  s.ptr = nullptr;
  s.bytes = 0;
  void* p = nullptr;
  ck(cudaMalloc(&p, bytes));
  s.ptr = static_cast<double*>(p);
  s.bytes = bytes;
}

cudaEvent_t Profiler::take() {
  if (!pool.empty()) {
    cudaEvent_t e = pool.back();
    pool.pop_back();
    return e;
  }
  cudaEvent_t e;
  ck(cudaEventCreate(&e));
  return e;
}

void Profiler::begin(int cls, double fl, cudaStream_t st, Rec* r) {
  if (serialize) ck(cudaDeviceSynchronize());
  r->a = take();
  r->b = take();
  r->cls = cls;
  r->flops = fl;
  ck(cudaEventRecord(r->a, st));
}

void Profiler::end(Rec& r, cudaStream_t st) {
  ck(cudaEventRecord(r.b, st));
  recs.push_back(r);
  if (serialize) ck(cudaEventSynchronize(r.b));
}

void Profiler::collect() {
  for (auto& r : recs) {
    ck(cudaEventSynchronize(r.b));
    float t = 0.f;
    ck(cudaEventElapsedTime(&t, r.a, r.b));
    launches[r.cls] += 1;
    ms[r.cls] += t;
    flops[r.cls] += r.flops;
    pool.push_back(r.a);
    pool.push_back(r.b);
  }
  recs.clear();
}

void Profiler::reset() {
  collect();
  for (int i = 0; i < kClasses; ++i) launches[i] = ms[i] = flops[i] = 0;
}

Profiler::~Profiler() {
  for (auto& r : recs) {
    cudaEventDestroy(r.a);
    cudaEventDestroy(r.b);
  }
  for (auto e : pool) cudaEventDestroy(e);
}

double* Context::dscal() { return buf("__scal", 64); }
double* Context::dpartial() { return buf("__partial", 4096); }
int* Context::dinfo() { return ibuf("__info", 1024); }

int* Context::oz_status_word() {
  const bool fresh = bufs_.find("oz_status") == bufs_.end();
  int* p = ibuf("oz_status", 1);
  if (fresh) ck(cudaMemsetAsync(p, 0, sizeof(int), stream_));
  return p;
}

}  // namespace zolo
