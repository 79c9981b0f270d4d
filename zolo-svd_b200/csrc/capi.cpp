// extern "C" boundary: handles, reference-named host-array entry points
// (1x1-grid descriptors, workspace queries, INFO codes) and the device-pointer
// hot path.  See include/zolo_b200.h for the contract of every symbol.
#include "../../include/zolo_b200.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <vector>

#include "coeff.h"
#include "context.h"
#include "eig.h"
#include "linalg.h"
#include "polar.h"

struct zolo_handle_s {
  explicit zolo_handle_s(int dev) : ctx(dev) {}
  zolo::Context ctx;
  zolo::BatchStats last_batch;  // the last zolo_qdwh_batch_dev call
};

namespace {

using zolo::Context;
using zolo::CudaFailure;

constexpr int kCudaBase = -1000;

// Makes the handle's device current for the call and restores the caller's current
// device on every exit path.
struct DeviceGuard {
  int saved = -1;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&saved) != cudaSuccess) saved = -1;
    if (saved != dev) zolo::ck(cudaSetDevice(dev));
  }
  ~DeviceGuard() {
    int cur = -1;
    if (saved >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != saved) cudaSetDevice(saved);
  }
};

template <class F>
int guarded(zolo_handle_t h, F&& f) {
  if (!h) return -999;
  std::lock_guard<std::mutex> lk(h->ctx.mu);
  try {
    DeviceGuard dg(h->ctx.device());
    const int r = f(h->ctx);
    h->ctx.sync_and_free_retired();  // blocks replaced while the call ran
    return r;
  } catch (const CudaFailure& e) {
    return kCudaBase - static_cast<int>(e.err);
  } catch (const std::bad_alloc&) {
    return kCudaBase - static_cast<int>(cudaErrorMemoryAllocation);
  }
}

std::mutex g_default_mu;
zolo_handle_t g_default = nullptr;

// 1x1-grid descriptor check; returns 0 or the reference-style INFO for argument `pos`.
int check_desc(const int* desc, int m, int n, int pos) {
  if (!desc) return -(pos * 100 + 1);
  if (desc[0] != 1) return -(pos * 100 + 1);
  if (desc[2] < m) return -(pos * 100 + 3);
  if (desc[3] < n) return -(pos * 100 + 4);
  if (desc[6] != 0) return -(pos * 100 + 7);
  if (desc[7] != 0) return -(pos * 100 + 8);
  if (desc[8] < std::max(1, desc[2])) return -(pos * 100 + 9);
  return 0;
}

// reference workspace minimums on a 1x1 grid (pqdwhfacs.f90:262-278)
void qdwh_lwork(int m, int n, const int* desca, const int* descw, double* lwin, double* lwin2) {
  const int nba = desca ? std::max(desca[5], 1) : 64;
  const int nbw = descw ? std::max(descw[5], 1) : nba;
  const double gecon = 5.0 * n + nba;                                   // PDGECON LWORK
  const double geqrf = static_cast<double>(nbw) * (3.0 * n + nbw);      // PDGEQRF LWORK for 2N x N
  *lwin = std::max(std::max(gecon + 1.0, 2.0 * n * static_cast<double>(n)), 2.0 * m * static_cast<double>(n));
  *lwin2 = std::max(geqrf + 1.0, static_cast<double>(m) * n);
}

struct DevView {
  double* p;
};

// PZOLOPD1 semantics with ZOLO_OPT_OWN_BOUNDS: the caller's ALPHA and BETA are replaced by
// the library's own (alpha = ||A||_F, beta from the QR of A/alpha) and that QR is reused by
// the first iteration.  The polar factor does not depend on the scaling of A, so Q is the
// same to rounding; SYM = 'S' keeps the caller's bounds.
int zolo_pd_entry(Context& c, char sym, int rk, int m, int n, double alpha, double beta, const double* dA, int64_t lda,
                  double* dQ, int64_t ldq, double* dH, int64_t ldh) {
  if (c.zolo_own_bounds && !(sym == 'S' || sym == 's') && m >= n && rk >= 1 && rk <= 8)
    return zolo::zolo_polar(c, rk, m, n, dA, lda, dQ, ldq, dH, ldh);
  return zolo::zolo_pd(c, sym, rk, m, n, alpha, beta, dA, lda, dQ, ldq, dH, ldh);
}

// One algorithm option of a handle (zolo_set_option); 0, -1 unknown option, -3 bad value.
int set_option(Context& c, int option, int value) {
  switch (option) {
    case ZOLO_OPT_SHARED_QR:
      c.zolo_shared_qr = value != 0;
      return 0;
    case ZOLO_OPT_NS_FINISH:
      c.zolo_ns_finish = value != 0;
      return 0;
    case ZOLO_OPT_CHOL_INVERSE:
      c.zolo_chol_inverse = value != 0;
      return 0;
    case ZOLO_OPT_BETA_FROB:
      c.zolo_beta_frob = value != 0;
      return 0;
    case ZOLO_OPT_TERM_PLAN:
      c.zolo_term_plan = value != 0;
      return 0;
    case ZOLO_OPT_MIXED:
      if (value < 0 || value > 1) return -3;
      c.zolo_mixed = value;
      return 0;
    case ZOLO_OPT_MIXED_SLICES:
      if (value < 6 || value > 8) return -3;
      c.oz_slices = value;
      return 0;
    case ZOLO_OPT_OWN_BOUNDS:
      c.zolo_own_bounds = value != 0;
      return 0;
    case ZOLO_OPT_INJECT_CHOL_FAIL:
      if (value < 0) return -3;
      c.inject_chol_fail = value;
      return 0;
    case ZOLO_OPT_NORM2_BOUND:
      c.zolo_norm2 = value != 0;
      return 0;
    case ZOLO_OPT_BATCH_GRAPH:
      if (value < 0 || value > 2) return -3;
      c.batch_graph = value;
      return 0;
    case ZOLO_OPT_INJECT_BATCH_ERR:
      c.inject_batch_err = value != 0;
      return 0;
    case ZOLO_OPT_EIG_ZOLO_MIN:
      if (value < 0) return -3;
      c.eig_zolo_min = value;
      return 0;
    default:
      return -1;
  }
}

// Options of the default handle from the environment, so that callers of the reference's
// entry points (pzolopd1_, pqdwhfacs_, ...) select them without a code change: ZOLO_FAST=1
// turns on every cost option (shared QR, Newton-Schulz finish, explicit-inverse Cholesky,
// Frobenius beta, term plan, own bounds); ZOLO_OPT_<NAME>=<value> sets one option and
// overrides ZOLO_FAST.  Unparsable or out-of-range values are ignored.
void apply_env_options(Context& c) {
  auto get = [](const char* name, int* v) {
    const char* s = std::getenv(name);
    if (!s || !*s) return false;
    char* end = nullptr;
    const long x = std::strtol(s, &end, 10);
    if (end == s || *end != '\0') return false;
    *v = static_cast<int>(x);
    return true;
  };
  int v = 0;
  if (get("ZOLO_FAST", &v) && v) {
    for (int o : {ZOLO_OPT_SHARED_QR, ZOLO_OPT_NS_FINISH, ZOLO_OPT_CHOL_INVERSE, ZOLO_OPT_BETA_FROB,
                  ZOLO_OPT_TERM_PLAN, ZOLO_OPT_OWN_BOUNDS})
      set_option(c, o, 1);
  }
  const std::pair<const char*, int> names[] = {
      {"ZOLO_OPT_SHARED_QR", ZOLO_OPT_SHARED_QR},   {"ZOLO_OPT_NS_FINISH", ZOLO_OPT_NS_FINISH},
      {"ZOLO_OPT_CHOL_INVERSE", ZOLO_OPT_CHOL_INVERSE}, {"ZOLO_OPT_BETA_FROB", ZOLO_OPT_BETA_FROB},
      {"ZOLO_OPT_TERM_PLAN", ZOLO_OPT_TERM_PLAN},   {"ZOLO_OPT_MIXED", ZOLO_OPT_MIXED},
      {"ZOLO_OPT_MIXED_SLICES", ZOLO_OPT_MIXED_SLICES}, {"ZOLO_OPT_OWN_BOUNDS", ZOLO_OPT_OWN_BOUNDS},
      {"ZOLO_OPT_NORM2_BOUND", ZOLO_OPT_NORM2_BOUND},   {"ZOLO_OPT_BATCH_GRAPH", ZOLO_OPT_BATCH_GRAPH},
      {"ZOLO_OPT_EIG_ZOLO_MIN", ZOLO_OPT_EIG_ZOLO_MIN}};
  for (const auto& nm : names)
    if (get(nm.first, &v)) set_option(c, nm.second, v);
}

int run_qdwh_host(char sym, int m, int n, double sigma, const double* a, int ia, int ja, const int* desca, double* q,
                  int iq, int jq, const int* descq, double* work, int lwork, const int* descw, double* work2,
                  int lwork2, char polar, bool zolopd_mode) {
  if (m < n) return -1;
  const bool query = (lwork == -1 || lwork2 == -1);
  // argument positions differ between PQDWHFACS and ZOLOPD (no SYM)
  const int off = zolopd_mode ? -1 : 0;
  if (m == 0 || n == 0) return 0;
  double lwin, lwin2;
  qdwh_lwork(m, n, desca, descw, &lwin, &lwin2);
  if (work) {  // WORK(1), WORK(2) are always set, as pqdwhfacs.f90:279-280 does
    work[0] = lwin;
    work[1] = lwin2;
  }
  if (query) return 0;
  if (ia != 1) return -(6 + off);
  if (ja != 1) return -(7 + off);
  if (int e = check_desc(desca, m, n, 8 + off)) return e;
  if (iq != 1) return -(10 + off);
  if (jq != 1) return -(11 + off);
  if (int e = check_desc(descq, m, n, 12 + off)) return e;
  if (lwork < lwin) return -12;
  if (lwork2 < lwin2) return -16;
  zolo_handle_t h = nullptr;
  if (int e = zolo_default_handle(&h)) return e;
  const bool want_h = (polar == 'T' || polar == 't');
  return guarded(h, [&](Context& c) -> int {
    // device copies of the caller's arrays: handle workspace, allocated once and reused
    const int64_t ld = m;
    const DevView dA{c.buf("host_a", static_cast<size_t>(m) * n)}, dQ{c.buf("host_q", static_cast<size_t>(m) * n)};
    const DevView dH{want_h ? c.buf("host_h", static_cast<size_t>(n) * n) : nullptr};
    zolo::ck(cudaMemcpy2DAsync(dA.p, ld * sizeof(double), a, desca[8] * sizeof(double), m * sizeof(double), n,
                               cudaMemcpyHostToDevice, c.stream()));
    zolo::QdwhOpts o;
    o.sym = zolopd_mode ? 'N' : sym;
    o.sigma = sigma;
    o.bounds = zolopd_mode ? zolo::BOUNDS_ZOLOPD : zolo::BOUNDS_PQDWHFACS;
    o.maxit = zolopd_mode ? -1 : 12;
    o.left_solve = zolopd_mode;
    const int info = zolo::qdwh(c, m, n, dA.p, ld, dQ.p, ld, want_h ? dH.p : nullptr, n, o);
    zolo::ck(cudaMemcpy2DAsync(q, descq[8] * sizeof(double), dQ.p, ld * sizeof(double), m * sizeof(double), n,
                               cudaMemcpyDeviceToHost, c.stream()));
    if (want_h && work2)
      zolo::ck(cudaMemcpy2DAsync(work2, descq[8] * sizeof(double), dH.p, n * sizeof(double), n * sizeof(double), n,
                                 cudaMemcpyDeviceToHost, c.stream()));
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return info;
  });
}

int run_zolo_host(char sym, int rk, int m, int n, double alpha, double beta, const double* as, int ia, int ja,
                  const int* desca, double* q, int iq, int jq, const int* descq) {
  if (rk < 1 || rk > 8) return -2;
  if (m < n) return -3;
  if (m == 0 || n == 0) return 0;
  if (!(alpha > 0.0)) return -5;
  if (!(beta > 0.0)) return -6;
  if (ia != 1) return -8;
  if (ja != 1) return -9;
  if (int e = check_desc(desca, m, n, 10)) return e;
  if (iq != 1) return -12;
  if (jq != 1) return -13;
  if (int e = check_desc(descq, m, n, 14)) return e;
  zolo_handle_t h = nullptr;
  if (int e = zolo_default_handle(&h)) return e;
  return guarded(h, [&](Context& c) -> int {
    // device copies of the caller's arrays: handle workspace, allocated once and reused
    const int64_t ld = m;
    const DevView dA{c.buf("host_a", static_cast<size_t>(m) * n)}, dQ{c.buf("host_q", static_cast<size_t>(m) * n)};
    zolo::ck(cudaMemcpy2DAsync(dA.p, ld * sizeof(double), as, desca[8] * sizeof(double), m * sizeof(double), n,
                               cudaMemcpyHostToDevice, c.stream()));
    const int info = zolo_pd_entry(c, sym, rk, m, n, alpha, beta, dA.p, ld, dQ.p, ld, nullptr, 0);
    zolo::ck(cudaMemcpy2DAsync(q, descq[8] * sizeof(double), dQ.p, ld * sizeof(double), m * sizeof(double), n,
                               cudaMemcpyDeviceToHost, c.stream()));
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return info;
  });
}

inline bool upper(char c) { return c == 'T' || c == 't' || c == 'C' || c == 'c'; }

}  // namespace

extern "C" {

const char* zolo_version(void) { return "zolo-b200 0.1 (sm_100a, FP64 DMMA)"; }

int zolo_create(int device, zolo_handle_t* handle) {
  if (!handle) return -2;
  try {
    *handle = new zolo_handle_s(device);
    return 0;
  } catch (const CudaFailure& e) {
    *handle = nullptr;
    return kCudaBase - static_cast<int>(e.err);
  }
}

int zolo_destroy(zolo_handle_t handle) {
  if (!handle) return 0;
  {
    std::lock_guard<std::mutex> lk(g_default_mu);
    if (handle == g_default) g_default = nullptr;
  }
  delete handle;
  return 0;
}

int zolo_default_handle(zolo_handle_t* handle) {
  std::lock_guard<std::mutex> lk(g_default_mu);
  if (!g_default) {
    int dev = 0;
    if (const char* s = std::getenv("ZOLO_DEVICE")) dev = std::atoi(s);
    const int e = zolo_create(dev, &g_default);
    if (e) return e;
    apply_env_options(g_default->ctx);
  }
  *handle = g_default;
  return 0;
}

int zolo_set_stream(zolo_handle_t h, void* s) {
  return guarded(h, [&](Context& c) {
    c.set_stream(static_cast<cudaStream_t>(s));
    return 0;
  });
}

int zolo_release_workspace(zolo_handle_t h) {
  return guarded(h, [&](Context& c) {
    c.release_all();
    return 0;
  });
}

int zolo_panel_cluster_size(int m, int w) { return zolo::qr_panel_config(m, w); }

int zolo_profile_enable(zolo_handle_t h, int on) {
  return guarded(h, [&](Context& c) {
    c.prof.on = on != 0;
    c.prof.serialize = on == 2;
    return 0;
  });
}

int zolo_set_option(zolo_handle_t h, int option, int value) {
  return guarded(h, [&](Context& c) { return set_option(c, option, value); });
}

int zolo_get_option(zolo_handle_t h, int option, int* value) {
  if (!value) return -3;
  return guarded(h, [&](Context& c) {
    switch (option) {
      case ZOLO_OPT_SHARED_QR: *value = c.zolo_shared_qr; return 0;
      case ZOLO_OPT_NS_FINISH: *value = c.zolo_ns_finish; return 0;
      case ZOLO_OPT_CHOL_INVERSE: *value = c.zolo_chol_inverse; return 0;
      case ZOLO_OPT_BETA_FROB: *value = c.zolo_beta_frob; return 0;
      case ZOLO_OPT_TERM_PLAN: *value = c.zolo_term_plan; return 0;
      case ZOLO_OPT_MIXED: *value = c.zolo_mixed; return 0;
      case ZOLO_OPT_MIXED_SLICES: *value = c.oz_slices; return 0;
      case ZOLO_OPT_OWN_BOUNDS: *value = c.zolo_own_bounds; return 0;
      case ZOLO_OPT_INJECT_CHOL_FAIL: *value = c.inject_chol_fail; return 0;
      case ZOLO_OPT_NORM2_BOUND: *value = c.zolo_norm2; return 0;
      case ZOLO_OPT_BATCH_GRAPH: *value = c.batch_graph; return 0;
      case ZOLO_OPT_INJECT_BATCH_ERR: *value = c.inject_batch_err; return 0;
      case ZOLO_OPT_EIG_ZOLO_MIN: *value = c.eig_zolo_min; return 0;
      default: return -1;
    }
  });
}

int zolo_profile_read(zolo_handle_t h, double* out, int reset) {
  return guarded(h, [&](Context& c) {
    c.prof.collect();
    for (int k = 0; k < zolo::Profiler::kClasses; ++k) {
      out[3 * k] = c.prof.launches[k];
      out[3 * k + 1] = c.prof.ms[k];
      out[3 * k + 2] = c.prof.flops[k];
    }
    if (reset) c.prof.reset();
    return 0;
  });
}

int zolo_get_stats(zolo_handle_t h, zolo_stats_t* out) {
  if (!h || !out) return -2;
  std::lock_guard<std::mutex> lk(h->ctx.mu);
  const zolo::Stats& s = h->ctx.stats;
  out->iterations = s.iterations;
  out->qr_iterations = s.qr_iterations;
  out->chol_iterations = s.chol_iterations;
  out->info = s.info;
  out->alpha = s.alpha;
  out->beta = s.beta;
  out->last_err = s.last_err;
  out->ms_total = s.ms_total;
  out->ms_bounds = s.ms_bounds;
  out->ms_iter = s.ms_iter;
  out->ms_h = s.ms_h;
  out->flops = s.flops;
  out->launches = s.launches;
  for (int i = 0; i < 16; ++i) {
    out->con[i] = s.con[i];
    out->err[i] = s.err[i];
    out->branch[i] = s.branch[i];
  }
  out->flops_executed = s.flops + s.flops_exec_delta;
  out->ns_steps = s.ns_steps;
  out->ns_finish = s.ns_finish;
  for (int i = 0; i < 16; ++i) out->ms_step[i] = s.ms_step[i];
  out->ms_finish = s.ms_finish;
  for (int i = 0; i < 16; ++i) out->terms[i] = s.terms[i];
  return 0;
}

int zolo_compute_coeff(double con, double tol, int rk, double* coeff) {
  if (rk < 1 || rk > 8 || !coeff) return -3;
  if (!(con >= 1.0)) return -1;
  zolo::compute_coeff(con, tol, rk, coeff);
  return 0;
}

int zolo_plan_terms(double con, int rk, int m, int n, int prefactored, int* terms, int* qr_form, int maxlen,
                    int* ns_steps) {
  return zolo::plan_terms(con, rk, m, n, prefactored != 0, terms, qr_form, maxlen, ns_steps);
}

int zolo_compute_coeff_kp(double con, double tol, int rk, double* coeff) {
  if (rk < 1 || rk > 8 || !coeff) return -3;
  if (!(con > 1.0) || !std::isfinite(con)) return -1;
  zolo::compute_coeff_kp(con, tol, rk, coeff);
  return 0;
}
void zolo_mellipke(double alpha, double tol, double* k, double* e) { zolo::mellipke(alpha, tol, k, e); }
void zolo_mellipj(double u, double alpha, double tol, double* sn, double* cn, double* dn) {
  zolo::mellipj(u, alpha, tol, sn, cn, dn);
}
int zolo_choosem(double con) { return zolo::choosem(con); }
double zolo_hfunc(double x) { return zolo::hfunc(x); }
void zolo_fone_next(double con, const double* coeff, int rk, double* fone, double* next_con) {
  const double f = zolo::zolo_fone(coeff, rk);
  if (fone) *fone = f;
  if (next_con) *next_con = zolo::zolo_next_con(con, coeff, rk, f);
}

void zolo_pqdwhfacs(char sym, int m, int n, double sigma, const double* a, int ia, int ja, const int* desca,
                    double* q, int iq, int jq, const int* descq, double* work, int lwork, const int* descw,
                    double* /*tau*/, double* work2, int lwork2, int* info, char polar) {
  const int r = run_qdwh_host(sym, m, n, sigma, a, ia, ja, desca, q, iq, jq, descq, work, lwork, descw, work2,
                              lwork2, polar, false);
  if (info) *info = r;
}

void zolo_zolopd(int m, int n, double sigma, const double* a, int ia, int ja, const int* desca, double* q, int iq,
                 int jq, const int* descq, double* work, int lwork, const int* descw, double* /*tau*/, double* work2,
                 int lwork2, int* info, char polar) {
  const int r = run_qdwh_host('N', m, n, sigma, a, ia, ja, desca, q, iq, jq, descq, work, lwork, descw, work2, lwork2,
                              polar, true);
  if (info) *info = r;
}

void zolo_pzolopd1(char sym, int rk, int m, int n, double alpha, double beta, const double* as, int ia, int ja,
                   const int* desca, double* q, int iq, int jq, const int* descq, int* info, char /*polar*/) {
  const int r = run_zolo_host(sym, rk, m, n, alpha, beta, as, ia, ja, desca, q, iq, jq, descq);
  if (info) *info = r;
}

void zolo_pzolopd2(char sym, int rk, int m, int n, double alpha, double beta, const double* as, int ia, int ja,
                   const int* desca, double* q, int iq, int jq, const int* descq, int* info, char polar) {
  zolo_pzolopd1(sym, rk, m, n, alpha, beta, as, ia, ja, desca, q, iq, jq, descq, info, polar);
}

void pqdwhfacs_(const char* sym, const int* m, const int* n, const double* sigma, const double* a, const int* ia,
                const int* ja, const int* desca, double* q, const int* iq, const int* jq, const int* descq,
                double* work, const int* lwork, const int* descw, double* tau, double* work2, const int* lwork2,
                int* info, const char* polar, size_t, size_t) {
  zolo_pqdwhfacs(*sym, *m, *n, *sigma, a, *ia, *ja, desca, q, *iq, *jq, descq, work, *lwork, descw, tau, work2,
                 *lwork2, info, *polar);
}

void zolopd_(const int* m, const int* n, const double* sigma, const double* a, const int* ia, const int* ja,
             const int* desca, double* q, const int* iq, const int* jq, const int* descq, double* work,
             const int* lwork, const int* descw, double* tau, double* work2, const int* lwork2, int* info,
             const char* polar, size_t) {
  zolo_zolopd(*m, *n, *sigma, a, *ia, *ja, desca, q, *iq, *jq, descq, work, *lwork, descw, tau, work2, *lwork2, info,
              *polar);
}

void pzolopd1_(const char* sym, const int* rk, const int* m, const int* n, const double* alpha, const double* beta,
               const double* as, const int* ia, const int* ja, const int* desca, double* q, const int* iq,
               const int* jq, const int* descq, int* info, const char* polar, size_t, size_t) {
  zolo_pzolopd1(*sym, *rk, *m, *n, *alpha, *beta, as, *ia, *ja, desca, q, *iq, *jq, descq, info, *polar);
}

void pzolopd2_(const char* sym, const int* rk, const int* m, const int* n, const double* alpha, const double* beta,
               const double* as, const int* ia, const int* ja, const int* desca, double* q, const int* iq,
               const int* jq, const int* descq, int* info, const char* polar, size_t, size_t) {
  zolo_pzolopd2(*sym, *rk, *m, *n, *alpha, *beta, as, *ia, *ja, desca, q, *iq, *jq, descq, info, *polar);
}

int zolo_qdwh_dev(zolo_handle_t h, char sym, int m, int n, double sigma, const double* dA, int64_t lda, double* dQ,
                  int64_t ldq, double* dH, int64_t ldh, int bounds_mode, int maxit, int left_solve) {
  return guarded(h, [&](Context& c) {
    zolo::QdwhOpts o;
    o.sym = sym;
    o.sigma = sigma;
    o.bounds = bounds_mode ? zolo::BOUNDS_ZOLOPD : zolo::BOUNDS_PQDWHFACS;
    o.maxit = maxit;
    o.left_solve = left_solve != 0;
    return zolo::qdwh(c, m, n, dA, lda, dQ, ldq, dH, ldh, o);
  });
}

int zolo_qdwh_batch_dev(zolo_handle_t h, int count, const int* m, const int* n, const double* const* dA,
                        const int64_t* lda, double* const* dQ, const int64_t* ldq, double* const* dH,
                        const int64_t* ldh, int* info, int* iterations) {
  if (count < 0) return -2;
  if (count > 0 && (!m || !n || !dA || !lda || !dQ || !ldq || !info || (dH && !ldh))) return -3;
  return guarded(h, [&](Context& c) {
    zolo::BatchStats bs;
    const int r = zolo::qdwh_batch(c, count, m, n, dA, lda, dQ, ldq, dH, ldh, info, iterations, &bs);
    h->last_batch = bs;
    return r;
  });
}

int zolo_batch_stats(zolo_handle_t h, double* out) {
  if (!h) return -999;
  if (!out) return -2;
  std::lock_guard<std::mutex> lk(h->ctx.mu);
  {
    const zolo::BatchStats& b = h->last_batch;
    const double v[12] = {static_cast<double>(b.buckets), static_cast<double>(b.max_iterations), b.flops,
                          b.flops_useful, b.ms, b.predicted_ms, static_cast<double>(b.graph_replays),
                          static_cast<double>(b.graph_captures), static_cast<double>(b.eager_scheduled),
                          static_cast<double>(b.sync_loops), static_cast<double>(b.restarts),
                          static_cast<double>(b.resumes)};
    for (int i = 0; i < 12; ++i) out[i] = v[i];
  }
  return 0;
}

int zolo_batch_autotune(zolo_handle_t h, double* model) {
  return guarded(h, [&](Context& c) {
    zolo::batch_autotune(c);
    if (model) {
      const zolo::BatchCostModel& md = c.batch_model;
      model[0] = md.lat0;
      model[1] = md.lat1;
      model[2] = md.rate_tflops;
      model[3] = md.nhalf;
      model[4] = md.streams;
    }
    return 0;
  });
}

int zolo_batch_set_model(zolo_handle_t h, const double* model) {
  if (!model) return -2;
  if (!(model[0] >= 0.0) || !(model[1] >= 0.0) || !(model[2] > 0.0) || !(model[3] >= 0.0) || !(model[4] >= 1.0) ||
      model[4] > 16.0)
    return -2;
  return guarded(h, [&](Context& c) {
    c.batch_model = zolo::BatchCostModel{model[0], model[1], model[2], model[3], static_cast<int>(model[4])};
    return 0;
  });
}

int zolo_batch_plan(int count, const int* m, const int* n, const double* model, int max_batch, int mode,
                    int* bucket, int* mb, int* nb, double* predicted_ms) {
  if (count < 0) return -1;
  if (count > 0 && (!m || !n || !bucket || !mb || !nb)) return -2;
  if (max_batch < 1) return -5;
  for (int i = 0; i < count; ++i)
    if (n[i] < 1 || m[i] < n[i]) return -3;
  zolo::BatchCostModel md;
  if (model) md = zolo::BatchCostModel{model[0], model[1], model[2], model[3], static_cast<int>(model[4])};
  const zolo::BucketPlan p = mode == 1 ? zolo::ladder_buckets(md, count, m, n, max_batch)
                                       : zolo::plan_buckets(md, count, m, n, max_batch);
  for (size_t b = 0; b < p.members.size(); ++b) {
    for (int i : p.members[b]) bucket[i] = static_cast<int>(b);
    mb[b] = p.mb[b];
    nb[b] = p.nb[b];
  }
  if (predicted_ms) *predicted_ms = p.total_ms;
  return static_cast<int>(p.members.size());
}

int zolo_batch_schedule(int count, const double* l0, int maxit, int max_steps, int* steps, int* qr, double* table,
                        int* ucount, int* last, int* cond) {
  if (count < 0 || max_steps < 0 || !steps || (count > 0 && !l0)) return -2;
  if (maxit < 0 || maxit > 100) return -3;
  std::vector<char> done(count);
  for (int b = 0; b < count; ++b) done[b] = !(l0[b] > 0.0 && l0[b] <= 1.0);
  const zolo::QdwhSchedule S = zolo::qdwh_schedule(count, l0, done.data(), 10.0 * zolo::eps_precision() / 2.0, maxit);
  *steps = S.steps;
  if (S.steps > max_steps) return -4;
  for (int k = 0; k < S.steps; ++k) {
    if (qr) qr[k] = S.qr[k];
    if (table)
      for (size_t i = 0; i < static_cast<size_t>(5) * count; ++i)
        table[static_cast<size_t>(k) * 5 * count + i] = S.table[static_cast<size_t>(k) * 5 * count + i];
  }
  for (int b = 0; b < count; ++b) {
    if (ucount) ucount[b] = S.count[b];
    if (last) last[b] = S.last[b];
    if (cond) cond[b] = S.cond[b];
  }
  return 0;
}

int zolo_polar_dev(zolo_handle_t h, int rk, int m, int n, const double* dA, int64_t lda, double* dQ, int64_t ldq,
                   double* dH, int64_t ldh) {
  if (m < n) return -3;
  if (lda < std::max(1, m) || ldq < std::max(1, m) || (dH && ldh < std::max(1, n))) return -6;
  return guarded(h, [&](Context& c) { return zolo::zolo_polar(c, rk, m, n, dA, lda, dQ, ldq, dH, ldh); });
}

int zolo_pzolopd1_dev(zolo_handle_t h, char sym, int rk, int m, int n, double alpha, double beta, const double* dA,
                      int64_t lda, double* dQ, int64_t ldq, double* dH, int64_t ldh) {
  return guarded(h, [&](Context& c) {
    return zolo_pd_entry(c, sym, rk, m, n, alpha, beta, dA, lda, dQ, ldq, dH, ldh);
  });
}

int zolo_bounds_dev(zolo_handle_t h, int m, int n, double sigma, const double* dA, int64_t lda, int mode,
                    double* alpha, double* beta) {
  if (m < n) return -2;
  if (mode < 0 || mode > 3) return -7;
  return guarded(h, [&](Context& c) {
    c.stats = zolo::Stats{};
    return zolo::bounds(c, m, n, sigma, dA, lda, static_cast<zolo::BoundsMode>(mode), alpha, beta);
  });
}

int zolo_form_h_dev(zolo_handle_t h, int m, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda,
                    double* dH, int64_t ldh) {
  return guarded(h, [&](Context& c) {
    zolo::form_h(c, m, n, dQ, ldq, dA, lda, dH, ldh);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_syev_dev(zolo_handle_t h, int n, const double* dH, int64_t ldh, double* dW, double* dZ, int64_t ldz) {
  if (n < 0) return -2;
  return guarded(h, [&](Context& c) {
    zolo::EigStats es;
    const int info = zolo::syev_dc(c, n, dH, ldh, dW, dZ, ldz, &es);
    c.stats = zolo::Stats{};
    c.stats.iterations = es.splits;
    c.stats.qr_iterations = es.qdwh_iterations;
    c.stats.chol_iterations = es.leaves;
    c.stats.last_err = es.max_split_residual;
    c.stats.flops = es.flops;
    // device ms: ms_step[l] = top-down level l, ms_finish = leaves, ms_h = back-transformation
    for (int l = 0; l < std::min(es.levels, 16); ++l) c.stats.ms_step[l] = es.ms_level[l];
    c.stats.ms_finish = es.ms_leaves;
    c.stats.ms_h = es.ms_back;
    c.stats.ms_total = es.ms_total;
    c.stats.ns_steps = es.subspace_passes;
    c.stats.terms[0] = es.qdwh_calls;
    c.stats.terms[1] = es.zolo_calls;
    c.stats.terms[2] = es.batched_nodes;
    c.stats.terms[3] = static_cast<int>(es.reallocs);
    // host wall ms of the levels' phases (diagnostic): con[0..3]
    c.stats.con[0] = es.wall_diag;
    c.stats.con[1] = es.wall_batch;
    c.stats.con[2] = es.wall_split;
    c.stats.con[3] = es.wall_free;
    return info;
  });
}

int zolo_svd_dev(zolo_handle_t h, int algo, int rk, int m, int n, const double* dA, int64_t lda, double* dU,
                 int64_t ldu, double* dS, double* dV, int64_t ldv) {
  if (m < n) return -4;
  if (algo == 1 && (rk < 1 || rk > 8)) return -3;
  return guarded(h, [&](Context& c) { return zolo::svd(c, m, n, dA, lda, algo, rk, dU, ldu, dS, dV, ldv, nullptr); });
}

int zolo_zoloeig_dev(zolo_handle_t h, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, int* rk,
                     double* dW, double* dZ, int64_t ldz) {
  if (n < 0) return -2;
  return guarded(h, [&](Context& c) {
    return zolo::zoloeig(c, n, dQ, ldq, dA, lda, rk, dW, dZ, ldz, nullptr, 0, nullptr, 0);
  });
}

void zolo_zoloeig(int n, int /*nblk*/, double* q, double* as, int /*contxt*/, int /*mpi_newcomm*/, double* work,
                  int lwork, double* /*work2*/, int lwork2, double* tau, int* info) {
  int r = 0;
  if (n < 0) r = -1;
  else if (lwork < n * n) r = -8;
  else if (lwork2 < n * n) r = -10;
  if (r == 0 && n > 0) {
    zolo_handle_t h = nullptr;
    r = zolo_default_handle(&h);
    if (r == 0)
      r = guarded(h, [&](Context& c) -> int {
        // device copies of the caller's arrays: handle workspace, allocated once and reused
        const size_t nn = static_cast<size_t>(n) * n;
        const DevView dQ{c.buf("host_q", nn)}, dA{c.buf("host_a", nn)}, dV{c.buf("host_v", nn)};
        const DevView dE{c.buf("host_e", nn)}, dW{c.buf("host_w", n)}, dZ{c.buf("host_z", nn)};
        zolo::ck(cudaMemcpyAsync(dQ.p, q, nn * 8, cudaMemcpyHostToDevice, c.stream()));
        zolo::ck(cudaMemcpyAsync(dA.p, as, nn * 8, cudaMemcpyHostToDevice, c.stream()));
        int rk = 0;
        const int inf = zolo::zoloeig(c, n, dQ.p, n, dA.p, n, &rk, dW.p, dZ.p, n, dV.p, n, dE.p, n);
        if (inf == 0 && rk > 0 && rk < n) {
          zolo::ck(cudaMemcpyAsync(q, dV.p, nn * 8, cudaMemcpyDeviceToHost, c.stream()));
          zolo::ck(cudaMemcpyAsync(as, dE.p, nn * 8, cudaMemcpyDeviceToHost, c.stream()));
          zolo::ck(cudaMemcpyAsync(tau, dW.p, static_cast<size_t>(rk) * 8, cudaMemcpyDeviceToHost, c.stream()));
          zolo::ck(cudaMemcpyAsync(work, dZ.p, static_cast<size_t>(n) * rk * 8, cudaMemcpyDeviceToHost, c.stream()));
        }
        zolo::ck(cudaStreamSynchronize(c.stream()));
        return inf;
      });
  }
  if (info) *info = r;
}

void zoloeig_(const int* n, const int* nblk, double* q, double* as, const int* contxt, const int* mpi_newcomm,
              double* work, const int* lwork, double* work2, const int* lwork2, double* tau, int* info) {
  zolo_zoloeig(*n, *nblk, q, as, *contxt, *mpi_newcomm, work, *lwork, work2, *lwork2, tau, info);
}

int zolo_dgemm_dev(zolo_handle_t h, char transa, char transb, int m, int n, int k, double alpha, const double* dA,
                   int64_t lda, const double* dB, int64_t ldb, double beta, double* dC, int64_t ldc, int tri,
                   int kfrom_n) {
  return guarded(h, [&](Context& c) {
    zolo::gemm(c, upper(transa), upper(transb), m, n, k, alpha, zolo::Mat{const_cast<double*>(dA), lda, 0},
               zolo::Mat{const_cast<double*>(dB), ldb, 0}, beta, zolo::Mat{dC, ldc, 0}, 1, nullptr, tri, kfrom_n);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_ozgemm_dev(zolo_handle_t h, char transa, char transb, int m, int n, int k, double alpha, const double* dA,
                    int64_t lda, const double* dB, int64_t ldb, double beta, double* dC, int64_t ldc, int tri,
                    int kfrom_n, int slices) {
  if (m < 0) return -4;
  if (n < 0) return -5;
  if (k < 0) return -6;
  if (slices < 6 || slices > 8) return -17;
  if (tri && m != n) return -15;
  if (!zolo::ozgemm_k_ok(slices, k)) return -6;
  return guarded(h, [&](Context& c) {
    zolo::ozgemm(c, upper(transa), upper(transb), m, n, k, alpha, zolo::Mat{const_cast<double*>(dA), lda, 0},
                 zolo::Mat{const_cast<double*>(dB), ldb, 0}, beta, zolo::Mat{dC, ldc, 0}, 1, slices, tri, kfrom_n);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    const int st = zolo::oz_status(c);
    return st ? -2000 - st : 0;
  });
}

int zolo_dpotrf_dev(zolo_handle_t h, int n, double* dA, int64_t lda) {
  return guarded(h, [&](Context& c) {
    int* dinfo = c.dinfo();
    zolo::ck(cudaMemsetAsync(dinfo, 0, sizeof(int), c.stream()));
    zolo::DiagInv D{c.buf("dinv", static_cast<size_t>(zolo::nblocks(n)) * 4096), 0};
    zolo::potrf(c, n, zolo::Mat{dA, lda, 0}, 1, dinfo, D);
    int info = 0;
    zolo::ck(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, c.stream()));
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return info;
  });
}

int zolo_dtrsm_dev(zolo_handle_t h, char trans, int m, int n, const double* dL, int64_t ldl, double* dX, int64_t ldx,
                   double* dY, int64_t ldy) {
  return guarded(h, [&](Context& c) {
    zolo::Mat L{const_cast<double*>(dL), ldl, 0}, X{dX, ldx, 0}, Y{dY, ldy, 0};
    zolo::DiagInv D{c.buf("dinv", static_cast<size_t>(zolo::nblocks(n)) * 4096), 0};
    zolo::diag_inverses(c, n, L, 1, D);
    if (upper(trans)) zolo::trsm_rlt(c, m, n, L, X, Y, 1, D);
    else zolo::trsm_rln(c, m, n, L, X, Y, 1, D);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_dtrtri_dev(zolo_handle_t h, int n, const double* dL, int64_t ldl, double* dY, int64_t ldy) {
  if (n < 0) return -2;
  if (ldl < std::max(1, n)) return -4;
  if (ldy < std::max(1, n)) return -6;
  if (n == 0) return 0;
  return guarded(h, [&](Context& c) {
    zolo::Mat L{const_cast<double*>(dL), ldl, 0}, Y{dY, ldy, 0};
    zolo::DiagInv D{c.buf("dinv", static_cast<size_t>(zolo::nblocks(n)) * 4096), 0};
    zolo::diag_inverses(c, n, L, 1, D);
    zolo::trtri_lower(c, n, L, Y, 1, D);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_dgeqrf_dev(zolo_handle_t h, int mtot, int n, int m_top, double* dW, int64_t ldw, double* dtau, double* dT) {
  if (mtot < n) return -2;
  return guarded(h, [&](Context& c) {
    zolo::geqrf(c, mtot, n, m_top, zolo::Mat{dW, ldw, 0}, dtau, dT, 1);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_dorgqr_dev(zolo_handle_t h, int mtot, int n, int m_top, const double* dW, int64_t ldw, const double* dT,
                    double* dQ, int64_t ldq) {
  if (mtot < n) return -2;
  return guarded(h, [&](Context& c) {
    zolo::orgqr(c, mtot, n, m_top, zolo::Mat{const_cast<double*>(dW), ldw, 0}, dT, zolo::Mat{dQ, ldq, 0}, 1);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_zoloqr_dev(zolo_handle_t h, int m, int n, const double* dX, int64_t ldx, double cc, double a, double* dZ,
                    int64_t ldz) {
  if (!(cc > 0.0)) return -6;
  return guarded(h, [&](Context& c) {
    const int mp = (m + 1) / 2 * 2;
    const int64_t ldw = (static_cast<int64_t>(mp) + n + 1) / 2 * 2;
    zolo::Mat W{c.buf("W", static_cast<size_t>(ldw) * n), ldw, 0};
    zolo::Mat Qf{c.buf("Qf", static_cast<size_t>(ldw) * n), ldw, 0};
    double* tau = c.buf("tau", n);
    double* T = c.buf("qr_t", static_cast<size_t>((n + 31) / 32) * 1024);
    const double s = std::sqrt(cc);
    zolo::ck(zolo::form_stack(m, mp, n, dX, ldx, W.p, W.ld, 0, nullptr, s, 1, c.stream()));
    zolo::geqrf(c, mp + n, n, mp, W, tau, T, 1);
    zolo::orgqr(c, mp + n, n, mp, W, T, Qf, 1);
    zolo::gemm(c, 0, 1, m, n, n, a / s, Qf, Qf.at(mp, 0), 0.0, zolo::Mat{dZ, ldz, 0}, 1, nullptr, 0, 1);
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return 0;
  });
}

int zolo_zolochol_dev(zolo_handle_t h, int m, int n, const double* dX, int64_t ldx, double cc, double a, double* dZ,
                      int64_t ldz) {
  return guarded(h, [&](Context& c) {
    const int64_t ldn = (n + 1) / 2 * 2, ldm = (m + 1) / 2 * 2;
    zolo::Mat G{c.buf("G", static_cast<size_t>(ldn) * n), ldn, 0};
    zolo::Mat Xc{c.buf("Xc", static_cast<size_t>(ldm) * n), ldm, 0};
    zolo::Mat Y{c.buf("Y", static_cast<size_t>(ldm) * n), ldm, 0};
    zolo::gemm(c, 1, 0, n, n, m, 1.0, zolo::Mat{const_cast<double*>(dX), ldx, 0},
               zolo::Mat{const_cast<double*>(dX), ldx, 0}, 0.0, G, 1, nullptr, 1, 0);
    zolo::ck(zolo::add_diag(n, G.p, G.ld, cc, c.stream()));
    int* dinfo = c.dinfo();
    zolo::ck(cudaMemsetAsync(dinfo, 0, sizeof(int), c.stream()));
    zolo::DiagInv D{c.buf("dinv", static_cast<size_t>(zolo::nblocks(n)) * 4096), 0};
    zolo::potrf(c, n, G, 1, dinfo, D);
    zolo::ck(zolo::scale_copy(m, n, a, dX, ldx, 0, Xc.p, Xc.ld, 0, 1, 0.0, c.stream()));
    zolo::trsm_rlt(c, m, n, G, Xc, Y, 1, D);
    zolo::trsm_rln(c, m, n, G, Y, zolo::Mat{dZ, ldz, 0}, 1, D);
    int info = 0;
    zolo::ck(cudaMemcpyAsync(&info, dinfo, sizeof(int), cudaMemcpyDeviceToHost, c.stream()));
    zolo::ck(cudaStreamSynchronize(c.stream()));
    return info;
  });
}

int zolo_formx2_dev(zolo_handle_t h, int m, int n, double fone, double* dX, int64_t ldx, const double* dZ,
                    int64_t ldz, double* err) {
  return guarded(h, [&](Context& c) {
    double* scal = c.dscal();
    zolo::ck(zolo::combine_update(m, n, dX, ldx, dZ, ldz, 0, 1, 1.0 / fone, 1.0 / fone, nullptr, c.dpartial(), scal,
                                  c.stream()));
    double e2 = 0.0;
    zolo::ck(cudaMemcpyAsync(&e2, scal, sizeof(double), cudaMemcpyDeviceToHost, c.stream()));
    zolo::ck(cudaStreamSynchronize(c.stream()));
    if (err) *err = std::sqrt(e2);
    return 0;
  });
}

}  // extern "C"
