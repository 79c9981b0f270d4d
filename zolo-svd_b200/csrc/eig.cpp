// Symmetric eigensolver by spectral divide-and-conquer on the polar
// decomposition (the reference's QDWH-eig split of pqdwheig.f90:168-228 /
// ZoloEig.f90:78-102 / pqdwhsubit.f90:227-312, applied recursively), with a
// batched Jacobi kernel at the leaves; ZoloEig; and the Zolo-SVD assembly of
// ZoloCHK1.f90:80-91 (H = sym(Q^T A), H = Z diag(w) Z^T, U = Q Z).
#include "eig.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <mutex>
#include <numeric>
#include <thread>
#include <vector>

#include "linalg.h"
#include "polar.h"

namespace zolo {

namespace {

inline int64_t even(int64_t x) { return (x + 1) / 2 * 2; }

double wall_ms_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

// The divide-and-conquer's node matrices: blocks from the handle's pool (reused across calls,
// cudaMalloc only when no free block fits), returned to it when released.  A block released
// between levels is reused by a later level's work only, which runs on streams ordered after
// the releasing level's (each level's workers wait for the previous level's).
struct DevMem {
  Context& pool;
  std::vector<std::pair<void*, size_t>> blocks;
  std::mutex mu;  // nodes of one level are split by concurrent workers
  explicit DevMem(Context& c) : pool(c) {}
  double* alloc(size_t elems) {
    std::lock_guard<std::mutex> lk(mu);
    size_t bytes = 0;
    void* p = pool.pool_take(std::max<size_t>(elems, 1) * sizeof(double), &bytes);
    blocks.emplace_back(p, bytes);
    return static_cast<double*>(p);
  }
  void release(double* p) {
    std::lock_guard<std::mutex> lk(mu);
    for (auto& b : blocks)
      if (b.first == p) {
        pool.pool_give(b.first, b.second);
        b.first = nullptr;
      }
  }
  // every block back to the pool once the work queued on the handle's and the workers'
  // streams has run (also on an error return)
  ~DevMem() {
    pool.sync_all();
    for (auto& b : blocks)
      if (b.first) pool.pool_give(b.first, b.second);
  }
};

double d2h(Context& c, const double* d) {
  double v = 0.0;
  ck(cudaMemcpyAsync(&v, d, sizeof(double), cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  return v;
}

struct Node {
  int n = 0;
  double* H = nullptr;  // node matrix (n x n, ld ldn)
  int64_t ld = 0;
  double* V = nullptr;  // split basis [V1 V2]
  double* Z = nullptr;  // eigenvectors
  double* w = nullptr;  // eigenvalues
  int k = 0;
  int left = -1, right = -1;
  bool leaf = false;
};

// Orthonormal basis of range(P) completed to an n x n orthogonal V = [V1 V2]:
// V from the Householder QR of X (n x k) with all n columns formed.
void basis_from(Context& c, int n, int k, Mat X, double* V, int64_t ldv) {
  double* tau = c.buf("eig_tau", k);
  double* T = c.buf("eig_t", static_cast<size_t>((k + 31) / 32) * 1024);
  geqrf(c, n, k, -1, X, tau, T, 1);
  orgqr(c, n, k, -1, X, T, Mat{V, ldv, 0}, 1, n);
}

// off = ||E(k:n, 0:k)||_F for E = V^T H V, returned in E; lower_only: only its lower triangle
// is formed (E is symmetric, and a split needs the diagonal blocks and the block below them)
double split_residual(Context& c, int n, int k, const double* H, int64_t ldh, const double* V, int64_t ldv, double* E,
                      int64_t lde, bool lower_only) {
  const int64_t ldn = even(n);
  double* HV = c.buf("eig_hv", static_cast<size_t>(ldn) * n);
  {
    OzScope mixed(c, c.zolo_mixed >= 1);  // normwise-accurate products in the mixed form
    gemm(c, 0, 0, n, n, n, 1.0, Mat{const_cast<double*>(H), ldh, 0}, Mat{const_cast<double*>(V), ldv, 0}, 0.0,
         Mat{HV, ldn, 0}, 1);
    gemm(c, 1, 0, n, n, n, 1.0, Mat{const_cast<double*>(V), ldv, 0}, Mat{HV, ldn, 0}, 0.0, Mat{E, lde, 0}, 1,
         nullptr, lower_only ? 1 : 0);
  }
  ck(frob2(n - k, k, E + k, lde, c.dpartial(), c.dscal() + 8, c.stream()));
  return std::sqrt(d2h(c, c.dscal() + 8));
}

// Runs task(ctx, i) for i in [0, count): on `c` itself for one task, otherwise on up to eight
// worker contexts (own stream and workspace each, one host thread each) that take the tasks
// in order.  Work queued on c.stream() before the call is visible to the tasks, and their work
// is ordered before anything queued on c.stream() after it.  Rethrows a task's CUDA failure.
// The tasks go to the workers by a fixed rule, the costliest first onto the least loaded
// worker (cost[i] estimates task i), so that the same nodes meet the same worker and its
// workspace on every call with the same split sizes.
template <class F>
void run_concurrent(Context& c, int count, const std::vector<double>& cost, F&& task) {
  if (count <= 0) return;
  const int W = std::min(count, 8);
  if (W == 1) {
    for (int i = 0; i < count; ++i) task(c, i);
    return;
  }
  while (static_cast<int>(c.workers.size()) < W) c.workers.emplace_back(new Context(c.device()));
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return cost[a] > cost[b]; });
  std::vector<std::vector<int>> assign(W);
  std::vector<double> load(W, 0.0);
  for (int i : order) {
    const int w = static_cast<int>(std::min_element(load.begin(), load.end()) - load.begin());
    assign[w].push_back(i);
    load[w] += cost[i] + 1.0;
  }
  ck(cudaEventRecord(c.event(0), c.stream()));
  std::atomic<bool> stop{false};
  std::vector<cudaError_t> err(W, cudaSuccess);
  std::vector<std::thread> th;
  for (int w = 0; w < W; ++w) {
    th.emplace_back([&, w] {
      try {
        Context& wc = *c.workers[w];
        ck(cudaSetDevice(wc.device()));
        ck(cudaStreamWaitEvent(wc.stream(), c.event(0), 0));
        wc.zolo_mixed = c.zolo_mixed;
        wc.oz_slices = c.oz_slices;
        wc.eig_zolo_min = c.eig_zolo_min;
        for (int i : assign[w]) {
          if (stop) break;
          task(wc, i);
        }
      } catch (const CudaFailure& e) {
        err[w] = e.err;
        stop = true;
      } catch (...) {
        err[w] = cudaErrorUnknown;
        stop = true;
      }
    });
  }
  for (auto& t : th) t.join();
  for (int w = 0; w < W; ++w) {
    Context& wc = *c.workers[w];
    ck(cudaEventRecord(wc.event(0), wc.stream()));
    ck(cudaStreamWaitEvent(c.stream(), wc.event(0), 0));
  }
  for (int w = 0; w < W; ++w)
    if (err[w] != cudaSuccess) throw CudaFailure{err[w]};
}

// Candidate shifts of a node from its diagonal: the median and the mean, then the median
// nudged by 1e-3 of the diagonal's span either way.
void split_candidates(const std::vector<double>& dg, double cand[4]) {
  const int m = static_cast<int>(dg.size());
  std::vector<double> srt = dg;
  std::sort(srt.begin(), srt.end());
  const double med = srt[m / 2], mean = std::accumulate(dg.begin(), dg.end(), 0.0) / m;
  const double span = std::max(srt.back() - srt.front(), 1e-300);
  cand[0] = 0.5 * (srt[(m - 1) / 2] + srt[m / 2]);
  cand[1] = mean;
  cand[2] = med + 1e-3 * span;
  cand[3] = med - 1e-3 * span;
}

// The Zolo-PD fast form on a context for the scope (shared QR, Newton-Schulz finish,
// explicit-inverse Cholesky, Frobenius beta, term plan; ||A||_F as alpha), restored on exit.
struct FastForm {
  Context& c;
  int saved[6];
  explicit FastForm(Context& ctx)
      : c(ctx),
        saved{ctx.zolo_shared_qr, ctx.zolo_ns_finish, ctx.zolo_chol_inverse, ctx.zolo_beta_frob, ctx.zolo_term_plan,
              ctx.zolo_norm2} {
    c.zolo_shared_qr = c.zolo_ns_finish = c.zolo_chol_inverse = c.zolo_beta_frob = c.zolo_term_plan = 1;
    c.zolo_norm2 = 0;
  }
  ~FastForm() {
    c.zolo_shared_qr = saved[0];
    c.zolo_ns_finish = saved[1];
    c.zolo_chol_inverse = saved[2];
    c.zolo_beta_frob = saved[3];
    c.zolo_term_plan = saved[4];
    c.zolo_norm2 = saved[5];
  }
};

bool zolo_node(const Context& c, int m) { return c.eig_zolo_min > 0 && m >= c.eig_zolo_min; }

// The polar factor of H - sigma I for the first candidate shift, computed before the node is
// split (the level's nodes in one batched solve): Up (ld even(m)), or info != 0 if it failed.
struct Presolved {
  const double* Up = nullptr;
  int info = 1;
};

// One node of the divide-and-conquer: a leaf (m <= kJacobiLeaf) or a split into the blocks of
// V^T H V above and below a shift (QDWH polar factor of H - sigma I, subspace basis of its
// projector).  Fills nd (k, V, Z, w) and the children L, R; returns false if no candidate
// shift splits the spectrum.  dg: the node's diagonal (empty for a leaf); pre: the first
// candidate's polar factor when already computed.
bool split_node(Context& c, Node& nd, Node& L, Node& R, DevMem& mem, double hnorm, uint64_t seed, EigStats& S,
                const std::vector<double>& dg, const Presolved& pre) {
  const double eps = 2.220446049250313e-16;
  const int m = nd.n;
  const int64_t ldm = even(m);
  nd.Z = mem.alloc(static_cast<size_t>(ldm) * m);
  nd.w = mem.alloc(m);
  if (m <= kJacobiLeaf) {
    nd.leaf = true;
    return true;
  }
  double cand[4];
  split_candidates(dg, cand);
  nd.V = mem.alloc(static_cast<size_t>(ldm) * m);
  double* Up = c.buf("eig_up", static_cast<size_t>(ldm) * m);
  double* P = c.buf("eig_p", static_cast<size_t>(ldm) * m);
  double* X = c.buf("eig_x", static_cast<size_t>(ldm) * m);
  double* E = c.buf("eig_e", static_cast<size_t>(ldm) * m);
  for (int a = 0; a < 4; ++a) {
    const double* Ua = Up;
    if (a == 0 && pre.Up) {
      if (pre.info != 0) continue;
      Ua = pre.Up;
    } else if (a == 0 && zolo_node(c, m)) {
      // a large node: the polar factor of H - sigma I by Zolo-PD (r = 8, fast form)
      double* Hs = c.buf("eig_hs", static_cast<size_t>(ldm) * m);
      ck(scale_copy(m, m, 1.0, nd.H, nd.ld, 0, Hs, ldm, 0, 1, 0.0, c.stream()));
      ck(add_diag(m, Hs, ldm, -cand[0], c.stream()));
      const Stats saved = c.stats;
      int info;
      {
        FastForm ff(c);
        info = zolo_polar(c, 8, m, m, Hs, ldm, Up, ldm, nullptr, 0);
      }
      S.zolo_calls++;
      S.qdwh_iterations += c.stats.iterations;
      S.flops += c.stats.flops;
      c.stats = saved;
      if (info != 0) continue;
    } else {
      QdwhOpts o;
      o.sym = 'N';
      o.sigma = cand[a];
      o.bounds = BOUNDS_PQDWHFACS;
      o.maxit = 12;
      const Stats saved = c.stats;
      const int info = qdwh(c, m, m, nd.H, nd.ld, Up, ldm, nullptr, 0, o);
      S.qdwh_calls++;
      S.qdwh_iterations += c.stats.iterations;
      S.flops += c.stats.flops;
      c.stats = saved;
      if (info != 0) continue;
    }
    // projector onto the eigenvalues above the split: P = (Up + I)/2, k = trace(P)
    ck(scale_copy(m, m, 0.5, Ua, ldm, 0, P, ldm, 0, 1, 0.5, c.stream()));
    ck(trace(m, P, ldm, c.dscal() + 10, c.stream()));
    const int k = static_cast<int>(std::lround(d2h(c, c.dscal() + 10)));
    if (k <= 0 || k >= m) continue;
    // subspace: V = full Q of QR(P * Omega); a second pass with X = P V1 if the split leaks
    double* Om = c.buf("eig_om", static_cast<size_t>(ldm) * k);
    ck(fill_random(m, k, Om, ldm, seed + a, c.stream()));
    {
      OzScope mixed(c, c.zolo_mixed >= 1);
      gemm(c, 0, 0, m, k, m, 1.0, Mat{P, ldm, 0}, Mat{Om, ldm, 0}, 0.0, Mat{X, ldm, 0}, 1);
    }
    basis_from(c, m, k, Mat{X, ldm, 0}, nd.V, ldm);
    const double tol = 10.0 * eps * std::sqrt(static_cast<double>(m)) * std::max(hnorm, 1e-300);
    double off = split_residual(c, m, k, nd.H, nd.ld, nd.V, ldm, E, ldm, true);
    S.subspace_passes++;
    for (int pass = 1; pass < 3 && off > tol; ++pass) {
      gemm(c, 0, 0, m, k, m, 1.0, Mat{P, ldm, 0}, Mat{nd.V, ldm, 0}, 0.0, Mat{X, ldm, 0}, 1);
      basis_from(c, m, k, Mat{X, ldm, 0}, nd.V, ldm);
      off = split_residual(c, m, k, nd.H, nd.ld, nd.V, ldm, E, ldm, true);
      S.subspace_passes++;
    }
    S.max_split_residual = std::max(S.max_split_residual, off / std::max(hnorm, 1e-300));
    nd.k = k;
    L = Node{};
    R = Node{};
    L.n = k;
    L.ld = even(k);
    L.H = mem.alloc(static_cast<size_t>(L.ld) * k);
    ck(scale_copy(k, k, 1.0, E, ldm, 0, L.H, L.ld, 0, 1, 0.0, c.stream()));
    ck(mirror_lower(k, L.H, L.ld, c.stream()));
    R.n = m - k;
    R.ld = even(m - k);
    R.H = mem.alloc(static_cast<size_t>(R.ld) * (m - k));
    ck(scale_copy(m - k, m - k, 1.0, E + k + static_cast<int64_t>(k) * ldm, ldm, 0, R.H, R.ld, 0, 1, 0.0,
                  c.stream()));
    ck(mirror_lower(m - k, R.H, R.ld, c.stream()));
    S.splits++;
    return true;
  }
  return false;
}

}  // namespace

int syev_dc(Context& c, int n, const double* dH, int64_t ldh, double* dW, double* dZ, int64_t ldz, EigStats* es) {
  if (n <= 0) return 0;
  EigStats local;
  EigStats& S = es ? *es : local;
  S = EigStats{};
  auto reallocs_now = [&]() {
    int64_t r = c.reallocs;
    for (auto& w : c.workers) r += w->reallocs;
    return r;
  };
  const int64_t reallocs0 = reallocs_now();
  EventTimer total(c.stream());
  DevMem mem(c);
  std::vector<Node> nodes;
  {
    Node root;
    root.n = n;
    root.ld = even(n);
    root.H = mem.alloc(static_cast<size_t>(root.ld) * n);
    ck(scale_copy(n, n, 1.0, dH, ldh, 0, root.H, root.ld, 0, 1, 0.0, c.stream()));
    nodes.push_back(root);
  }
  double hnorm;
  ck(frob2(n, n, nodes[0].H, nodes[0].ld, c.dpartial(), c.dscal() + 9, c.stream()));
  hnorm = std::sqrt(d2h(c, c.dscal() + 9));

  // ---- top-down splits, one level at a time: the nodes of a level run concurrently ----
  std::vector<std::pair<size_t, size_t>> levels;
  for (size_t lo = 0; lo < nodes.size();) {
    const size_t hi = nodes.size();
    levels.emplace_back(lo, hi);
    const int cnt = static_cast<int>(hi - lo);
    EventTimer tl(c.stream());
    std::vector<Node> kids(2 * cnt);
    std::vector<EigStats> st(cnt);
    std::vector<char> ok(cnt, 1);
    // the diagonals of the level's inner nodes (one read-back), their candidate shifts
    auto w0 = std::chrono::steady_clock::now();
    std::vector<std::vector<double>> dg(cnt);
    std::vector<int> inner;
    {
      size_t tot = 0;
      for (int i = 0; i < cnt; ++i)
        if (nodes[lo + i].n > kJacobiLeaf) {
          inner.push_back(i);
          tot += nodes[lo + i].n;
        }
      // (the large nodes' Zolo-PD runs inside their split; the batch takes the others)
      double* dd = c.buf("eig_diag", std::max<size_t>(tot, 1));
      std::vector<double> hd(tot);
      size_t off = 0;
      for (int i : inner) {
        ck(get_diag(nodes[lo + i].n, nodes[lo + i].H, nodes[lo + i].ld, dd + off, c.stream()));
        off += nodes[lo + i].n;
      }
      if (tot) {
        ck(cudaMemcpyAsync(hd.data(), dd, sizeof(double) * tot, cudaMemcpyDeviceToHost, c.stream()));
        ck(cudaStreamSynchronize(c.stream()));
      }
      off = 0;
      for (int i : inner) {
        dg[i].assign(hd.begin() + off, hd.begin() + off + nodes[lo + i].n);
        off += nodes[lo + i].n;
      }
    }
    // with two or more inner nodes, the QDWH of every node's H - sigma_0 I as one batched solve
    // (zolo_qdwh_batch_dev's buckets and graphs; PQDWHFACS bounds per member)
    S.wall_diag += wall_ms_since(w0);
    w0 = std::chrono::steady_clock::now();
    std::vector<Presolved> pre(cnt);
    double* arena = nullptr;
    std::vector<int> small;
    for (int i : inner)
      if (!zolo_node(c, nodes[lo + i].n)) small.push_back(i);
    inner.swap(small);
    if (inner.size() >= 2) {
      size_t tot = 0;
      for (int i : inner) tot += 2 * static_cast<size_t>(even(nodes[lo + i].n)) * nodes[lo + i].n;
      arena = mem.alloc(tot);
      const int nb = static_cast<int>(inner.size());
      std::vector<int> mm(nb), inf(nb, 0), its(nb, 0);
      std::vector<const double*> pa(nb);
      std::vector<double*> pq(nb);
      std::vector<int64_t> ld(nb);
      size_t off = 0;
      for (int j = 0; j < nb; ++j) {
        const Node& nd = nodes[lo + inner[j]];
        const int64_t ldm = even(nd.n);
        double cand[4];
        split_candidates(dg[inner[j]], cand);
        double* Hs = arena + off;
        double* Up = Hs + ldm * nd.n;
        off += 2 * static_cast<size_t>(ldm) * nd.n;
        ck(scale_copy(nd.n, nd.n, 1.0, nd.H, nd.ld, 0, Hs, ldm, 0, 1, 0.0, c.stream()));
        ck(add_diag(nd.n, Hs, ldm, -cand[0], c.stream()));
        mm[j] = nd.n;
        pa[j] = Hs;
        pq[j] = Up;
        ld[j] = ldm;
      }
      BatchStats bs;
      const Stats saved = c.stats;
      // the schedule issued eagerly: the split sizes, and with them the bucket shapes, rarely
      // recur, so a captured graph would be replayed seldom and its capture costs more than it
      // saves
      const int saved_graph = c.batch_graph;
      if (c.batch_graph == 1) c.batch_graph = 2;
      int rb = -1;
      try {
        rb = qdwh_batch(c, nb, mm.data(), mm.data(), pa.data(), ld.data(), pq.data(), ld.data(), nullptr, nullptr,
                        inf.data(), its.data(), &bs);
      } catch (...) {
        c.batch_graph = saved_graph;
        throw;
      }
      c.batch_graph = saved_graph;
      c.stats = saved;
      if (rb != 0) std::fill(inf.begin(), inf.end(), 1);  // each node then solves on its own
      S.qdwh_calls += nb;
      for (int j = 0; j < nb; ++j) {
        S.qdwh_iterations += its[j];
        pre[inner[j]] = Presolved{pq[j], inf[j]};
      }
      S.flops += bs.flops_useful;
      S.batched_nodes += nb;
    }
    S.wall_batch += wall_ms_since(w0);
    w0 = std::chrono::steady_clock::now();
    std::vector<double> cost(cnt);
    for (int i = 0; i < cnt; ++i) cost[i] = std::pow(static_cast<double>(nodes[lo + i].n), 3);
    run_concurrent(c, cnt, cost, [&](Context& wc, int i) {
      ok[i] = split_node(wc, nodes[lo + i], kids[2 * i], kids[2 * i + 1], mem, hnorm,
                         0x5EEDull + (lo + i) * 7919ull, st[i], dg[i], pre[i]) ? 1 : 0;
    });
    S.wall_split += wall_ms_since(w0);
    w0 = std::chrono::steady_clock::now();
    if (arena) mem.release(arena);
    for (int i = 0; i < cnt; ++i) {
      S.qdwh_calls += st[i].qdwh_calls;
      S.zolo_calls += st[i].zolo_calls;
      S.qdwh_iterations += st[i].qdwh_iterations;
      S.subspace_passes += st[i].subspace_passes;
      S.splits += st[i].splits;
      S.flops += st[i].flops;
      S.max_split_residual = std::max(S.max_split_residual, st[i].max_split_residual);
    }
    const double ms_lv = tl.stop();
    if (S.levels < 16) S.ms_level[S.levels] = ms_lv;
    S.levels++;
    for (int i = 0; i < cnt; ++i)
      if (!ok[i]) return 2;  // no usable split point (all candidates failed)
    for (int i = 0; i < cnt; ++i) {
      Node& nd = nodes[lo + i];
      if (nd.leaf) continue;
      nd.left = static_cast<int>(nodes.size());
      nd.right = nd.left + 1;
      nodes.push_back(kids[2 * i]);
      nodes.push_back(kids[2 * i + 1]);
    }
    // the split nodes' matrices are no longer needed (freed between levels: cudaFree waits)
    for (size_t i = lo; i < hi; ++i)
      if (i != 0 && !nodes[i].leaf) mem.release(nodes[i].H);
    S.wall_free += wall_ms_since(w0);
    lo = hi;
  }

  // ---- leaves: one batched Jacobi launch ----
  std::vector<JacobiLeaf> leaves;
  for (auto& nd : nodes)
    if (nd.leaf) leaves.push_back(JacobiLeaf{nd.H, nd.ld, nd.n, nd.w, nd.Z, even(nd.n)});
  S.leaves = static_cast<int>(leaves.size());
  EventTimer tleaf(c.stream());
  {
    void* dl = mem.alloc((sizeof(JacobiLeaf) * leaves.size() + sizeof(double) - 1) / sizeof(double));
    int* dsw = c.ibuf("eig_sweeps", leaves.size());
    ck(cudaMemcpyAsync(dl, leaves.data(), sizeof(JacobiLeaf) * leaves.size(), cudaMemcpyHostToDevice, c.stream()));
    ck(jacobi_leaves(static_cast<JacobiLeaf*>(dl), static_cast<int>(leaves.size()), 30, dsw, c.stream()));
    std::vector<int> sw(leaves.size());
    ck(cudaMemcpyAsync(sw.data(), dsw, sizeof(int) * sw.size(), cudaMemcpyDeviceToHost, c.stream()));
    ck(cudaStreamSynchronize(c.stream()));
    for (int s : sw) S.max_jacobi_sweeps = std::max(S.max_jacobi_sweeps, s);
  }
  S.ms_leaves = tleaf.stop();
  EventTimer tback(c.stream());

  // ---- bottom-up back-transformation, one level at a time (concurrent within a level) ----
  for (auto lv = levels.rbegin(); lv != levels.rend(); ++lv) {
    const size_t lo = lv->first;
    const int cnt = static_cast<int>(lv->second - lv->first);
    std::vector<double> cost(cnt);
    for (int i = 0; i < cnt; ++i) cost[i] = nodes[lo + i].leaf ? 0.0 : std::pow(static_cast<double>(nodes[lo + i].n), 3);
    run_concurrent(c, cnt, cost, [&](Context& wc, int i) {
      Node& nd = nodes[lo + i];
      if (nd.leaf) return;
      const Node& L = nodes[nd.left];
      const Node& R = nodes[nd.right];
      const int m = nd.n, k = nd.k;
      const int64_t ldm = even(m);
      OzScope mixed(wc, wc.zolo_mixed >= 1);
      gemm(wc, 0, 0, m, k, k, 1.0, Mat{nd.V, ldm, 0}, Mat{L.Z, even(L.n), 0}, 0.0, Mat{nd.Z, ldm, 0}, 1);
      gemm(wc, 0, 0, m, m - k, m - k, 1.0, Mat{nd.V + static_cast<int64_t>(k) * ldm, ldm, 0},
           Mat{R.Z, even(R.n), 0}, 0.0, Mat{nd.Z + static_cast<int64_t>(k) * ldm, ldm, 0}, 1);
      ck(cudaMemcpyAsync(nd.w, L.w, sizeof(double) * k, cudaMemcpyDeviceToDevice, wc.stream()));
      ck(cudaMemcpyAsync(nd.w + k, R.w, sizeof(double) * (m - k), cudaMemcpyDeviceToDevice, wc.stream()));
    });
    for (int i = 0; i < cnt; ++i) {
      const Node& nd = nodes[lo + i];
      if (!nd.leaf)
        S.flops += 2.0 * nd.n * (static_cast<double>(nd.k) * nd.k + static_cast<double>(nd.n - nd.k) * (nd.n - nd.k));
    }
  }

  S.ms_back = tback.stop();
  // ---- ascending order (dsyevd / ELPA convention) ----
  const Node& root = nodes[0];
  std::vector<double> w(n);
  ck(cudaMemcpyAsync(w.data(), root.w, sizeof(double) * n, cudaMemcpyDeviceToHost, c.stream()));
  ck(cudaStreamSynchronize(c.stream()));
  std::vector<int> perm(n);
  std::iota(perm.begin(), perm.end(), 0);
  std::stable_sort(perm.begin(), perm.end(), [&](int a, int b) { return w[a] < w[b]; });
  std::vector<double> ws(n);
  for (int i = 0; i < n; ++i) ws[i] = w[perm[i]];
  int* dperm = c.ibuf("eig_perm", n);
  ck(cudaMemcpyAsync(dperm, perm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, c.stream()));
  ck(cudaMemcpyAsync(dW, ws.data(), sizeof(double) * n, cudaMemcpyHostToDevice, c.stream()));
  ck(gather_columns(n, n, root.Z, even(n), dperm, dZ, ldz, c.stream()));
  S.ms_total = total.stop();
  S.reallocs = reallocs_now() - reallocs0;
  return 0;
}

int zoloeig(Context& c, int n, const double* dQ, int64_t ldq, const double* dA, int64_t lda, int* rk_out,
            double* dW, double* dZ, int64_t ldz, double* dVfull, int64_t ldv, double* dE, int64_t lde) {
  const int64_t ldn = even(n);
  const double eps = 2.220446049250313e-16;
  const double tol1 = 10.0 * eps / 2.0;
  // C = (Q - I)/2: minus the projector onto the eigenvalues below the shift (pqdwhsubit.f90:228-239)
  double* C = c.buf("ze_c", static_cast<size_t>(ldn) * n);
  ck(scale_copy(n, n, 0.5, dQ, ldq, 0, C, ldn, 0, 1, -0.5, c.stream()));
  ck(frob2(n, n, C, ldn, c.dpartial(), c.dscal() + 11, c.stream()));
  const double alpha = d2h(c, c.dscal() + 11);  // ||C||_F^2 (pqdwhsubit.f90:241-243)
  const int rk = static_cast<int>(std::lround(alpha));
  *rk_out = rk;
  ck(frob2(n, n, dA, lda, c.dpartial(), c.dscal() + 12, c.stream()));
  const double norma = std::sqrt(d2h(c, c.dscal() + 12));
  if (rk <= 0 || rk >= n) return rk <= 0 ? 0 : 0;
  int kk = std::min(rk + 3, n);  // oversampling pp = 3 (pqdwhsubit.f90:225)
  double* X = c.buf("ze_x", static_cast<size_t>(ldn) * n);
  double* Y = c.buf("ze_y", static_cast<size_t>(ldn) * n);
  double* V = dVfull ? dVfull : c.buf("ze_v", static_cast<size_t>(ldn) * n);
  const int64_t ldvv = dVfull ? ldv : ldn;
  double* E = dE ? dE : c.buf("ze_e", static_cast<size_t>(ldn) * n);
  const int64_t ldee = dE ? lde : ldn;
  ck(fill_random(n, kk, X, ldn, 0xC0FFEEull, c.stream()));
  for (int it = 1; it <= 2; ++it) {
    // orthonormal basis of X (n x kk), then X = C * basis, then the full n x n Q of its QR
    double* tau = c.buf("eig_tau", kk);
    double* T = c.buf("eig_t", static_cast<size_t>((kk + 31) / 32) * 1024);
    geqrf(c, n, kk, -1, Mat{X, ldn, 0}, tau, T, 1);
    orgqr(c, n, kk, -1, Mat{X, ldn, 0}, T, Mat{Y, ldn, 0}, 1, kk);
    gemm(c, 0, 0, n, kk, n, 1.0, Mat{C, ldn, 0}, Mat{Y, ldn, 0}, 0.0, Mat{X, ldn, 0}, 1);
    basis_from(c, n, kk, Mat{X, ldn, 0}, V, ldvv);
    const double off = split_residual(c, n, rk, dA, lda, V, ldvv, E, ldee, false) / norma;
    // err is the leading-rows block of the reference (E(1:Rk, Rk+1:N)); E is symmetric here
    if (off <= 4.0 * tol1 || it == 2) break;
    ck(scale_copy(n, rk, 1.0, V, ldvv, 0, Y, ldn, 0, 1, 0.0, c.stream()));
    gemm(c, 0, 0, n, rk, n, 1.0, Mat{C, ldn, 0}, Mat{Y, ldn, 0}, 0.0, Mat{X, ldn, 0}, 1);
    kk = rk;
  }
  // eigenpairs of the leading Rk block (PDSYEVD in ZoloEig.f90:98-99), then V1 * VV1
  const int64_t ldr = even(rk);
  double* Er = c.buf("ze_er", static_cast<size_t>(ldr) * rk);
  double* VV = c.buf("ze_vv", static_cast<size_t>(ldr) * rk);
  ck(scale_copy(rk, rk, 1.0, E, ldee, 0, Er, ldr, 0, 1, 0.0, c.stream()));
  ck(symmetrize(rk, Er, ldr, c.stream()));
  const int info = syev_dc(c, rk, Er, ldr, dW, VV, ldr, nullptr);
  if (info != 0) return info;
  gemm(c, 0, 0, n, rk, rk, 1.0, Mat{V, ldvv, 0}, Mat{VV, ldr, 0}, 0.0, Mat{dZ, ldz, 0}, 1);
  ck(cudaStreamSynchronize(c.stream()));
  return 0;
}

int svd(Context& c, int m, int n, const double* dA, int64_t lda, int algo, int rk, double* dU, int64_t ldu,
        double* dS, double* dV, int64_t ldv, EigStats* es) {
  if (m < n) return -2;
  const int64_t ldm = even(m), ldn = even(n);
  double* Q = c.buf("svd_q", static_cast<size_t>(ldm) * n);
  double* H = c.buf("svd_h", static_cast<size_t>(ldn) * n);
  int info;
  if (algo == 0) {
    QdwhOpts o;
    info = qdwh(c, m, n, dA, lda, Q, ldm, H, ldn, o);
  } else {
    // bounds + Zolo-PD + H; the first QR iteration reuses the bounds' QR of A/alpha
    info = zolo_polar(c, rk, m, n, dA, lda, Q, ldm, H, ldn);
  }
  if (info != 0) return info;
  const Stats pd = c.stats;
  info = syev_dc(c, n, H, ldn, dS, dV, ldv, es);
  if (info != 0) return info;
  {
    OzScope mixed(c, c.zolo_mixed >= 1);
    gemm(c, 0, 0, m, n, n, 1.0, Mat{Q, ldm, 0}, Mat{dV, ldv, 0}, 0.0, Mat{dU, ldu, 0}, 1);
  }
  ck(cudaStreamSynchronize(c.stream()));
  c.stats = pd;
  return 0;
}

}  // namespace zolo
