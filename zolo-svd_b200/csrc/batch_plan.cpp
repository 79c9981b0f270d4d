// Bucket plan of the batched QDWH solver; see batch_plan.h.
#include "batch_plan.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <numeric>

#include "coeff.h"

namespace zolo {

namespace {
inline int up32(int x) { return (x + 31) / 32 * 32; }

double latency_ms(const BatchCostModel& mdl, int NB) { return mdl.lat0 + mdl.lat1 * NB / 32.0; }

double work_ms(const BatchCostModel& mdl, int B, int MB, int NB) {
  const double rate = mdl.rate_tflops * 1e9 * NB / (NB + mdl.nhalf);  // flops per ms
  return B * batch_member_flops(MB, NB) / rate;
}

// longest-processing-time assignment of the buckets to the workers: per-worker latency sums
double worker_latency(const BatchCostModel& mdl, const BucketPlan& p) {
  const int w = std::max(1, mdl.streams);
  std::vector<double> lat(p.nb.size());
  for (size_t b = 0; b < p.nb.size(); ++b) lat[b] = latency_ms(mdl, p.nb[b]);
  std::vector<size_t> order(lat.size());
  std::iota(order.begin(), order.end(), 0);
  std::sort(order.begin(), order.end(), [&](size_t a, size_t b) { return lat[a] > lat[b]; });
  std::vector<double> load(w, 0.0);
  for (size_t b : order) *std::min_element(load.begin(), load.end()) += lat[b];
  return *std::max_element(load.begin(), load.end());
}
}  // namespace

double batch_member_flops(int MB, int NB) {
  const double m = MB, n = NB;
  // bounds (QR of A, triangular inverse) + 2 QR-form iterations (4 m n^2 + n^3 each)
  // + 4 Cholesky-form iterations (3 m n^2 + n^3 / 3 each) + H (2 m n^2)
  return (4.0 / 3.0 * n * n * n + 2.0 * m * n * n) + 2.0 * (4.0 * m * n * n + n * n * n) +
         4.0 * (3.0 * m * n * n + n * n * n / 3.0) + 2.0 * m * n * n;
}

double batch_bucket_ms(const BatchCostModel& mdl, int B, int MB, int NB) {
  return latency_ms(mdl, NB) + work_ms(mdl, B, MB, NB);
}

void batch_pad(const std::vector<int>& ms, const std::vector<int>& ns, int* MB, int* NB) {
  int nb = 0;
  for (int v : ns) nb = std::max(nb, v);
  nb = up32(nb);
  int mb = nb;
  for (size_t i = 0; i < ms.size(); ++i) mb = std::max(mb, ms[i] + nb - ns[i]);
  *NB = nb;
  *MB = up32(mb);
}

double plan_predicted_ms(const BatchCostModel& mdl, const BucketPlan& p) {
  double work = 0.0;
  for (size_t b = 0; b < p.nb.size(); ++b)
    work += work_ms(mdl, static_cast<int>(p.members[b].size()), p.mb[b], p.nb[b]);
  return work + worker_latency(mdl, p);
}

BucketPlan plan_buckets(const BatchCostModel& mdl, int count, const int* m, const int* n, int max_batch) {
  BucketPlan p;
  if (count <= 0) return p;
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] != n[b] ? n[a] < n[b] : m[a] < m[b]; });
  // best[j]: cheapest plan of the first j sorted members; each bucket is charged its work
  // plus its latency shared by the concurrent worker streams
  const double share = 1.0 / std::max(1, mdl.streams);
  std::vector<double> best(count + 1, std::numeric_limits<double>::infinity());
  std::vector<int> from(count + 1, 0);
  best[0] = 0.0;
  for (int j = 0; j < count; ++j) {
    const int NB = up32(n[order[j]]);
    int MB = NB;
    for (int i = j; i >= 0 && j - i + 1 <= max_batch; --i) {
      MB = std::max(MB, up32(m[order[i]] + NB - n[order[i]]));
      const double c = best[i] + share * latency_ms(mdl, NB) + work_ms(mdl, j - i + 1, MB, NB);
      if (c < best[j + 1]) {
        best[j + 1] = c;
        from[j + 1] = i;
      }
    }
  }
  std::vector<std::pair<int, int>> runs;
  for (int j = count; j > 0; j = from[j]) runs.emplace_back(from[j], j);
  std::reverse(runs.begin(), runs.end());
  for (const auto& r : runs) {
    std::vector<int> idx(order.begin() + r.first, order.begin() + r.second), ms, ns;
    for (int i : idx) {
      ms.push_back(m[i]);
      ns.push_back(n[i]);
    }
    int MB, NB;
    batch_pad(ms, ns, &MB, &NB);
    p.members.push_back(idx);
    p.mb.push_back(MB);
    p.nb.push_back(NB);
    p.ms.push_back(batch_bucket_ms(mdl, static_cast<int>(idx.size()), MB, NB));
  }
  p.total_ms = plan_predicted_ms(mdl, p);
  return p;
}

BucketPlan ladder_buckets(const BatchCostModel& mdl, int count, const int* m, const int* n, int max_batch) {
  static const int ladder[] = {32,  64,  96,  128, 160, 192,  224,  256,  320,  384,  448,  512,
                               640, 768, 896, 1024, 1280, 1536, 1792, 2048, 2560, 3072, 3584, 4096};
  auto size_of = [](int v) {
    for (int l : ladder)
      if (v <= l) return l;
    return (v + 511) / 512 * 512;
  };
  BucketPlan p;
  std::vector<int> order(count);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return n[a] < n[b]; });
  size_t i = 0;
  while (i < order.size()) {
    const int NB = size_of(n[order[i]]);
    std::vector<int> idx;
    while (i < order.size() && size_of(n[order[i]]) == NB && static_cast<int>(idx.size()) < max_batch)
      idx.push_back(order[i++]);
    int MB = NB;
    for (int k : idx) MB = std::max(MB, m[k] + NB - n[k]);
    MB = up32(MB);
    p.members.push_back(idx);
    p.mb.push_back(MB);
    p.nb.push_back(NB);
    p.ms.push_back(batch_bucket_ms(mdl, static_cast<int>(idx.size()), MB, NB));
  }
  p.total_ms = plan_predicted_ms(mdl, p);
  return p;
}

QdwhSchedule qdwh_schedule(int B, const double* l0, const char* done, double tol1, int maxit) {
  QdwhSchedule S;
  S.count.assign(B, 0);
  S.last.assign(B, -1);
  S.cond.assign(B, -1);
  S.l_uncond.assign(l0, l0 + B);
  S.l_cond.assign(l0, l0 + B);
  std::vector<char> act(B), pend(B, 0);
  std::vector<double> l(l0, l0 + B), ak(B), bk(B), ck(B), ln(B);
  for (int b = 0; b < B; ++b) act[b] = !done[b];
  while (true) {
    bool any = false, qr = false;
    for (int b = 0; b < B; ++b) {
      if (!act[b]) continue;
      any = true;
      qdwh_weights(l[b], &ak[b], &bk[b], &ck[b], &ln[b]);
      qr = qr || ck[b] > 100.0;
    }
    if (!any) break;
    const int k = S.steps++;
    S.qr.push_back(qr);
    S.table.resize(static_cast<size_t>(k + 1) * 5 * B, 0.0);
    double* row = S.table.data() + static_cast<size_t>(k) * 5 * B;
    for (int b = 0; b < B; ++b) {
      if (!act[b]) {
        row[b] = qr ? 1.0 : 0.0;
        row[B + b] = 1.0;
        row[2 * B + b] = 0.0;
        continue;
      }
      const double sck = std::sqrt(ck[b]);
      row[b] = qr ? 1.0 / sck : ck[b];
      row[B + b] = bk[b] / ck[b];
      row[2 * B + b] = qr ? (ak[b] - bk[b] / ck[b]) / sck : ak[b] - bk[b] / ck[b];
      l[b] = ln[b];
      if (pend[b]) {  // the conditional step: the member's last scheduled one
        row[4 * B + b] = 1.0;
        S.cond[b] = k;
        S.l_cond[b] = l[b];
        act[b] = 0;
        continue;
      }
      ++S.count[b];
      S.l_uncond[b] = l[b];
      S.l_cond[b] = l[b];
      S.last[b] = k;
      if (S.count[b] > maxit) {
        act[b] = 0;
      } else if (!(std::fabs(1.0 - l[b]) > tol1)) {
        pend[b] = 1;
      }
    }
  }
  return S;
}

}  // namespace zolo
