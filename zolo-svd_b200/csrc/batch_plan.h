// Bucket plan of the batched QDWH solver (host only): which members share one padded
// batched solve.  A bucket of B members padded to MB x NB costs a launch-chain latency
// (its kernels run one after another, each too small to fill the GPU) plus B times the
// padded member's work; fewer, larger buckets pay less latency but more padding.  The plan
// minimizes the predicted time over all partitions of the members sorted by n into
// contiguous runs (dynamic programming), with the latency of buckets that run concurrently
// on `streams` worker streams counted once per stream.
#pragma once
#include <vector>

namespace zolo {

struct BatchCostModel {
  // milliseconds of one bucket: lat0 + lat1 * NB/32 + B * flops(MB, NB) / rate(NB),
  // rate(NB) = rate_tflops * 1e9 * NB / (NB + nhalf) flops per millisecond
  double lat0 = 4.0;
  double lat1 = 0.35;
  double rate_tflops = 25.0;
  double nhalf = 384.0;
  int streams = 8;  // worker streams the buckets are spread over
};

// Executed FP64 flops of one padded member's PQDWHFACS solve (bounds, two QR-form and four
// Cholesky-form iterations, H), the model's unit of work.
double batch_member_flops(int MB, int NB);
// Predicted milliseconds of one bucket.
double batch_bucket_ms(const BatchCostModel& mdl, int B, int MB, int NB);
// Padded sizes of a bucket holding members with these n and m: NB = max n rounded up to 32,
// MB = max (m + NB - n) rounded up to 32.
void batch_pad(const std::vector<int>& ms, const std::vector<int>& ns, int* MB, int* NB);

struct BucketPlan {
  std::vector<std::vector<int>> members;  // member indices per bucket
  std::vector<int> mb, nb;                // padded sizes per bucket
  std::vector<double> ms;                 // predicted milliseconds per bucket
  double total_ms = 0.0;                  // predicted time of the whole batch
};
// The cheapest partition under `mdl`, at most max_batch members per bucket.
BucketPlan plan_buckets(const BatchCostModel& mdl, int count, const int* m, const int* n, int max_batch);
// The fixed ladder of padded sizes (multiples of 32 about 1.2x apart), for comparison.
BucketPlan ladder_buckets(const BatchCostModel& mdl, int count, const int* m, const int* n, int max_batch);
// Predicted time of a set of buckets spread over mdl.streams workers (longest first onto the
// least loaded worker): the sum of the work plus the largest per-worker latency chain.
double plan_predicted_ms(const BatchCostModel& mdl, const BucketPlan& p);

// Step schedule of one bucket of B members (PQDWHFACS, pqdwhfacs.f90:359-372 per member),
// computed before any step runs: L_k of a member follows from L_0 alone, so every step's
// form and weights are known in advance.  A member steps unconditionally while
// |1 - L| > tol1 and IT <= maxit; once L has converged it takes one more step only while its
// error (measured on the device) is above TOL1^(1/3): that step is scheduled as conditional.
// Step k is the QR form when some member scheduled at k has c_k > 100.
struct QdwhSchedule {
  int steps = 0;
  std::vector<char> qr;           // per step: 1 = QR form, 0 = Cholesky form
  // per step 5 B doubles: the form's coefficient (c, or 1/sqrt(c) for the QR stack),
  // cx = b/c, cz = a - b/c (divided by sqrt(c) in the QR form), an error slot (0) and the
  // conditional flag; members not scheduled at a step get the neutral values (0 or 1, 1, 0)
  std::vector<double> table;
  std::vector<int> count;         // per member: unconditional steps
  std::vector<int> last;          // per member: its last unconditional step (-1 = none)
  std::vector<int> cond;          // per member: its conditional step (-1 = none)
  std::vector<double> l_uncond;   // per member: L after its last unconditional step
  std::vector<double> l_cond;     // per member: L after its conditional step
};
// done[b] != 0: member b takes no step (its bounds failed).
QdwhSchedule qdwh_schedule(int B, const double* l0, const char* done, double tol1, int maxit);

}  // namespace zolo
