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
  int streams = 4;  // worker streams the buckets are spread over
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

}  // namespace zolo
