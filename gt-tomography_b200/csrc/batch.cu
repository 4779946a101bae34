// batch.cu -- concurrent reconstruction of many independent scans.
//
// Each scan is one plan with its own buffers and its own captured CUDA graph
// (solver.cu).  Small scans do not fill a B200, so replaying the graphs of
// several scans on separate streams lets their kernels overlap; scans whose
// forward launches already fill the GPU several times over run one after
// another (measured: eight such scans at once ran 6 % slower than in
// sequence, sharing L2).  Work is assigned largest-first to the least-loaded
// stream (LPT); the assignment depends only on the items' shapes, and no
// kernel reads another item's memory, so results do not depend on the batch
// they run in.
#include <algorithm>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "cbct_internal.h"

namespace cbct {

namespace {

// Streams of the pool, per device, created on first use and kept.
std::vector<cudaStream_t>& stream_pool(int n) {
  static std::mutex mu;
  static std::vector<std::vector<cudaStream_t>> pools;
  int dev = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)pools.size() <= dev) pools.resize(dev + 1);
  auto& pool = pools[dev];
  while ((int)pool.size() < n) {
    cudaStream_t s;
    CBCT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    pool.push_back(s);
  }
  return pool;
}

// Forward-projector CTAs of the item's largest subset, in waves of a full GPU
// (148 SMs x 3 resident CTAs).  An item of several waves keeps every SM busy
// on its own; running two such items at once only makes them share L2.
double waves_of(const cbct_batch_item& it) {
  const cbct_plan* p = it.plan;
  int m = 0;
  for (int s = 0; s < p->n_subsets; ++s) m = std::max(m, p->count[s]);
  const double ctas = double((p->g.width + kTU - 1) / kTU) * ((p->g.height + kTV - 1) / kTV) * m;
  return ctas / (148.0 * 3.0);
}

constexpr double kFillWaves = 4.0;

// Work estimate of one reconstruction: forward samples + voxel-view updates.
double work_of(const cbct_batch_item& it) {
  const cbct_geometry& g = it.plan->g;
  const double passes = it.params.iterations + 1.0;
  const double rays = double(g.width) * g.height * it.plan->n_views;
  const double nvox = double(g.nx) * g.ny * g.nz;
  return passes * (rays * it.plan->gc.N + nvox * it.plan->n_views);
}

}  // namespace

void batch_osmom(const cbct_batch_item* items, int n, int n_streams, cudaStream_t caller) {
  if (n <= 0) return;
  CBCT_REQUIRE(items != nullptr, "items is NULL");
  CBCT_REQUIRE(n_streams >= 1, "n_streams must be >= 1");
  for (int i = 0; i < n; ++i) {
    CBCT_REQUIRE(items[i].plan && items[i].b && items[i].z_out, "batch item with a NULL plan or array");
    for (int j = 0; j < i; ++j) CBCT_REQUIRE(items[j].plan != items[i].plan, "batch items share a plan");
  }
  const int S = std::min(n_streams, n);
  auto& pool = stream_pool(S);
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::vector<double> work(n);
  for (int i = 0; i < n; ++i) work[i] = work_of(items[i]);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return work[a] > work[b]; });
  std::vector<double> load(S, 0.0);
  // The pool streams are non-blocking: order them after the caller's stream.
  cudaEvent_t ready;
  CBCT_CUDA(cudaEventCreateWithFlags(&ready, cudaEventDisableTiming));
  CBCT_CUDA(cudaEventRecord(ready, caller));
  for (int s = 0; s < S; ++s) CBCT_CUDA(cudaStreamWaitEvent(pool[s], ready, 0));
  CBCT_CUDA(cudaEventDestroy(ready));
  // Items that fill the GPU run one after another on stream 0; the others are
  // spread over the remaining streams (all streams when no item is that
  // large), largest first onto the least-loaded stream.
  bool any_large = false;
  for (int i = 0; i < n; ++i) any_large = any_large || waves_of(items[i]) >= kFillWaves;
  const int s_small0 = (any_large && S > 1) ? 1 : 0;
  // Plans record their graphs on first use (host-side capture); the replays
  // then run asynchronously on the pool's streams.
  for (int i : order) {
    int s = 0;
    if (!(any_large && waves_of(items[i]) >= kFillWaves))
      s = s_small0 + int(std::min_element(load.begin() + s_small0, load.end()) - (load.begin() + s_small0));
    load[s] += work[i];
    cbct_solver_params prm = items[i].params;
    prm.use_graph = 1;
    osmom_solve(items[i].plan, items[i].b, items[i].x0, items[i].z_out, prm, items[i].resid_norm2_out, pool[s]);
  }
  for (int s = 0; s < S; ++s) CBCT_CUDA(cudaStreamSynchronize(pool[s]));
  // Device-side status of every item (each plan's flag words are read and
  // cleared); the first failing item's status is returned.
  std::string first_msg;
  cbct_status first = CBCT_OK;
  for (int i = 0; i < n; ++i) {
    try {
      plan_check_flags(items[i].plan, pool[0]);
    } catch (const Error& e) {
      if (first == CBCT_OK) {
        first = e.status;
        first_msg = "batch item " + std::to_string(i) + ": " + e.what();
      }
    }
  }
  if (first != CBCT_OK) throw Error(first, first_msg);
}

}  // namespace cbct

