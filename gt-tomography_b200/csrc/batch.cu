// batch.cu -- concurrent reconstruction of many independent scans.
//
// Each scan is one plan with its own buffers and its own captured CUDA graph
// (solver.cu).  Small scans do not fill a B200 (a 96^3 volume with 90 views
// launches a few thousand CTAs per kernel), so replaying the graphs of several
// scans on separate streams lets their kernels overlap.  Work is assigned
// largest-first to the least-loaded stream (LPT); the assignment depends only
// on the items' shapes, and no kernel reads another item's memory, so results
// do not depend on the batch they run in.
#include <algorithm>
#include <mutex>
#include <numeric>
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
  // Plans record their graphs on first use (host-side capture); the replays
  // then run asynchronously on the pool's streams.
  for (int i : order) {
    const int s = int(std::min_element(load.begin(), load.end()) - load.begin());
    load[s] += work[i];
    cbct_solver_params prm = items[i].params;
    prm.use_graph = 1;
    osmom_solve(items[i].plan, items[i].b, items[i].x0, items[i].z_out, prm, items[i].resid_norm2_out, pool[s]);
  }
  for (int s = 0; s < S; ++s) CBCT_CUDA(cudaStreamSynchronize(pool[s]));
}

}  // namespace cbct

