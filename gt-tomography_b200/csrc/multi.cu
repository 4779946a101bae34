// multi.cu -- fused batch OS-MOM: many scans advanced in lockstep through
// work-list launches.
//
// Every item is an independent osMOMSolverD reconstruction (the semantics of
// cbct_osmom_solve with FP32 storage).  The items are split into groups that
// run side by side (CBCT_FUSED_BRANCHES); step k of a group is subset
// k mod S_i of iteration k / S_i of every item of the group that has one: one work-list
// forward launch per projector kind and box width over all those items'
// residuals (after one launch for all the items' volume transposes), then one
// work-list back-projection per box width with the OS-MOM update fused in.
// An item whose own launch would fill the GPU for kMultiFillWaves waves keeps
// its one-scan launch in the same schedule.  The preconditioner is built the
// same way.  The whole schedule is captured in one CUDA graph, and the last
// one is replayed while the calls repeat.  Each work-list item runs the
// one-scan kernels' body, so every result is bitwise the one-scan solve's.
#include <algorithm>
#include <cmath>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>
#ifdef CBCT_SETUP_TIMING
#include <chrono>
#include <cstdio>
#endif

#include "cbct_internal.h"

namespace cbct {

int resident_grid(const void* func, int threads, size_t smem) {
  static std::mutex mu;
  static std::map<std::tuple<int, const void*, int, size_t>, int> cache;
  int dev = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  const auto key = std::make_tuple(dev, func, threads, smem);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(key);
    if (it != cache.end()) return it->second;
  }
  int sms = 0, nb = 0;
  CBCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CBCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, func, threads, smem));
  if (nb < 1) throw Error(CBCT_ERR_INTERNAL, "work-list kernel does not fit an SM");
  std::lock_guard<std::mutex> lock(mu);
  cache[key] = nb * sms;
  return nb * sms;
}

namespace {

struct ItemState {
  cbct_plan* p;
  const cbct_batch_item* it;
  float *xold, *D, *r;
  size_t nv, plane;
  int S, steps;
  double t = 1.0, told = 1.0;
};

// Records and instantiated graph of one fused schedule, released on every
// exit path.  The last one is kept and replayed when the next call has the
// same key: the same plans in the same states (serial, generation, device
// buffers) with the same arrays and parameters.
struct FusedRun {
  std::vector<uint64_t> key;
  std::vector<unsigned char*> dev;   // records and counters of each branch
  std::vector<cudaStream_t> cap;     // capture streams, one per branch
  std::vector<cudaEvent_t> ev;       // fork and join events of the capture
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  ~FusedRun() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    for (cudaEvent_t e : ev) cudaEventDestroy(e);
    for (cudaStream_t c : cap) cudaStreamDestroy(c);
    for (unsigned char* d : dev) cudaFree(d);
  }
};

// Branches of the fused schedule: the items are split into this many
// lockstep groups (largest work first onto the least-loaded group) whose
// schedules run side by side in the graph, so one group's launches fill the
// SMs that the other group's launch tails leave idle.
#ifndef CBCT_FUSED_BRANCHES
#define CBCT_FUSED_BRANCHES 2
#endif

// The kept schedule is replaced (and its graph and memory released) by the
// next call with another key; the last one is left to the process's exit, so
// no CUDA call runs from a static destructor after the runtime has gone.
std::mutex g_fused_mu;
FusedRun* g_fused_last = nullptr;

uint64_t bits_of(float f) {
  uint32_t u;
  std::memcpy(&u, &f, 4);
  return u;
}

std::unique_ptr<FusedRun> build_fused(std::vector<ItemState>& S, std::vector<uint64_t>&& key);

}  // namespace

void batch_osmom_fused(const cbct_batch_item* items, int n, cudaStream_t st) {
  if (n <= 0) return;
  CBCT_REQUIRE(items != nullptr, "items is NULL");
  std::vector<ItemState> S;
  S.reserve(n);
  for (int i = 0; i < n; ++i) {
    const cbct_batch_item& it = items[i];
    CBCT_REQUIRE(it.plan && it.b && it.z_out, "batch item with a NULL plan or array");
    for (int j = 0; j < i; ++j) {
      CBCT_REQUIRE(items[j].plan != it.plan, "batch items share a plan");
      CBCT_REQUIRE(items[j].z_out != it.z_out, "batch items share an output");
    }
    const cbct_solver_params& prm = it.params;
    if (prm.storage != CBCT_F32 || prm.tv_weight > 0.f || it.plan->n_bins > 1)
      throw Error(CBCT_ERR_UNSUPPORTED, "fused batch: fp32 volume storage, no bins, no regulariser");
    CBCT_REQUIRE(prm.proj_storage == CBCT_F32 || prm.proj_storage == CBCT_F16 || prm.proj_storage == CBCT_BF16,
                 "unknown projection storage type");
    CBCT_REQUIRE(prm.iterations >= 0, "iterations must be >= 0");
    ItemState s;
    s.p = it.plan;
    s.it = &it;
    s.nv = (size_t)s.p->g.nx * s.p->g.ny * s.p->g.nz;
    s.plane = (size_t)s.p->g.width * s.p->g.height;
    const size_t np = s.plane * s.p->n_views;
    float* ws = solver_workspace(s.p, 2 * s.nv + np);
    s.xold = ws;
    s.D = ws + s.nv;
    s.r = ws + 2 * s.nv;
    s.S = s.p->n_subsets;
    s.steps = prm.iterations * s.S;
    S.push_back(s);
  }

  int device = 0;
  CBCT_CUDA(cudaGetDevice(&device));
  std::vector<uint64_t> key = {(uint64_t)device, (uint64_t)n};
  for (const ItemState& s : S) {
    const cbct_plan* p = s.p;
    const cbct_solver_params& prm = s.it->params;
    for (uint64_t v : {p->serial, p->generation, (uint64_t)s.it->b, (uint64_t)s.it->x0, (uint64_t)s.it->z_out,
                       (uint64_t)s.it->resid_norm2_out, (uint64_t)prm.iterations, bits_of(prm.beta),
                       bits_of(prm.gamma), (uint64_t)prm.non_negativity, (uint64_t)prm.proj_storage,
                       (uint64_t)s.xold, (uint64_t)p->d_volT, (uint64_t)p->d_partials, (uint64_t)p->d_flags,
                       (uint64_t)p->d_views, (uint64_t)p->d_mask, (uint64_t)p->d_pweights})
      key.push_back(v);
  }
  std::lock_guard<std::mutex> lock(g_fused_mu);
  if (!g_fused_last || g_fused_last->key != key) {
    delete g_fused_last;
    g_fused_last = nullptr;
    g_fused_last = build_fused(S, std::move(key)).release();
  }
  CBCT_CUDA(cudaGraphLaunch(g_fused_last->exec, st));
  CBCT_CUDA(cudaStreamSynchronize(st));
  // Device-side status of every item; the first failing item's is returned.
  std::string first_msg;
  cbct_status first = CBCT_OK;
  for (int i = 0; i < n; ++i) {
    try {
      plan_check_flags(items[i].plan, st);
    } catch (const Error& e) {
      if (first == CBCT_OK) {
        first = e.status;
        first_msg = "batch item " + std::to_string(i) + ": " + e.what();
      }
    }
  }
  if (first != CBCT_OK) throw Error(first, first_msg);
}

namespace {

// Lockstep schedule of one group of items, appended to A.
void schedule(WorkArena& A, std::vector<ItemState*>& group) {
  std::vector<std::reference_wrapper<ItemState>> S;
  for (ItemState* p : group) S.push_back(*p);
  A.ops.push_back([&A](cudaStream_t cs) {
    CBCT_CUDA(cudaMemsetAsync(A.dev + A.counters_offset(), 0, sizeof(int) * (size_t)std::max(A.n_counters, 1), cs));
  });
  // Preconditioner: D = 1/max(A^T (W A 1), 1e-6), as cbct_osmom_solve builds it.
  int s_max = 0, k_max = 0;
  for (ItemState& s : S) {
    float* x = s.xold;
    const size_t nv = s.nv;
    A.ops.push_back([x, nv](cudaStream_t cs) { fill_launch(x, nv, 1.f, cs); });
    s_max = std::max(s_max, s.S);
    k_max = std::max(k_max, s.steps);
  }
  for (int sub = 0; sub < s_max; ++sub) {
    std::vector<MultiFwdJob> fj;
    for (ItemState& s : S)
      if (sub < s.S)
        fj.push_back(MultiFwdJob{s.p, sub, s.xold, s.r + s.plane * s.p->first[sub], nullptr, CBCT_F32,
                                 s.p->offcorr[sub], nullptr});
    forward_multi(A, fj);
  }
  {
    std::vector<MultiBpJob> bj;
    for (ItemState& s : S) bj.push_back(MultiBpJob{s.p, s.S, s.r, s.D, nullptr, nullptr, 0.f, 0.f, 0});
    backproject_multi(A, 0, bj);
  }
  // z = x0 or 0; xold = z
  for (ItemState& s : S) {
    float* z = s.it->z_out;
    float* xo = s.xold;
    const float* x0 = s.it->x0;
    const size_t bytes = s.nv * sizeof(float);
    A.ops.push_back([z, xo, x0, bytes](cudaStream_t cs) {
      if (x0) {
        CBCT_CUDA(cudaMemcpyAsync(z, x0, bytes, cudaMemcpyDeviceToDevice, cs));
        CBCT_CUDA(cudaMemcpyAsync(xo, x0, bytes, cudaMemcpyDeviceToDevice, cs));
      } else {
        CBCT_CUDA(cudaMemsetAsync(z, 0, bytes, cs));
        CBCT_CUDA(cudaMemsetAsync(xo, 0, bytes, cs));
      }
    });
  }
  // Subset steps in lockstep.
  for (int k = 0; k < k_max; ++k) {
    std::vector<MultiFwdJob> fj;
    std::vector<MultiBpJob> bj;
    for (ItemState& s : S) {
      if (k >= s.steps) continue;
      const cbct_solver_params& prm = s.it->params;
      const int it = k / s.S, sub = k % s.S;
      s.t = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * s.t * s.t));
      float* rs = s.r + s.plane * s.p->first[sub];
      const void* bs = static_cast<const char*>(s.it->b) + s.plane * s.p->first[sub] * dtype_size(prm.proj_storage);
      fj.push_back(MultiFwdJob{s.p, sub, s.it->z_out, rs, bs, prm.proj_storage, s.p->offcorr[sub],
                               s.it->resid_norm2_out ? s.it->resid_norm2_out + k : nullptr});
      const double stepsz = double(prm.beta) / (1.0 + double(prm.gamma) * it) * s.S;
      const double mom = (s.told - 1.0) / s.t;
      bj.push_back(MultiBpJob{s.p, sub, rs, s.it->z_out, s.xold, s.D, float(stepsz), float(mom),
                              prm.non_negativity});
      s.told = s.t;
    }
    forward_multi(A, fj);
    backproject_multi(A, 1, bj);
  }
}

// Work of one reconstruction: forward samples + voxel-view updates.
double item_work(const ItemState& s) {
  const cbct_geometry& g = s.p->g;
  const double passes = s.it->params.iterations + 1.0;
  return passes * (double(g.width) * g.height * s.p->n_views * s.p->gc.N + double(s.nv) * s.p->n_views);
}

// The fused schedule of the items, captured and instantiated.
std::unique_ptr<FusedRun> build_fused(std::vector<ItemState>& S, std::vector<uint64_t>&& key) {
#ifdef CBCT_SETUP_TIMING
  const auto t0 = std::chrono::steady_clock::now();
#endif
  const int nb = std::max(1, std::min<int>(CBCT_FUSED_BRANCHES, (int)S.size()));
  std::vector<int> order(S.size());
  for (size_t i = 0; i < S.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return item_work(S[a]) > item_work(S[b]); });
  std::vector<double> load(nb, 0.0);
  std::vector<std::vector<int>> idx(nb);
  for (int i : order) {
    const int b = int(std::min_element(load.begin(), load.end()) - load.begin());
    load[b] += item_work(S[i]);
    idx[b].push_back(i);
  }
  std::vector<WorkArena> A(nb);
  for (int b = 0; b < nb; ++b) {
    std::sort(idx[b].begin(), idx[b].end());
    std::vector<ItemState*> group;
    for (int i : idx[b]) group.push_back(&S[i]);
    schedule(A[b], group);
  }
#ifdef CBCT_SETUP_TIMING
  // Build-time switch: host phases of the call on stderr.
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  const auto t1 = now();
#endif
  auto run = std::make_unique<FusedRun>();
  run->key = std::move(key);
  run->dev.assign(nb, nullptr);
  run->cap.assign(nb, nullptr);
  run->ev.assign(nb, nullptr);
  for (int b = 0; b < nb; ++b) {
    CBCT_CUDA(cudaMalloc(&run->dev[b], A[b].bytes()));
    A[b].dev = run->dev[b];
    if (!A[b].host.empty())
      CBCT_CUDA(cudaMemcpy(run->dev[b], A[b].host.data(), A[b].host.size(), cudaMemcpyHostToDevice));
    CBCT_CUDA(cudaStreamCreateWithFlags(&run->cap[b], cudaStreamNonBlocking));
    CBCT_CUDA(cudaEventCreateWithFlags(&run->ev[b], cudaEventDisableTiming));
  }
  // Branch 0's stream starts the capture; the others fork from it and join
  // it at the end.
  CBCT_CUDA(cudaStreamBeginCapture(run->cap[0], cudaStreamCaptureModeThreadLocal));
  try {
    CBCT_CUDA(cudaEventRecord(run->ev[0], run->cap[0]));
    for (int b = 1; b < nb; ++b) CBCT_CUDA(cudaStreamWaitEvent(run->cap[b], run->ev[0], 0));
    for (int b = 0; b < nb; ++b)
      for (auto& op : A[b].ops) op(run->cap[b]);
    for (int b = 1; b < nb; ++b) {
      CBCT_CUDA(cudaEventRecord(run->ev[b], run->cap[b]));
      CBCT_CUDA(cudaStreamWaitEvent(run->cap[0], run->ev[b], 0));
    }
  } catch (...) {
    cudaStreamEndCapture(run->cap[0], &run->graph);
    throw;
  }
  CBCT_CUDA(cudaStreamEndCapture(run->cap[0], &run->graph));
  CBCT_CUDA(cudaGraphInstantiate(&run->exec, run->graph, 0));
#ifdef CBCT_SETUP_TIMING
  size_t nodes = 0, bytes = 0;
  cudaGraphGetNodes(run->graph, nullptr, &nodes);
  for (auto& a : A) bytes += a.host.size();
  std::fprintf(stderr, "fused: schedule %.1f ms, upload+capture+instantiate %.1f ms (%zu nodes, %zu record bytes)\n",
               ms(t0, t1), ms(t1, now()), nodes, bytes);
#endif
  return run;
}

}  // namespace

}  // namespace cbct
