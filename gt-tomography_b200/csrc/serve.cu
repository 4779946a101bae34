// serve.cu -- serving loop: continuous batching of FDK and OS-MOM requests.
//
// A server holds `max_inflight` slots.  Each slot is a host worker thread with
// its own non-blocking CUDA stream; all slots draw device memory from one
// stream-ordered pool, so a request's set-up, copies and kernels never pass
// through cudaMalloc/cudaFree (whose implicit device synchronisation would
// serialise the slots).  Admission: a worker that becomes idle takes the
// oldest waiting request whose footprint fits into the budget left by the
// admitted ones; a request passed over kMaxBypass times blocks younger ones
// until it fits, so large requests are not starved by a stream of small ones.
//
// Per request the worker runs the reference's set-up rules
// (CBSubsetOperator::setup, CBSubsetOperator.cpp:52-115: angles shifted to
// start at 0, round-robin subsets, per-subset offset override;
// hoCuConebeamProjectionOperator::setup, .h:57-78: short scan and offset
// override), builds a plan on the slot stream, copies the projections host ->
// device in subset order (consecutive runs in one copy, as
// conebeam_projection.cu:1441-1462 does), reconstructs (FDK as
// hoCuConebeamProjectionOperator::mult_MH with FBP; OS-MOM as
// osMOMSolverD::solve), copies the volume device -> host and frees the plan
// in stream order.  Kernels of one request read only that request's buffers:
// results do not depend on what else runs.
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <unordered_map>

#include "cbct_internal.h"

namespace cbct {
namespace {

constexpr int kMaxBypass = 8;
constexpr size_t kAllocSlack = 4096;  // per-buffer rounding allowance of the estimate

struct Request {
  uint64_t id = 0;
  cbct_request r{};
  std::vector<float> angles, offsets, filter;
  size_t bytes = 0;
  double t_submit = 0, t_admit = 0, t_done = 0;
  int bypassed = 0;
  int slot = -1;
  bool done = false;
  cbct_status status = CBCT_OK;
  std::string message;
  size_t peak = 0;
};

size_t vol_bytes(const cbct_geometry& g) { return (size_t)g.nx * g.ny * g.nz * sizeof(float); }
size_t plane(const cbct_geometry& g) { return (size_t)g.width * g.height; }

void validate_request(const cbct_request& r) {
  validate_geometry(&r.geometry);
  CBCT_REQUIRE(r.kind == CBCT_REQ_FDK || r.kind == CBCT_REQ_OSMOM, "unknown request kind");
  CBCT_REQUIRE(r.n_views > 0 && r.angles_deg && r.proj_host && r.vol_host, "request with no views or a NULL array");
  CBCT_REQUIRE(r.storage == CBCT_F32 || r.storage == CBCT_F16 || r.storage == CBCT_BF16, "unknown storage type");
  CBCT_REQUIRE(r.kind == CBCT_REQ_FDK || (r.n_subsets >= 1 && r.n_subsets <= r.n_views),
               "OS-MOM request needs 1 <= n_subsets <= n_views");
  CBCT_REQUIRE(r.kind == CBCT_REQ_FDK || r.params.iterations >= 0, "iterations must be >= 0");
  CBCT_REQUIRE(r.offset_correction >= -1 && r.offset_correction <= 1, "offset_correction must be -1, 0 or 1");
}

// Device footprint: every buffer plan_alloc will hand out for this request,
// each with a rounding allowance.  Mirrors plan_create, forward_prepare,
// fdk_state, fdk_run, osmom_solve's workspace and the request's own buffers.
size_t request_bytes(const cbct_request& r) {
  const cbct_geometry& g = r.geometry;
  const size_t P = (size_t)r.n_views, pl = plane(g), nv = (size_t)g.nx * g.ny * g.nz;
  const size_t tiles = forward_tiles(g.width, g.height);
  size_t b = 0;
  int n = 0;
  auto add = [&](size_t x) { b += x; ++n; };
  add(sizeof(ViewParams) * P);
  add(sizeof(double) * std::max<size_t>(tiles * P, 148 * 4));
  add(sizeof(int) * 4);
  add(pl * P * dtype_size(r.storage));  // projections
  add(nv * sizeof(float));              // volume
  if (r.kind == CBCT_REQ_FDK) {
    size_t L = 2;
    while (L < 2 * (size_t)g.width - 1) L <<= 1;
    add(sizeof(float2) * (L / 2));
    add(sizeof(float) * L);
    add(sizeof(float) * pl);
    add(sizeof(float) * g.width * P);
    add(sizeof(float) * g.width * P);
    if (r.storage != CBCT_F32) add(sizeof(float) * pl * P);  // FP32 filtered copy
  } else {
    add(nv * sizeof(float));  // transposed volume of the forward projector (upper bound)
    add((2 * nv + pl * P) * sizeof(float));  // solver workspace (FP32 volume input)
  }
  return b + n * kAllocSlack;
}

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace
}  // namespace cbct

struct cbct_server {
  cbct_server_config cfg{};
  cudaMemPool_t pool = nullptr;
  std::vector<cudaStream_t> streams;
  std::vector<std::thread> workers;
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<std::shared_ptr<cbct::Request>> pending;
  std::unordered_map<uint64_t, std::shared_ptr<cbct::Request>> live;
  size_t in_use = 0;
  uint64_t next_id = 1;
  bool stop = false;
  std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now();
};

namespace cbct {
namespace {

// The admission rule (called with the server lock held).
std::shared_ptr<Request> admit(cbct_server* sv) {
  const size_t room = sv->cfg.hbm_budget_bytes - sv->in_use;
  for (auto it = sv->pending.begin(); it != sv->pending.end(); ++it) {
    if ((*it)->bytes <= room) {
      std::shared_ptr<Request> r = *it;
      for (auto jt = sv->pending.begin(); jt != it; ++jt) ++(*jt)->bypassed;
      sv->pending.erase(it);
      sv->in_use += r->bytes;
      return r;
    }
    if ((*it)->bypassed >= kMaxBypass) break;
  }
  return nullptr;
}

// Copies the projections into subset order: position i of the plan holds
// acquisition view order[i]; runs of consecutive views go in one copy.
void upload_views(const cbct_request& r, const std::vector<int>& order, void* dst, cudaStream_t st) {
  const size_t vb = plane(r.geometry) * dtype_size(r.storage);
  const char* src = static_cast<const char*>(r.proj_host);
  char* d = static_cast<char*>(dst);
  const int P = r.n_views;
  for (int i = 0; i < P;) {
    int n = 1;
    while (i + n < P && order[i + n] == order[i + n - 1] + 1) ++n;
    CBCT_CUDA(cudaMemcpyAsync(d + (size_t)i * vb, src + (size_t)order[i] * vb, (size_t)n * vb,
                              cudaMemcpyHostToDevice, st));
    i += n;
  }
}

void run_request(cbct_server* sv, Request& q, cudaStream_t st) {
  const cbct_request& r = q.r;
  const cbct_geometry& g = r.geometry;
  const int P = r.n_views;
  // Angles start at 0 (CBSubsetOperator.cpp:58-61; transform_angles of
  // cuConebeamProjectionOperator::setup, .cpp:157-161).
  const float amin = *std::min_element(q.angles.begin(), q.angles.end());
  std::vector<int> order(P), sizes;
  int S = 1;
  if (r.kind == CBCT_REQ_OSMOM) {
    S = r.n_subsets;
    sizes.resize(S);
    int n = 0;
    subset_partition(P, nullptr, S, order.data(), sizes.data(), &n);
  } else {
    for (int i = 0; i < P; ++i) order[i] = i;
    sizes.assign(1, P);
  }
  std::vector<float> ang(P), off(2 * (size_t)P);
  for (int i = 0; i < P; ++i) {
    ang[i] = q.angles[order[i]] - amin;
    off[2 * i] = q.offsets[2 * (size_t)order[i]];
    off[2 * i + 1] = q.offsets[2 * (size_t)order[i] + 1];
  }
  std::vector<int> offcorr(S, 0);
  for (int s = 0, f = 0; s < S; f += sizes[s], ++s) {
    if (r.offset_correction >= 0) offcorr[s] = r.offset_correction;
    else offcorr[s] = sizes[s] > 0 && offset_override_rule(g, off.data() + 2 * (size_t)f, sizes[s]);
  }
  std::unique_ptr<cbct_plan, void (*)(cbct_plan*)> plan(
      plan_create(&g, ang.data(), off.data(), P, sizes.data(), S, offcorr.data(), sv->pool, st,
                  r.kind == CBCT_REQ_OSMOM),
      plan_free);
  cbct_plan* p = plan.get();
  const float* filter = q.filter.empty() ? nullptr : q.filter.data();
  if (r.kind == CBCT_REQ_FDK) fdk_prepare(p, filter);
  void* proj = plan_alloc(p, plane(g) * P * dtype_size(r.storage));
  float* vol = static_cast<float*>(plan_alloc(p, vol_bytes(g)));
  upload_views(r, order, proj, st);
  if (r.kind == CBCT_REQ_FDK) {
    uint32_t flags = r.fdk_flags;
    if (short_scan_rule(g, ang.data(), P)) flags |= CBCT_FDK_PARKER;
    if (offcorr[0]) flags |= CBCT_FDK_OFFSET;
    float* work = r.storage == CBCT_F32 ? static_cast<float*>(proj) : nullptr;
    fdk_run(p, proj, vol, filter, flags, work, st, r.storage);
  } else {
    // Only the measured projections take the request's storage type: a 16-bit
    // copy of the volume for the forward projector saves no memory (the FP32
    // master stays) and its reads cost a conversion per tap.
    cbct_solver_params prm = r.params;
    prm.storage = CBCT_F32;
    prm.proj_storage = r.storage;
    osmom_solve(p, proj, nullptr, vol, prm, nullptr, st);
  }
  CBCT_CUDA(cudaMemcpyAsync(r.vol_host, vol, vol_bytes(g), cudaMemcpyDeviceToHost, st));
  CBCT_CUDA(cudaStreamSynchronize(st));
  q.peak = p->dev_bytes_peak;
  plan_check_flags(p, st);   // a kernel that gave up a wait or overflowed a box fails the request
}

void worker(cbct_server* sv, int slot) {
  cudaSetDevice(sv->cfg.device);
  cudaStream_t st = sv->streams[slot];
  for (;;) {
    std::shared_ptr<Request> q;
    {
      std::unique_lock<std::mutex> lk(sv->mu);
      for (;;) {
        q = admit(sv);
        if (q || (sv->stop && sv->pending.empty())) break;
        sv->cv_work.wait(lk);
      }
      if (!q) return;
      q->t_admit = seconds_since(sv->t0);
      q->slot = slot;
    }
    cbct_status status = CBCT_OK;
    std::string msg;
    try {
      run_request(sv, *q, st);
    } catch (const Error& e) {
      status = e.status;
      msg = e.what();
    } catch (const std::exception& e) {
      status = CBCT_ERR_INTERNAL;
      msg = e.what();
    }
    if (status != CBCT_OK) cudaStreamSynchronize(st);  // the plan's frees were enqueued on st
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      q->t_done = seconds_since(sv->t0);
      q->status = status;
      q->message = msg;
      q->done = true;
      sv->in_use -= q->bytes;
    }
    sv->cv_done.notify_all();
    sv->cv_work.notify_all();
  }
}

void server_destroy(cbct_server* sv) {
  {
    std::lock_guard<std::mutex> lk(sv->mu);
    sv->stop = true;
  }
  sv->cv_work.notify_all();
  for (auto& t : sv->workers)
    if (t.joinable()) t.join();
  for (cudaStream_t s : sv->streams) cudaStreamDestroy(s);
  if (sv->pool) cudaMemPoolDestroy(sv->pool);
  delete sv;
}

}  // namespace
}  // namespace cbct

using namespace cbct;

extern "C" {

cbct_status cbct_server_create(const cbct_server_config* cfg, cbct_server** out) {
  return guard([&] {
    CBCT_REQUIRE(cfg && out, "NULL argument");
    CBCT_REQUIRE(cfg->max_inflight >= 1 && cfg->max_inflight <= 64, "max_inflight must be in [1, 64]");
    CBCT_REQUIRE(cfg->hbm_budget_bytes > 0, "hbm_budget_bytes must be positive");
    *out = nullptr;
    std::unique_ptr<cbct_server, void (*)(cbct_server*)> sv(new cbct_server(), server_destroy);
    sv->cfg = *cfg;
    CBCT_CUDA(cudaSetDevice(cfg->device));
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = cfg->device;
    CBCT_CUDA(cudaMemPoolCreate(&sv->pool, &props));
    // Keep freed memory in the pool, and never let one slot's allocation wait
    // on another slot's stream (no hidden ordering between requests).
    uint64_t keep = UINT64_MAX;
    CBCT_CUDA(cudaMemPoolSetAttribute(sv->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    int no = 0;
    CBCT_CUDA(cudaMemPoolSetAttribute(sv->pool, cudaMemPoolReuseAllowInternalDependencies, &no));
    for (int i = 0; i < cfg->max_inflight; ++i) {
      cudaStream_t s;
      CBCT_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
      sv->streams.push_back(s);
    }
    for (int i = 0; i < cfg->max_inflight; ++i) sv->workers.emplace_back(worker, sv.get(), i);
    *out = sv.release();
  });
}

cbct_status cbct_server_request_bytes(const cbct_request* req, size_t* bytes_out) {
  return guard([&] {
    CBCT_REQUIRE(req && bytes_out, "NULL argument");
    validate_request(*req);
    *bytes_out = request_bytes(*req);
  });
}

cbct_status cbct_server_submit(cbct_server* sv, const cbct_request* req, uint64_t* ticket_out) {
  return guard([&] {
    CBCT_REQUIRE(sv && req && ticket_out, "NULL argument");
    validate_request(*req);
    auto q = std::make_shared<Request>();
    q->r = *req;
    const int P = req->n_views;
    q->angles.assign(req->angles_deg, req->angles_deg + P);
    if (req->offsets_xy) q->offsets.assign(req->offsets_xy, req->offsets_xy + 2 * (size_t)P);
    else q->offsets.assign(2 * (size_t)P, 0.f);
    for (int i = 0; i < P; ++i)
      CBCT_REQUIRE(std::isfinite(q->angles[i]) && std::isfinite(q->offsets[2 * i]) &&
                       std::isfinite(q->offsets[2 * i + 1]),
                   "non-finite angle or offset");
    if (req->kind == CBCT_REQ_FDK && req->filter)
      q->filter.assign(req->filter, req->filter + req->geometry.width + 1);
    q->r.angles_deg = nullptr;
    q->r.offsets_xy = nullptr;
    q->r.filter = nullptr;
    q->bytes = request_bytes(*req);
    if (q->bytes > sv->cfg.hbm_budget_bytes)
      throw Error(CBCT_ERR_BUDGET, "request needs " + std::to_string(q->bytes) + " device bytes; the budget is " +
                                       std::to_string(sv->cfg.hbm_budget_bytes));
    {
      std::lock_guard<std::mutex> lk(sv->mu);
      CBCT_REQUIRE(!sv->stop, "server is shutting down");
      q->id = sv->next_id++;
      q->t_submit = seconds_since(sv->t0);
      sv->pending.push_back(q);
      sv->live[q->id] = q;
      *ticket_out = q->id;
    }
    sv->cv_work.notify_all();
  });
}

cbct_status cbct_server_wait(cbct_server* sv, uint64_t ticket, double timeout_s, cbct_request_info* info) {
  return guard([&] {
    CBCT_REQUIRE(sv && info, "NULL argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->live.find(ticket);
    CBCT_REQUIRE(it != sv->live.end(), "unknown or already collected ticket");
    std::shared_ptr<Request> q = it->second;
    auto ready = [&] { return q->done; };
    if (timeout_s < 0) sv->cv_done.wait(lk, ready);
    else if (!sv->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), ready))
      throw Error(CBCT_ERR_TIMEOUT, "request has not completed");
    std::memset(info, 0, sizeof(*info));
    info->status = q->status;
    info->slot = q->slot;
    info->t_submit = q->t_submit;
    info->t_admit = q->t_admit;
    info->t_done = q->t_done;
    info->bytes_reserved = q->bytes;
    info->bytes_peak = q->peak;
    std::strncpy(info->message, q->message.c_str(), sizeof(info->message) - 1);
    sv->live.erase(it);
  });
}

cbct_status cbct_server_now(cbct_server* sv, double* t_out) {
  return guard([&] {
    CBCT_REQUIRE(sv && t_out, "NULL argument");
    *t_out = seconds_since(sv->t0);
  });
}

cbct_status cbct_server_destroy(cbct_server* sv) {
  return guard([&] {
    if (sv) server_destroy(sv);
  });
}

}  // extern "C"
