// abi.cu -- C ABI of the B200 cone-beam library (declared in include/cbct.h).
//
// Every entry point converts internal exceptions into a cbct_status and a
// thread-local message; nothing throws across the boundary.  Host-side setup
// logic restates the reference's operator setup (cited per function).
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>

#include "device_common.cuh"

namespace cbct {

void fdk_state_free(cbct_plan* p);
void graph_cache_free(cbct_plan* p);
void fill_launch(float* x, size_t n, float v, cudaStream_t st);
void convert_launch(const float* src, void* dst, size_t n, cbct_dtype dt, cudaStream_t st);
void backproject_recip_launch(cbct_plan* p, int s, const float* proj, float* out, cudaStream_t st);
void osmom_solve(cbct_plan* p, const void* b, const float* x0, float* z, const cbct_solver_params& prm,
                 double* resid, cudaStream_t st);
void ossart_solve(cbct_plan* p, const float* b, const float* x0, float* x, const cbct_solver_params& prm,
                  double* cost, cudaStream_t st);
void fdk_run(cbct_plan* p, const void* proj, float* vol, const float* filter, uint32_t flags, float* work,
             cudaStream_t st, cbct_dtype proj_dtype);
void phantom_voxelize_launch(const GridConst& gc, const float* ell, int K, int ss, float* vol, cudaStream_t st);
void phantom_project_launch(cbct_plan* p, int s, const float* ell, int K, float* proj, cudaStream_t st);
void batch_osmom(const cbct_batch_item* items, int n, int n_streams, cudaStream_t caller);

std::string& last_error_slot() {
  static thread_local std::string msg;
  return msg;
}

void ensure_smem_attr(const void* func, size_t bytes) {
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, size_t> done;
  // The 48 KB default covers static plus dynamic shared memory, so the limit
  // is raised for any dynamic size (once per kernel, device and size).
  if (bytes == 0) return;
  int dev = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lk(mu);
  size_t& cur = done[{dev, func}];
  if (cur >= bytes) return;
  CBCT_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
  cur = bytes;
}

void* plan_alloc(cbct_plan* p, size_t bytes) {
  if (bytes == 0) return nullptr;
  void* ptr = nullptr;
  if (p->pool) CBCT_CUDA(cudaMallocFromPoolAsync(&ptr, bytes, p->pool, p->pool_stream));
  else CBCT_CUDA(cudaMalloc(&ptr, bytes));
  p->allocs.emplace_back(ptr, bytes);
  p->dev_bytes += bytes;
  p->dev_bytes_peak = std::max(p->dev_bytes_peak, p->dev_bytes);
  return ptr;
}

void plan_dealloc(cbct_plan* p, void* ptr) {
  if (!ptr) return;
  for (size_t i = 0; i < p->allocs.size(); ++i) {
    if (p->allocs[i].first != ptr) continue;
    p->dev_bytes -= p->allocs[i].second;
    p->allocs.erase(p->allocs.begin() + i);
    if (p->pool) cudaFreeAsync(ptr, p->pool_stream);
    else cudaFree(ptr);
    return;
  }
}

void plan_upload(cbct_plan* p, void* dst, const void* src, size_t bytes) {
  if (bytes == 0) return;
  if (p->pool) {
    // Stream-ordered after the pool allocation; the host buffer may go away
    // when this returns, so wait for the copy (plan set-up only).
    CBCT_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, p->pool_stream));
    CBCT_CUDA(cudaStreamSynchronize(p->pool_stream));
  } else {
    CBCT_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyHostToDevice));
  }
}

void plan_memset(cbct_plan* p, void* dst, int value, size_t bytes) {
  if (bytes == 0) return;
  if (p->pool) CBCT_CUDA(cudaMemsetAsync(dst, value, bytes, p->pool_stream));
  else CBCT_CUDA(cudaMemset(dst, value, bytes));
}

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* ptr = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(ptr);
  });
  if (!fn) throw Error(CBCT_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the driver");
  return fn;
}

// hoCuConebeamProjectionOperator::compute_default_frequency_filter
// (hoCuConebeamProjectionOperator.cpp:26-62): Guo et al. filter on W+1 bins,
// evaluated in float, normalised to an absolute sum of W+1.
void default_filter(int W, float* out) {
  const int K = W + 1;
  const float A2 = float(0.2 * double(K) * double(K));
  double sum = 0.0;
  for (int i = 0; i < K; ++i) {
    const float k = float(i);
    out[i] = (k * k < A2) ? k * A2 / (A2 - k * k) * std::exp(-A2 / (A2 - k * k)) : 0.f;
    sum += std::fabs(double(out[i]));
  }
  for (int i = 0; i < K; ++i) out[i] = float(double(out[i]) * (double(K) / sum));
}

// CBSubsetOperator<ARRAY>::setup, CBSubsetOperator.cpp:66-104.
void subset_partition(int n_views, const int* view_bin, int n_subsets, int* order, int* sizes, int* n_out) {
  std::map<unsigned, unsigned> bins;
  for (int i = 0; i < n_views; ++i) {
    const int b = view_bin ? view_bin[i] : 0;
    if (b >= 0) bins[(unsigned)i] = (unsigned)b;
  }
  std::vector<std::vector<unsigned>> sub(n_subsets);
  int k = 0;
  for (int i = 0; i < n_views; ++i)
    if (bins.find((unsigned)i) != bins.end()) sub[k++ % n_subsets].push_back((unsigned)i);
  for (auto& s : sub)
    std::sort(s.begin(), s.end(), [&](unsigned a, unsigned b) { return bins[a] < bins[b]; });
  int n = 0;
  for (int s = 0; s < n_subsets; ++s) {
    sizes[s] = (int)sub[s].size();
    for (unsigned v : sub[s]) order[n++] = (int)v;
  }
  *n_out = n;
}

// Short-scan test of cuConebeamProjectionOperator::setup (.cpp:166-174) and
// hoCuConebeamProjectionOperator::setup (.h:57-66), in float as there: the
// largest angle (angles start at 0) against pi + 3 delta.
bool short_scan_rule(const cbct_geometry& g, const float* angles, int n) {
  const float span = *std::max_element(angles, angles + n);
  const float delta = std::atan(g.fov_u / (2.0f * g.SDD));
  const float pi = 3.14159265358979f;
  return !(span * pi / 180.0f > pi + 3.0f * delta);
}

// Offset-correction override (cuConebeamProjectionOperator.cpp:176-181,
// hoCuConebeamProjectionOperator.h:72-76): |mean offset_x| > 0.1 fov_u.
bool offset_override_rule(const cbct_geometry& g, const float* offsets, int n) {
  float mx = 0.f;
  for (int i = 0; i < n; ++i) mx += offsets[2 * i];
  mx /= float(n);
  return std::fabs(mx) > g.fov_u * 0.1f;
}

void validate_geometry(const cbct_geometry* g) {
  CBCT_REQUIRE(g != nullptr, "geometry is NULL");
  CBCT_REQUIRE(g->width > 0 && g->height > 0, "detector size must be positive");
  CBCT_REQUIRE(g->nx > 0 && g->ny > 0 && g->nz > 0, "volume size must be positive");
  CBCT_REQUIRE(g->lx > 0 && g->ly > 0 && g->lz > 0, "volume size in mm must be positive");
  CBCT_REQUIRE(g->fov_u > 0 && g->fov_v > 0, "detector size in mm must be positive");
  CBCT_REQUIRE(g->SAD > 0 && g->SDD > g->SAD, "need 0 < SAD < SDD");
  CBCT_REQUIRE(g->samples_per_pixel > 0, "samples_per_pixel must be positive");
  CBCT_REQUIRE((long)(g->samples_per_pixel * float(g->nx)) >= 1, "fewer than one sample per ray");
}

static GridConst make_grid(const cbct_geometry& g) {
  GridConst c{};
  c.nx = g.nx; c.ny = g.ny; c.nz = g.nz;
  c.W = g.width; c.H = g.height;
  c.N = (int)(g.samples_per_pixel * float(g.nx));  // conebeam_projection.cu:625
  c.hx = g.lx * 0.5f; c.hy = g.ly * 0.5f; c.hz = g.lz * 0.5f;
  c.kx = float(double(g.nx) / g.lx); c.ky = float(double(g.ny) / g.ly); c.kz = float(double(g.nz) / g.lz);
  c.bx = g.nx * 0.5f - 0.5f; c.by = g.ny * 0.5f - 0.5f; c.bz = g.nz * 0.5f - 0.5f;
  c.vx = float(double(g.lx) / g.nx); c.vy = float(double(g.ly) / g.ny); c.vz = float(double(g.lz) / g.nz);
  c.SAD = g.SAD; c.SDD = g.SDD;
  c.fov_u = g.fov_u; c.fov_v = g.fov_v;
  c.ku = float(double(g.width) / g.fov_u); c.kv = float(double(g.height) / g.fov_v);
  c.bu = g.width * 0.5f - 0.5f; c.bv = g.height * 0.5f - 0.5f;
  c.invN = 1.f / float(c.N);
  c.wait_limit = kWaitLimit;
  return c;
}

// Per-view constants in FP64 (conebeam_projection.cu:441-473 restated so the
// detector point is affine in the pixel indices).
static ViewParams make_view(const cbct_geometry& g, double angle_deg, double ox, double oy) {
  const double pi = 3.14159265358979323846;
  const double th = angle_deg * (pi / 180.0);
  const double cs = std::cos(th), sn = std::sin(th);
  const double SAD = g.SAD, SDD = g.SDD, ADD = SDD - SAD;
  const double du = double(g.fov_u) / g.width, dv = double(g.fov_v) / g.height;
  const double q0 = (0.5 / g.width - 0.5) * g.fov_u + ox;
  const double r0 = (0.5 / g.height - 0.5) * g.fov_v + oy;
  const double Sx = SAD * sn, Sy = -SAD * cs;
  ViewParams v{};
  v.cs = float(cs); v.sn = float(sn);
  v.Sx = float(Sx); v.Sy = float(Sy);
  v.D0x = float(cs * q0 - sn * ADD - Sx);
  v.D0y = float(sn * q0 + cs * ADD - Sy);
  v.D0z = float(r0);
  v.Eux = float(cs * du); v.Euy = float(sn * du);
  v.Evz = float(dv);
  v.ox = float(ox); v.oy = float(oy);
  // central ray direction is R (0,1,0) = (-sn, cs, 0)
  if (std::fabs(cs) >= std::fabs(sn)) { v.dom = 1; v.dsgn = cs >= 0 ? 1 : -1; }
  else { v.dom = 0; v.dsgn = -sn >= 0 ? 1 : -1; }
  return v;
}

void plan_free(cbct_plan* p) {
  if (!p) return;
  fdk_state_free(p);
  graph_cache_free(p);
  while (!p->allocs.empty()) plan_dealloc(p, p->allocs.back().first);
  delete p;
}

cbct_plan* plan_create(const cbct_geometry* g, const float* angles, const float* offsets, int n_views,
                       const int* subset_sizes, int n_subsets, const int* offcorr, cudaMemPool_t pool,
                       cudaStream_t pool_stream, bool forward_buffers) {
  validate_geometry(g);
  CBCT_REQUIRE(n_views > 0, "n_views must be positive");
  CBCT_REQUIRE(angles && offsets, "angles/offsets are NULL");
  CBCT_REQUIRE(n_subsets >= 1, "n_subsets must be >= 1");
  CBCT_REQUIRE(n_subsets == 1 || subset_sizes, "subset_sizes is NULL with several subsets");
  static std::atomic<uint64_t> serials{0};
  std::unique_ptr<cbct_plan, void (*)(cbct_plan*)> p(new cbct_plan(), plan_free);
  p->serial = ++serials;
  p->g = *g;
  p->gc = make_grid(*g);
  p->n_views = n_views;
  p->n_subsets = n_subsets;
  int acc = 0;
  for (int s = 0; s < n_subsets; ++s) {
    const int c = subset_sizes ? subset_sizes[s] : n_views;
    CBCT_REQUIRE(c >= 0, "negative subset size");
    p->first.push_back(acc);
    p->count.push_back(c);
    p->offcorr.push_back(offcorr ? (offcorr[s] != 0) : 0);
    acc += c;
    p->max_subset = std::max(p->max_subset, c);
  }
  CBCT_REQUIRE(acc == n_views, "subset sizes do not sum to n_views");
  // index n_subsets addresses every view
  p->first.push_back(0);
  p->count.push_back(n_views);
  p->offcorr.push_back(0);
  p->seg_begin.assign(n_subsets, 0);
  p->seg_end.assign(n_subsets, 0);
  p->seg_bin.assign(n_subsets + 1, -1);
  p->angles.assign(angles, angles + n_views);
  p->offsets.assign(offsets, offsets + 2 * (size_t)n_views);
  for (int i = 0; i < n_views; ++i) {
    CBCT_REQUIRE(std::isfinite(angles[i]) && std::isfinite(offsets[2 * i]) && std::isfinite(offsets[2 * i + 1]),
                 "non-finite angle or offset");
    p->hviews.push_back(make_view(*g, angles[i], offsets[2 * i], offsets[2 * i + 1]));
  }
  CBCT_CUDA(cudaGetDevice(&p->device));
  p->pool = pool;
  p->pool_stream = pool_stream;
  p->d_views = plan_alloc_n<ViewParams>(p.get(), n_views);
  plan_upload(p.get(), p->d_views, p->hviews.data(), sizeof(ViewParams) * n_views);
  const size_t tiles = forward_tiles(g->width, g->height);
  p->n_partials = std::max<size_t>(tiles * n_views, 148 * 4);
  p->d_partials = plan_alloc_n<double>(p.get(), p->n_partials);
  p->d_flags = plan_alloc_n<int>(p.get(), 4);
  plan_memset(p.get(), p->d_flags, 0, sizeof(int) * 4);
  // Plans that never project forward skip the box sizing (a host loop over
  // every view, tile and slab); a forward call on them takes the gather kernel.
  if (!forward_buffers) p->fwd_pref = 2;
#ifdef CBCT_SETUP_TIMING
  // Build-time switch: the set-up phases' host times on stderr.
  auto now = [] { return std::chrono::steady_clock::now(); };
  auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };
  const auto t0 = now();
  forward_choose_variant(p.get());
  const auto t1 = now();
  if (forward_buffers) forward_prepare(p.get());
  const auto t2 = now();
  backproject_choose_variant(p.get());
  const auto t3 = now();
  backproject_prepare(p.get());
  const auto t4 = now();
  std::fprintf(stderr, "plan set-up ms: forward_choose %.1f forward_prepare %.1f bp_choose %.1f bp_prepare %.1f\n",
               ms(t0, t1), ms(t1, t2), ms(t2, t3), ms(t3, t4));
#else
  forward_choose_variant(p.get());
  if (forward_buffers) forward_prepare(p.get());
  backproject_choose_variant(p.get());
  backproject_prepare(p.get());
#endif
  return p.release();
}

bool stream_capturing(cudaStream_t st) {
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cs) != cudaSuccess) {
    // Querying the legacy stream while another stream captures in global mode
    // is itself refused: treat that as capturing (no synchronisation allowed).
    (void)cudaGetLastError();
    return true;
  }
  return cs != cudaStreamCaptureStatusNone;
}

void plan_check_flags(cbct_plan* p, cudaStream_t st) {
  int h[4] = {0, 0, 0, 0};
  CBCT_CUDA(cudaMemcpyAsync(h, p->d_flags, sizeof(h), cudaMemcpyDeviceToHost, st));
  CBCT_CUDA(cudaStreamSynchronize(st));
  if (h[0] == 0 && h[1] == 0) return;
  CBCT_CUDA(cudaMemsetAsync(p->d_flags, 0, sizeof(h), st));
  CBCT_CUDA(cudaStreamSynchronize(st));
  if (h[1] != 0)
    throw Error(CBCT_ERR_TIMEOUT, std::to_string(h[1]) + " thread block(s) gave up a bounded wait for a TMA stage "
                                  "(their rays or voxels are incomplete); " + std::to_string(h[0]) +
                                  " range-check event(s)");
  throw Error(CBCT_ERR_DEVICE_CHECK, std::to_string(h[0]) + " device range-check event(s): a footprint did not fit "
                                     "its shared-memory box or an index left its range; results are incomplete");
}

// The solve and FDK entry points report the device flags on return unless the
// caller turned that off or is capturing the stream.
static void check_on_return(cbct_plan* p, cudaStream_t st) {
  if (p->status_check && !stream_capturing(st)) plan_check_flags(p, st);
}

static int subset_index(const cbct_plan* p, int s) {
  CBCT_REQUIRE(p != nullptr, "plan is NULL");
  CBCT_REQUIRE(s >= -1 && s < p->n_subsets, "subset index out of range");
  return s < 0 ? p->n_subsets : s;
}

static void require_one_bin(const cbct_plan* p, const char* what) {
  if (p->n_bins > 1) throw Error(CBCT_ERR_UNSUPPORTED, std::string(what) + " does not take a binned plan");
}

static float* proj_scratch(cbct_plan* p, size_t elems) {
  if (p->proj_scratch_elems < elems) {
    plan_dealloc(p, p->d_proj_scratch);
    p->d_proj_scratch = nullptr;
    p->proj_scratch_elems = 0;
    p->d_proj_scratch = plan_alloc_n<float>(p, elems);
    p->proj_scratch_elems = elems;
  }
  return p->d_proj_scratch;
}

static cudaStream_t S(void* s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace cbct

using namespace cbct;

extern "C" {

const char* cbct_status_string(cbct_status s) {
  switch (s) {
    case CBCT_OK: return "CBCT_OK";
    case CBCT_ERR_INVALID_ARGUMENT: return "CBCT_ERR_INVALID_ARGUMENT";
    case CBCT_ERR_CUDA: return "CBCT_ERR_CUDA";
    case CBCT_ERR_OUT_OF_MEMORY: return "CBCT_ERR_OUT_OF_MEMORY";
    case CBCT_ERR_UNSUPPORTED: return "CBCT_ERR_UNSUPPORTED";
    case CBCT_ERR_DEVICE_CHECK: return "CBCT_ERR_DEVICE_CHECK";
    case CBCT_ERR_TIMEOUT: return "CBCT_ERR_TIMEOUT";
    case CBCT_ERR_BUDGET: return "CBCT_ERR_BUDGET";
    case CBCT_ERR_CANCELLED: return "CBCT_ERR_CANCELLED";
    case CBCT_ERR_INTERNAL: return "CBCT_ERR_INTERNAL";
  }
  return "CBCT_ERR_UNKNOWN";
}

const char* cbct_last_error(void) { return last_error_slot().c_str(); }
const char* cbct_version(void) { return "gt-tomography_b200 0.1 (sm_100a)"; }

cbct_status cbct_subset_partition(int32_t n_views, const int32_t* view_bin, int32_t n_subsets, int32_t* order_out,
                                  int32_t* subset_sizes_out, int32_t* n_out) {
  return guard([&] {
    CBCT_REQUIRE(n_views >= 0 && n_subsets >= 1, "bad sizes");
    CBCT_REQUIRE(order_out && subset_sizes_out && n_out, "NULL output");
    subset_partition(n_views, view_bin, n_subsets, order_out, subset_sizes_out, n_out);
  });
}

cbct_status cbct_default_frequency_filter(int32_t W, float* out) {
  return guard([&] {
    CBCT_REQUIRE(W > 0 && out, "bad arguments");
    default_filter(W, out);
  });
}

cbct_status cbct_cosine_weights(const cbct_geometry* g, float* out) {
  return guard([&] {
    validate_geometry(g);
    CBCT_REQUIRE(out, "NULL output");
    const double SAD = g->SAD, SDD = g->SDD;
    for (int y = 0; y < g->height; ++y)
      for (int x = 0; x < g->width; ++x) {
        const double xx = (double(x) / g->width - 0.5) * g->fov_u, yy = (double(y) / g->height - 0.5) * g->fov_v;
        const double s = SAD * xx / SDD, v = SAD * yy / SDD;
        out[(size_t)y * g->width + x] = float(SAD / std::sqrt(SAD * SAD + s * s + v * v));
      }
  });
}

cbct_status cbct_is_short_scan(const cbct_geometry* g, const float* angles, int32_t n, int32_t* out) {
  return guard([&] {
    CBCT_REQUIRE(g && angles && out && n > 0, "bad arguments");
    *out = short_scan_rule(*g, angles, n) ? 1 : 0;
  });
}

cbct_status cbct_offset_override(const cbct_geometry* g, const float* offsets, int32_t n, int32_t* out) {
  return guard([&] {
    CBCT_REQUIRE(g && offsets && out && n > 0, "bad arguments");
    *out = offset_override_rule(*g, offsets, n) ? 1 : 0;
  });
}

cbct_status cbct_plan_create(const cbct_geometry* g, const float* angles_deg, const float* offsets_xy,
                             int32_t n_views, const int32_t* subset_sizes, int32_t n_subsets,
                             const int32_t* offset_correction, cbct_plan** plan_out) {
  return guard([&] {
    CBCT_REQUIRE(plan_out, "plan_out is NULL");
    *plan_out = nullptr;
    *plan_out = plan_create(g, angles_deg, offsets_xy, n_views, subset_sizes, n_subsets, offset_correction, nullptr,
                            nullptr, true);
  });
}

cbct_status cbct_plan_destroy(cbct_plan* plan) {
  return guard([&] { plan_free(plan); });
}

cbct_status cbct_plan_subset(const cbct_plan* plan, int32_t s, int32_t* first_out, int32_t* count_out) {
  return guard([&] {
    const int i = subset_index(plan, s);
    if (first_out) *first_out = plan->first[i];
    if (count_out) *count_out = plan->count[i];
  });
}

const char* cbct_plan_forward_variant(const cbct_plan* plan) {
  if (!plan) return "";
  return plan->fwd_variant == 4   ? "tma-quad"
         : plan->fwd_variant == 3 ? "tma-pair"
         : plan->fwd_variant == 2 ? "tma-fan"
         : plan->fwd_variant == 1 ? "tma-slab"
                                  : "gather";
}

cbct_status cbct_plan_set_option(cbct_plan* plan, int32_t option, int32_t value) {
  return guard([&] {
    CBCT_REQUIRE(plan, "plan is NULL");
    if (option == CBCT_OPT_DEBUG_CHECKS) {
      plan->debug_checks = value != 0;
    } else if (option == CBCT_OPT_WAIT_LIMIT) {
      CBCT_REQUIRE(value >= 0, "the wait limit must be >= 0 polls");
      plan->gc.wait_limit = (unsigned)value;
      graph_cache_free(plan);   // captured graphs hold the kernels' old constants
    } else if (option == CBCT_OPT_STATUS_CHECK) {
      plan->status_check = value != 0;
    } else if (option == CBCT_OPT_FORCE_GATHER || option == CBCT_OPT_FORWARD_KERNEL) {
      if (option == CBCT_OPT_FORCE_GATHER) plan->force_gather = value != 0;
      else {
        CBCT_REQUIRE(value >= 0 && value <= 5, "forward kernel must be 0 (automatic), 1 (slab), 2 (gather), 3 (fan), "
                                              "4 (row pairs) or 5 (row quads)");
        plan->fwd_pref = value;
      }
      graph_cache_free(plan);
      forward_choose_variant(plan);
      forward_prepare(plan);
      backproject_choose_variant(plan);
      backproject_prepare(plan);
    } else {
      throw Error(CBCT_ERR_INVALID_ARGUMENT, "unknown option");
    }
  });
}

cbct_status cbct_plan_autotune(cbct_plan* plan, float* times_ms_out, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(plan && times_ms_out, "NULL argument");
    plan_autotune(plan, times_ms_out, S(stream));
  });
}

cbct_status cbct_plan_check(cbct_plan* plan, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(plan, "plan is NULL");
    plan_check_flags(plan, S(stream));
  });
}

cbct_status cbct_microbench_interp(int32_t kind, int32_t groups, double* rate_out, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(kind == 2 || kind == 3, "kind must be 3 (trilinear) or 2 (bilinear)");
    CBCT_REQUIRE(groups >= 1 && rate_out, "bad arguments");
    *rate_out = microbench_interp(kind, groups, 5, S(stream));
  });
}

cbct_status cbct_plan_read_flags(cbct_plan* plan, int32_t* flags_out, int32_t reset) {
  return guard([&] {
    CBCT_REQUIRE(plan && flags_out, "bad arguments");
    CBCT_CUDA(cudaDeviceSynchronize());
    int h[4];
    CBCT_CUDA(cudaMemcpy(h, plan->d_flags, sizeof(h), cudaMemcpyDeviceToHost));
    flags_out[0] = h[0];
    flags_out[1] = h[1];
    if (reset) CBCT_CUDA(cudaMemset(plan->d_flags, 0, sizeof(h)));
  });
}

// Segments (view ranges of one bin) of subset i, or of every subset for the
// all-views entry, in view order.
static std::vector<int> segments_of(const cbct_plan* p, int i) {
  std::vector<int> ks;
  const int s0 = i < p->n_subsets ? i : 0, s1 = i < p->n_subsets ? i + 1 : p->n_subsets;
  for (int s = s0; s < s1; ++s)
    for (int k = p->seg_begin[s]; k < p->seg_end[s]; ++k) ks.push_back(k);
  return ks;
}

cbct_status cbct_forward(cbct_plan* plan, int32_t s, cbct_dtype vol_dtype, const void* vol, float* proj,
                         int32_t accumulate, void* stream) {
  return guard([&] {
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(vol && proj, "NULL array");
    if (plan->n_bins > 1) {
      // Each bin's views project that bin's volume (cuConebeamProjectionOperator.cpp:49-78).
      const size_t plane = (size_t)plan->g.width * plan->g.height;
      const size_t vb = (size_t)plan->g.nx * plan->g.ny * plan->g.nz * dtype_size(vol_dtype);
      for (int k : segments_of(plan, i))
        forward_launch(plan, k, vol_dtype, static_cast<const char*>(vol) + vb * plan->seg_bin[k],
                       proj + plane * (plan->first[k] - plan->first[i]), nullptr, 1.f, 0, 0, accumulate, nullptr,
                       S(stream));
      return;
    }
    forward_launch(plan, i, vol_dtype, vol, proj, nullptr, 1.f, 0, 0, accumulate, nullptr, S(stream));
  });
}

// mult_MH of one view range (a subset, a bin segment, or every view: i =
// n_subsets) into one volume.
static void backproject_range(cbct_plan* plan, int i, const float* proj, float* vol, uint32_t flags,
                              int32_t use_plan_offset, int32_t accumulate, cudaStream_t st) {
  const size_t plane = (size_t)plan->g.width * plan->g.height;
  const bool single = i != plan->n_subsets;
  // Which views get the Wang weight: every view of the call with the explicit
  // flag, else the subsets whose offset correction is on (all subsets, s = -1).
  auto weighted = [&](int k) {
    return (flags & CBCT_BP_OFFSET_WEIGHT) != 0 || (use_plan_offset && plan->offcorr[k] != 0);
  };
  bool any = plan->d_pweights != nullptr || (flags & CBCT_BP_OFFSET_WEIGHT) != 0;
  if (!any && use_plan_offset) {
    if (single) any = weighted(i);
    else for (int k = 0; k < plan->n_subsets; ++k) any = any || weighted(k);
  }
  const float* in = proj;
  if (any) {
    // mult_MH works on a weighted copy of its input (CBSubsetWeightOperator.h:44-49,
    // cuConebeamProjectionOperator.cpp:101-102); the input itself is not modified.
    float* w = proj_scratch(plan, plane * plan->count[i]);
    const int k0 = single ? i : 0, k1 = single ? i + 1 : plan->n_subsets;
    for (int k = k0; k < k1; ++k) {
      const size_t o = single ? 0 : plane * plan->first[k];
      const size_t n = plane * plan->count[k];
      if (n == 0) continue;
      const float* src = proj + o;
      if (plan->d_pweights) {
        mul_launch(w + o, src, plan->d_pweights + plane * plan->first[k], n, st);
        src = w + o;
      }
      const bool off = weighted(k);
      if (off) offset_weight_launch(plan, k, src, w + o, 0, st);
      else if (src != w + o) CBCT_CUDA(cudaMemcpyAsync(w + o, src, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
    }
    in = w;
  }
  backproject_launch(plan, i, in, vol, (flags & CBCT_BP_FDK_WEIGHT) ? 1 : 0, accumulate, 1.f, st);
}

cbct_status cbct_backproject(cbct_plan* plan, int32_t s, const float* proj, float* vol, uint32_t flags,
                             int32_t use_plan_offset, int32_t accumulate, void* stream) {
  return guard([&] {
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(vol && proj, "NULL array");
    CBCT_REQUIRE((flags & ~(CBCT_BP_OFFSET_WEIGHT | CBCT_BP_FDK_WEIGHT)) == 0, "unknown flags");
    if (plan->n_bins > 1) {
      // Every bin's volume receives its own views; a bin without views in the
      // call is cleared unless accumulating (cuConebeamProjectionOperator.cpp:82-116).
      const size_t plane = (size_t)plan->g.width * plan->g.height;
      const size_t nv = (size_t)plan->g.nx * plan->g.ny * plan->g.nz;
      std::vector<int> seen(plan->n_bins, 0);
      for (int k : segments_of(plan, i)) {
        const int b = plan->seg_bin[k];
        backproject_range(plan, k, proj + plane * (plan->first[k] - plan->first[i]), vol + nv * b, flags,
                          use_plan_offset, accumulate || seen[b], S(stream));
        seen[b] = 1;
      }
      for (int b = 0; b < plan->n_bins; ++b)
        if (!seen[b] && !accumulate) CBCT_CUDA(cudaMemsetAsync(vol + nv * b, 0, nv * sizeof(float), S(stream)));
      return;
    }
    backproject_range(plan, i, proj, vol, flags, use_plan_offset, accumulate, S(stream));
  });
}

cbct_status cbct_plan_set_bins(cbct_plan* plan, int32_t n_bins, const int32_t* view_bin) {
  return guard([&] {
    CBCT_REQUIRE(plan, "plan is NULL");
    const int S = plan->n_subsets;
    // Back to the subsets and the all-views entry.
    plan->first.resize(S + 1);
    plan->count.resize(S + 1);
    plan->offcorr.resize(S + 1);
    plan->seg_begin.assign(S, 0);
    plan->seg_end.assign(S, 0);
    plan->seg_bin.assign(S + 1, -1);
    plan->n_bins = 1;
    graph_cache_free(plan);
    if (view_bin && n_bins > 1) {
      for (int v = 0; v < plan->n_views; ++v)
        CBCT_REQUIRE(view_bin[v] >= 0 && view_bin[v] < n_bins, "view bin out of range");
      for (int s = 0; s < S; ++s) {
        plan->seg_begin[s] = (int)plan->first.size();
        std::vector<int> used(n_bins, 0);
        for (int i = 0; i < plan->count[s];) {
          const int v = plan->first[s] + i, b = view_bin[v];
          int n = 1;
          while (i + n < plan->count[s] && view_bin[v + n] == b) ++n;
          // CBSubsetOperator::setup sorts each subset by bin (CBSubsetOperator.cpp:86-87).
          CBCT_REQUIRE(!used[b], "the views of a bin must be contiguous within each subset");
          used[b] = 1;
          plan->first.push_back(v);
          plan->count.push_back(n);
          plan->offcorr.push_back(plan->offcorr[s]);
          plan->seg_bin.push_back(b);
          i += n;
        }
        plan->seg_end[s] = (int)plan->first.size();
      }
      plan->n_bins = n_bins;
    }
    forward_choose_variant(plan);
    forward_prepare(plan);
  });
}

cbct_status cbct_plan_set_projection_weights(cbct_plan* plan, const float* weights) {
  return guard([&] {
    CBCT_REQUIRE(plan, "plan is NULL");
    plan->d_pweights = weights;
    graph_cache_free(plan);   // captured solver graphs hold the old pointer
  });
}

cbct_status cbct_offset_correct(cbct_plan* plan, int32_t s, float* proj, int32_t variant, void* stream) {
  return guard([&] {
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(proj, "NULL array");
    CBCT_REQUIRE(variant == 0 || variant == 1, "variant must be 0 or 1");
    offset_weight_launch(plan, i, proj, proj, variant, S(stream));
  });
}

cbct_status cbct_fdk_filter(cbct_plan* plan, int32_t s, const float* proj_in, float* proj_out, const float* filter,
                            uint32_t flags, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_fdk_filter");
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(proj_in && proj_out, "NULL array");
    fdk_filter_launch(plan, i, proj_in, proj_out, filter, flags, S(stream));
  });
}

cbct_status cbct_fdk(cbct_plan* plan, const float* proj, float* vol, const float* filter, uint32_t flags,
                     float* work, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_fdk");
    CBCT_REQUIRE(plan && proj && vol, "NULL argument");
    fdk_run(plan, proj, vol, filter, flags, work, S(stream), CBCT_F32);
    check_on_return(plan, S(stream));
  });
}

static void require_dtype(cbct_dtype dt) {
  CBCT_REQUIRE(dt == CBCT_F32 || dt == CBCT_F16 || dt == CBCT_BF16, "unknown storage type");
}

cbct_status cbct_fdk_filter_ex(cbct_plan* plan, int32_t s, cbct_dtype proj_dtype, const void* proj_in,
                               float* proj_out, const float* filter, uint32_t flags, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_fdk_filter_ex");
    const int i = subset_index(plan, s);
    require_dtype(proj_dtype);
    CBCT_REQUIRE(proj_in && proj_out, "NULL array");
    CBCT_REQUIRE(proj_dtype == CBCT_F32 || (const void*)proj_out != proj_in,
                 "a 16-bit input cannot be filtered in place");
    fdk_filter_launch(plan, i, proj_in, proj_out, filter, flags, S(stream), proj_dtype);
  });
}

cbct_status cbct_fdk_ex(cbct_plan* plan, cbct_dtype proj_dtype, const void* proj, float* vol, const float* filter,
                        uint32_t flags, float* work, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_fdk_ex");
    CBCT_REQUIRE(plan && proj && vol, "NULL argument");
    require_dtype(proj_dtype);
    CBCT_REQUIRE(proj_dtype == CBCT_F32 || (const void*)work != proj, "a 16-bit input cannot be filtered in place");
    fdk_run(plan, proj, vol, filter, flags, work, S(stream), proj_dtype);
    check_on_return(plan, S(stream));
  });
}

cbct_status cbct_spacecarver(cbct_plan* plan, int32_t s, const float* proj, float limit, uint8_t* mask,
                             int32_t combine, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_spacecarver");
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(proj && mask, "NULL array");
    spacecarver_launch(plan, i, proj, limit, mask, combine, S(stream));
  });
}

cbct_status cbct_apply_mask(float* vol, const uint8_t* mask, size_t n, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(vol && mask, "NULL array");
    apply_mask_launch(vol, mask, n, S(stream));
  });
}

cbct_status cbct_plan_set_mask(cbct_plan* plan, const uint8_t* mask) {
  return guard([&] {
    CBCT_REQUIRE(plan, "plan is NULL");
    plan->d_mask = mask;
    // A captured solver graph holds the old mask pointer; drop it.
    graph_cache_free(plan);
  });
}

cbct_status cbct_forward_residual(cbct_plan* plan, int32_t s, cbct_dtype vol_dtype, const void* vol, const float* b,
                                  float* r, float scale, int32_t apply_offset, double* norm2_out, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_forward_residual");
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(vol && b && r, "NULL array");
    forward_launch(plan, i, vol_dtype, vol, r, b, scale, 1, apply_offset, 0, norm2_out, S(stream));
  });
}

cbct_status cbct_osmom_precon(cbct_plan* plan, float* precon_out, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_osmom_precon");
    CBCT_REQUIRE(plan && precon_out, "NULL argument");
    osmom_precon(plan, precon_out, S(stream));
  });
}

cbct_status cbct_osmom_step(cbct_plan* plan, int32_t s, cbct_dtype b_dtype, const void* b_s, float* z, float* xold,
                            const float* precon, float* r_work, float step, float mom, int32_t nonneg,
                            double* norm2_out, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_osmom_step");
    CBCT_REQUIRE(plan && s >= 0 && s < plan->n_subsets, "subset index out of range (one subset per step)");
    require_dtype(b_dtype);
    CBCT_REQUIRE(b_s && z && xold && precon && r_work, "NULL array");
    osmom_step(plan, s, b_dtype, b_s, z, xold, precon, r_work, step, mom, nonneg, norm2_out, S(stream));
  });
}

cbct_status cbct_osmom_update(float* z, float* xold, const float* precon, const float* g, size_t n, float step,
                              float mom, int32_t nonneg, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(z && xold && precon && g, "NULL array");
    osmom_update_launch(z, xold, precon, g, n, step, mom, nonneg, S(stream));
  });
}

cbct_status cbct_reduce_f64(int32_t kind, const float* a, const float* b, size_t n, double* out_dev, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(kind >= 0 && kind <= 2, "kind must be 0, 1 or 2");
    CBCT_REQUIRE(a && out_dev && (kind != 0 || b), "NULL array");
    // The partial sums take a buffer from the device's stream-ordered pool on
    // the caller's stream and give it back in stream order: calls on
    // different streams or threads never share it, and nothing outlives the call.
    double* partials = nullptr;
    CBCT_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&partials), sizeof(double) * 148 * 4, S(stream)));
    try {
      reduce_launch(kind, a, b, n, partials, 148 * 4, out_dev, S(stream));
    } catch (...) {
      cudaFreeAsync(partials, S(stream));
      throw;
    }
    CBCT_CUDA(cudaFreeAsync(partials, S(stream)));
  });
}

cbct_status cbct_reduce_f64_noalloc(int32_t kind, const float* a, const float* b, size_t n, double* out_dev,
                                    void* stream) {
  return guard([&] {
    CBCT_REQUIRE(kind >= 0 && kind <= 2, "kind must be 0, 1 or 2");
    CBCT_REQUIRE(a && out_dev && (kind != 0 || b), "NULL array");
    reduce_noalloc_launch(kind, a, b, n, out_dev, S(stream));
  });
}

static cbct_solver_params solver_defaults(const cbct_solver_params* p) {
  cbct_solver_params d{};
  d.iterations = 10;
  d.beta = 1.f;
  d.gamma = 0.f;
  d.non_negativity = 0;
  d.use_graph = 0;
  d.storage = CBCT_F32;
  d.refine_every = 0;
  d.proj_storage = CBCT_F32;
  d.tv_weight = 0.f;
  d.tv_alpha = 0.f;
  d.tau = 1e-3f;
  d.reg_steps = 1;
  return p ? *p : d;
}

cbct_status cbct_osmom_solve(cbct_plan* plan, const void* b, const float* x0, float* z_out,
                             const cbct_solver_params* params, double* resid_norm2_out, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(plan && b && z_out, "NULL argument");
    const cbct_solver_params prm = solver_defaults(params);
    CBCT_REQUIRE(prm.iterations >= 0, "iterations must be >= 0");
    osmom_solve(plan, b, x0, z_out, prm, resid_norm2_out, S(stream));
    check_on_return(plan, S(stream));
  });
}

cbct_status cbct_ossart_solve(cbct_plan* plan, const float* b, const float* x0, float* x_out,
                              const cbct_solver_params* params, double* cost_out, void* stream) {
  return guard([&] {
    if (plan) require_one_bin(plan, "cbct_ossart_solve");
    CBCT_REQUIRE(plan && b && x_out, "NULL argument");
    const cbct_solver_params prm = solver_defaults(params);
    CBCT_REQUIRE(prm.iterations >= 0, "iterations must be >= 0");
    if (prm.proj_storage != CBCT_F32) throw Error(CBCT_ERR_UNSUPPORTED, "OS-SART takes float projections");
    if (prm.tv_weight > 0.f) throw Error(CBCT_ERR_UNSUPPORTED, "OS-SART has no regulariser (osSARTSolver.h)");
    ossart_solve(plan, b, x0, x_out, prm, cost_out, S(stream));
    check_on_return(plan, S(stream));
  });
}

cbct_status cbct_tv_step(float* x, float* P, const float* s, const float* D, int32_t nx, int32_t ny, int32_t nz,
                         float scale, float tau, float tau_lambda, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(x && P && s && D, "NULL array");
    CBCT_REQUIRE(nx > 0 && ny > 0 && nz > 0, "image size must be positive");
    tv_primal_launch(x, P, nx, ny, nz, scale, S(stream));
    tv_update_launch(P, x, s, D, nx, ny, nz, 1.f, tau, tau_lambda, S(stream));
  });
}

cbct_status cbct_host_forward(cbct_plan* plan, int32_t s_first, int32_t n_batches, const float* vol_host,
                              float* proj_host, const int32_t* view_index, int32_t offset_sqrt, void* stream) {
  return guard([&] {
    host_forward(plan, s_first, n_batches, vol_host, proj_host, view_index, offset_sqrt, S(stream));
  });
}

cbct_status cbct_host_backproject(cbct_plan* plan, int32_t s_first, int32_t n_batches, const float* proj_host,
                                  float* vol_host, const int32_t* view_index, int32_t fbp, const float* filter,
                                  uint32_t fdk_flags, int32_t offset_sqrt, float scale, int32_t accumulate,
                                  void* stream) {
  return guard([&] {
    host_backproject(plan, s_first, n_batches, proj_host, vol_host, view_index, fbp, filter, fdk_flags, offset_sqrt,
                     scale, accumulate, S(stream));
  });
}

cbct_status cbct_batch_osmom(const cbct_batch_item* items, int32_t n, int32_t n_streams, void* stream) {
  return guard([&] { batch_osmom(items, n, n_streams, S(stream)); });
}

cbct_status cbct_batch_osmom_fused(const cbct_batch_item* items, int32_t n, void* stream) {
  return guard([&] { batch_osmom_fused(items, n, S(stream)); });
}

cbct_status cbct_phantom_voxelize(const cbct_geometry* g, const float* ell, int32_t n, int32_t ss, float* vol,
                                  void* stream) {
  return guard([&] {
    validate_geometry(g);
    CBCT_REQUIRE(ell && vol && n >= 0 && ss >= 1, "bad arguments");
    phantom_voxelize_launch(make_grid(*g), ell, n, ss, vol, S(stream));
  });
}

cbct_status cbct_phantom_project(cbct_plan* plan, int32_t s, const float* ell, int32_t n, float* proj, void* stream) {
  return guard([&] {
    const int i = subset_index(plan, s);
    CBCT_REQUIRE(ell && proj && n >= 0, "bad arguments");
    phantom_project_launch(plan, i, ell, n, proj, S(stream));
  });
}

cbct_status cbct_convert(const float* src, void* dst, size_t n, cbct_dtype dt, void* stream) {
  return guard([&] {
    CBCT_REQUIRE(src && dst, "NULL array");
    convert_launch(src, dst, n, dt, S(stream));
  });
}

}  // extern "C"
