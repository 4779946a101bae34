// cbct_internal.h -- shared declarations of the B200 cone-beam library.
#pragma once

#include <cuda_runtime.h>
#include <cudaTypedefs.h>
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <functional>
#include <new>
#include <stdexcept>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cbct.h"

namespace cbct {

// ---------------------------------------------------------------- errors
// Internal code throws cbct::Error; the C ABI (abi.cu) converts it into a
// status code and a thread-local message.  Nothing throws across the ABI.
struct Error : std::runtime_error {
  cbct_status status;
  Error(cbct_status s, const std::string& m) : std::runtime_error(m), status(s) {}
};

#define CBCT_CUDA(call)                                                                 \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess)                                                              \
      throw ::cbct::Error(e_ == cudaErrorMemoryAllocation ? CBCT_ERR_OUT_OF_MEMORY      \
                                                          : CBCT_ERR_CUDA,              \
                          std::string(#call) + ": " + cudaGetErrorString(e_));          \
  } while (0)

#define CBCT_REQUIRE(cond, msg)                                                         \
  do {                                                                                  \
    if (!(cond)) throw ::cbct::Error(CBCT_ERR_INVALID_ARGUMENT, msg);                   \
  } while (0)

// Thread-local message of the calling thread's last failed entry point (abi.cu).
std::string& last_error_slot();

// Runs f and converts what it throws into a status and the thread's message.
// Every C entry point is one guard call; nothing throws across the ABI.
template <class F>
cbct_status guard(F&& f) {
  try {
    f();
    last_error_slot().clear();
    return CBCT_OK;
  } catch (const Error& e) {
    last_error_slot() = e.what();
    return e.status;
  } catch (const std::bad_alloc&) {
    last_error_slot() = "host allocation failed";
    return CBCT_ERR_OUT_OF_MEMORY;
  } catch (const std::exception& e) {
    last_error_slot() = e.what();
    return CBCT_ERR_INTERNAL;
  } catch (...) {
    last_error_slot() = "unknown error";
    return CBCT_ERR_INTERNAL;
  }
}

// Host threads used for plan set-up loops.
inline int host_threads() {
  const unsigned hc = std::thread::hardware_concurrency();
  return (int)std::min(32u, std::max(1u, hc));
}

// Runs f(begin, end, thread_index) over [0, n) split into contiguous chunks on
// host_threads() threads (the calling thread takes the first chunk).
template <class F>
void parallel_for(int n, F&& f) {
  const int T = std::max(1, std::min(host_threads(), n));
  std::vector<std::thread> th;
  const int chunk = (n + T - 1) / T;
  for (int t = 1; t < T; ++t) {
    const int lo = t * chunk, hi = std::min(n, lo + chunk);
    if (lo < hi) th.emplace_back([&f, lo, hi, t] { f(lo, hi, t); });
  }
  f(0, std::min(n, chunk), 0);
  for (auto& x : th) x.join();
}

// Bytes per element of a storage type.
inline size_t dtype_size(cbct_dtype dt) { return dt == CBCT_F32 ? 4 : 2; }

inline void check_launch(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    throw Error(CBCT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// ---------------------------------------------------------------- geometry
// Per-view constants, computed in FP64 on the host and stored as float.
// A ray of detector pixel (u,v) runs from S to E(u,v) = S + D0 + u*Eu + v*Ev
// (conebeam_projection.cu:441-473 with the detector point expanded linearly
// in u and v).  Back-projection uses the inverse rotation of :975-984.
struct ViewParams {
  float cs, sn;          // cos(theta), sin(theta)
  float Sx, Sy;          // source position (S_z = 0)
  float D0x, D0y, D0z;   // direction E(0,0) - S
  float Eux, Euy;        // dE/du (in plane)
  float Evz;             // dE/dv (along z)
  float ox, oy;          // detector offsets, mm
  int dom;               // dominant in-plane axis of the view's rays: 0 = x, 1 = y
  int dsgn;              // sign of the ray direction along that axis (+1/-1)
  float pad0, pad1;
};
static_assert(sizeof(ViewParams) == 64, "ViewParams is 64 bytes");

// Kernel-side constants of the volume grid and detector.
struct GridConst {
  int nx, ny, nz;
  int W, H;
  int N;                  // samples per ray
  float hx, hy, hz;       // half volume size, mm
  float kx, ky, kz;       // voxels per mm: texel = world*k + b
  float bx, by, bz;       // n/2 - 0.5
  float vx, vy, vz;       // voxel size, mm
  float SAD, SDD;
  float fov_u, fov_v;
  float ku, kv;           // pixels per mm on the detector
  float bu, bv;           // W/2 - 0.5, H/2 - 0.5
  float invN;
  unsigned wait_limit;    // polls of a kernel's bounded wait for its next TMA stage
};

// Default poll limit of the bounded mbarrier waits (CBCT_OPT_WAIT_LIMIT).  A
// CTA whose wait gives up still drains the loads it has in flight with this
// default limit before it exits, so a shortened limit never leaves a copy
// writing into shared memory after its CTA is gone.
constexpr uint32_t kWaitLimit = 1u << 22;

// Box of the TMA slab forward projector, in the view's frame (e, d, z):
// e = in-plane cross axis (memory x), d = slab axis (memory y), z.
struct SlabBox {
  int bx, by, bz;         // TMA box (elements) in memory order x, y, z
  int valid;
};

// Forward projector tiling (compile-time): CTA = TU x TV rays of one view,
// slabs of TS voxels along the view's dominant in-plane axis, NSTAGE-deep
// TMA pipeline.  The box holds TS+1 rows of the slab axis padded to kBoxY so
// that neighbouring rows and planes fall in different shared-memory banks.
constexpr int kTU = 16;
constexpr int kTV = 16;
constexpr int kTS = 8;
constexpr int kBoxY = 10;
#ifndef CBCT_NSTAGE
#define CBCT_NSTAGE 2
#endif
constexpr int kNStage = CBCT_NSTAGE;
constexpr int kSlabBase = -1;      // slab m covers texel rows [kSlabBase + m*kTS, +kTS)
constexpr int kMaxSlabs = 260;
constexpr int kSmemBudget = 200 * 1024;
// Box widths (memory x) the slab kernel is compiled for; each is 8 mod 16.
constexpr int kBoxWidths[] = {40, 56, 72, 104, 136};
// Fan forward projector: kFU detector columns (one per warp) x kFV rows per
// CTA; the column's samples are interpolated in e and d kFKC at a time.
constexpr int kFU = 8;
constexpr int kFV = 32;
constexpr int kFKC = 16;
constexpr int kFanWidths[] = {24, 40, 56, 72};
// Row-pair forward projector: kPU detector columns x kPV rows per CTA, each
// thread marching two vertically adjacent rays of one column.
#ifndef CBCT_PAIR_ROWS
#define CBCT_PAIR_ROWS 16
#endif
#ifndef CBCT_PAIR_COLS
#define CBCT_PAIR_COLS 16
#endif
constexpr int kPU = CBCT_PAIR_COLS;
constexpr int kPV = CBCT_PAIR_ROWS;
constexpr int kPairThreads = kPU * kPV / 2;
// Row-quad forward projector: kQU columns x kQV rows per CTA, four adjacent
// rows of a column per thread.
#ifndef CBCT_QUAD_ROWS
#define CBCT_QUAD_ROWS 32
#endif
constexpr int kQU = 16;
constexpr int kQV = CBCT_QUAD_ROWS;
constexpr int kQuadThreads = kQU * kQV / 4;

// Forward-projector blocks per view: the largest of the slab, pair, quad and fan
// tilings (one FP64 partial sum per block).
inline size_t forward_tiles(int W, int H) {
  const size_t slab = (size_t)((W + kTU - 1) / kTU) * ((H + kTV - 1) / kTV);
  const size_t pair = (size_t)((W + kPU - 1) / kPU) * ((H + kPV - 1) / kPV);
  const size_t quad = (size_t)((W + kQU - 1) / kQU) * ((H + kQV - 1) / kQV);
  const size_t fan = (size_t)((W + kFU - 1) / kFU) * ((H + kFV - 1) / kFV);
  return std::max(std::max(slab, pair), std::max(quad, fan));
}


}  // namespace cbct

// ---------------------------------------------------------------- the plan
struct cbct_plan {
  cbct_geometry g{};
  cbct::GridConst gc{};
  int n_views = 0, n_subsets = 0;
  std::vector<int> first, count, offcorr;
  std::vector<float> angles, offsets;
  std::vector<cbct::ViewParams> hviews;
  cbct::ViewParams* d_views = nullptr;
  int device = 0;
  int max_subset = 0;

  // forward variant: 0 = gather (global loads), 1 = TMA slab, 2 = TMA fan, 3 = TMA row pairs,
  // 4 = TMA row quads
  int fwd_variant = 0;
  int fwd_pref = 0;         // CBCT_OPT_FORWARD_KERNEL: 0 automatic, 1 slab, 2 gather, 3 fan, 4 pair, 5 quad
  cbct::SlabBox pair{};     // row-pair kernel box for fp32 storage
  cbct::SlabBox pair16{};   // row-pair kernel box for 16-bit storage
  cbct::SlabBox quad{};     // row-quad kernel box for fp32 storage
  cbct::SlabBox quad16{};   // row-quad kernel box for 16-bit storage
  cbct::SlabBox fan{};      // fan kernel box for fp32 storage
  cbct::SlabBox fan16{};    // fan kernel box for 16-bit storage
  int fan_lz = 0;           // line length (planes) of the fan kernel, odd
  cbct::SlabBox slab{};     // box in the view frame for fp32 storage (x starts aligned to 4)
  cbct::SlabBox slab16{};   // box for 16-bit storage (x starts aligned to 8)
  size_t slab_smem = 0;     // dynamic shared memory of the fp32 slab kernel (bytes)
  std::vector<int> subset_has_xdom;  // per subset (and all-views entry): any x-dominant view
  void* d_volT = nullptr;   // x/y-transposed volume for x-dominant views (fp32 capacity)
  int bp_variant = 0;       // 0 = global loads, 1 = TMA-staged detector boxes
  int bp_pref = 0;          // 0: TMA-staged where it fits, 1: global loads (autotuner)
  cbct::SlabBox bp_box{};   // detector box (bx = u width, by = v rows)
  int bp_max_views = 0;     // views per launch the TMA back-projector holds

  // scratch owned by the plan (allocated at creation or first use, reused)
  float* d_proj_scratch = nullptr;  // weighted copies of projections (mult_MH with offset weight)
  size_t proj_scratch_elems = 0;
  double* d_partials = nullptr;     // per-block FP64 partial sums
  size_t n_partials = 0;
  int* d_flags = nullptr;           // [0] device range-check violations, [1] wait timeouts
  void* fdk_state = nullptr;        // FDK tables (weights.cu)
  float* d_fdk_work = nullptr;      // filtered projections for cbct_fdk
  size_t fdk_work_elems = 0;
  void* graph_cache = nullptr;      // captured solver graph (solver.cu)
  float* d_stream_buf[2] = {nullptr, nullptr};  // batch buffers of the host-array operators
  size_t stream_buf_elems = 0;
  float* d_stream_vol = nullptr;    // bin volume of the host-array operators

  // solver workspace (allocated on first solve, reused)
  float* ws = nullptr;
  size_t ws_elems = 0;

  // Identity for caches that outlive one call: serial is unique per plan in
  // the process; generation grows with every change of the plan's state
  // (options, mask, bins, weights, autotuning: every graph_cache_free).
  uint64_t serial = 0, generation = 0;

  int debug_checks = 0;
  int force_gather = 0;
  int status_check = 1;     // CBCT_OPT_STATUS_CHECK: solve/FDK entry points read the flag words on return
  const unsigned char* d_mask = nullptr;  // voxel mask applied after back-projection (caller-owned)
  const float* d_pweights = nullptr;      // projection weights, all views in subset order (caller-owned)

  // Bins (CBCT_binning): with n_bins > 1 every view belongs to one bin and
  // images hold n_bins volumes.  Subset s splits into the runs of its views
  // that share a bin ("segments"); they are kept as further view ranges after
  // index n_subsets of first/count/offcorr: range indices seg_begin[s] ..
  // seg_end[s]-1, bin seg_bin[k] (-1 for the subsets and the all-views entry).
  int n_bins = 1;
  std::vector<int> seg_begin, seg_end, seg_bin;

  // Device memory source.  Plans of the serving loop draw every buffer from
  // its stream-ordered pool on `pool_stream` (cudaMallocFromPoolAsync /
  // cudaFreeAsync), so that concurrent requests never meet the implicit
  // device synchronisation of cudaMalloc/cudaFree; such a plan is used on
  // `pool_stream` only.  Other plans use cudaMalloc.
  cudaMemPool_t pool = nullptr;
  cudaStream_t pool_stream = nullptr;
  std::vector<std::pair<void*, size_t>> allocs;  // live plan-owned buffers
  size_t dev_bytes = 0, dev_bytes_peak = 0;
};

namespace cbct {

PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder();

// Plan-owned device memory (abi.cu): cudaMalloc, or the serving pool in
// stream order (see cbct_plan::pool).  plan_upload copies host data that may
// be released as soon as the call returns.
void* plan_alloc(cbct_plan* p, size_t bytes);
void plan_dealloc(cbct_plan* p, void* ptr);
void plan_upload(cbct_plan* p, void* dst, const void* src, size_t bytes);
void plan_memset(cbct_plan* p, void* dst, int value, size_t bytes);
template <class T>
T* plan_alloc_n(cbct_plan* p, size_t n) {
  return static_cast<T*>(plan_alloc(p, n * sizeof(T)));
}

// Raises a kernel's dynamic shared-memory limit to `bytes` once per kernel
// and device (no-op when already high enough, so it is safe to call before
// launches that may be captured).
void ensure_smem_attr(const void* func, size_t bytes);

// forward.cu
void forward_prepare(cbct_plan* p);
// b: measured projections of storage type b_dtype (residual mode).
void forward_launch_ex(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out, const void* b,
                       const float* pw, float scale, int mode, int apply_offset, int accumulate,
                       double* norm2_out, cudaStream_t st, cbct_dtype b_dtype = CBCT_F32);
void forward_launch(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out,
                    const float* b, float scale, int mode, int apply_offset, int accumulate,
                    double* norm2_out, cudaStream_t st);
void forward_choose_variant(cbct_plan* p);
// backproject.cu
void backproject_choose_variant(cbct_plan* p);
void backproject_prepare(cbct_plan* p);
void backproject_launch(cbct_plan* p, int s, const float* proj, float* vol, int fdk_weight,
                        int accumulate, float out_scale, cudaStream_t st);
// weights.cu
void offset_weight_launch(cbct_plan* p, int s, const float* in, float* out, int variant,
                          cudaStream_t st);
// in: projections of storage type in_dtype; out: float (may alias in when float).
void fdk_filter_launch(cbct_plan* p, int s, const void* in, float* out, const float* filter,
                       uint32_t flags, cudaStream_t st, cbct_dtype in_dtype = CBCT_F32);
// Builds the FDK tables for `filter` now (they are otherwise made on first use).
void fdk_prepare(cbct_plan* p, const float* filter);
// solver.cu
void reduce_launch(int kind, const float* a, const float* b, size_t n, double* partials,
                   size_t n_partials, double* out, cudaStream_t st);
void finalize_partials(const double* partials, int n, double* out, cudaStream_t st);
void reduce_noalloc_launch(int kind, const float* a, const float* b, size_t n, double* out, cudaStream_t st);
void osmom_update_launch(float* z, float* xold, const float* precon, const float* g, size_t n,
                         float step, float mom, int nonneg, cudaStream_t st);

// host_stream.cu: host-array operators over the plan's subsets [s0, s0 + ns)
void host_forward(cbct_plan* p, int s0, int ns, const float* vol_host, float* proj_host, const int* view_index,
                  int offset_sqrt, cudaStream_t caller);
void host_backproject(cbct_plan* p, int s0, int ns, const float* proj_host, float* vol_host, const int* view_index,
                      int fbp, const float* filter, uint32_t fdk_flags, int offset_sqrt, float scale, int accumulate,
                      cudaStream_t caller);

// tv.cu: primal and fused dual + data-resolvent steps of the TV regulariser
void tv_primal_launch(const float* x, float* P, int nx, int ny, int nz, float scale, cudaStream_t st);
void tv_update_launch(const float* P, float* x, const float* s, const float* D, int nx, int ny, int nz, float w,
                      float tau, float tau_lambda, cudaStream_t st);

// autotune.cu: times the plan's projector variants on its largest subset and
// keeps the fastest; times[5] = forward slab, fan, gather, back-projection
// TMA, global (ms per launch, -1 where unavailable)
void plan_autotune(cbct_plan* p, float* times, cudaStream_t st);
void graph_cache_free(cbct_plan* p);

// microbench.cu: interpolations per second of the projectors' inner operation
// from shared memory (kind 3 = trilinear, 2 = bilinear)
double microbench_interp(int kind, int groups, int reps, cudaStream_t st);

// mask.cu
void spacecarver_launch(cbct_plan* p, int s, const float* proj, float limit, unsigned char* mask, int combine,
                        cudaStream_t st);
void apply_mask_launch(float* vol, const unsigned char* mask, size_t n, cudaStream_t st);
void mul_launch(float* out, const float* in, const float* w, size_t n, cudaStream_t st);

// plans and set-up rules (abi.cu)
void validate_geometry(const cbct_geometry* g);
// Reads the plan's device flag words after the work enqueued on `st` (a
// stream synchronisation), clears them, and throws CBCT_ERR_TIMEOUT (an
// expired bounded wait) or CBCT_ERR_DEVICE_CHECK (a range-check violation or
// a footprint that did not fit its box) when any is set.
void plan_check_flags(cbct_plan* p, cudaStream_t st);
// True while `st` is being captured into a CUDA graph.
bool stream_capturing(cudaStream_t st);
// forward_buffers = false leaves out the forward projector's transposed-volume
// buffer (plans that only back-project; their forward calls take the gather path).
cbct_plan* plan_create(const cbct_geometry* g, const float* angles, const float* offsets, int n_views,
                       const int* subset_sizes, int n_subsets, const int* offcorr, cudaMemPool_t pool,
                       cudaStream_t pool_stream, bool forward_buffers);
void plan_free(cbct_plan* p);
bool short_scan_rule(const cbct_geometry& g, const float* angles, int n);
bool offset_override_rule(const cbct_geometry& g, const float* offsets, int n);
// solver.cu
void osmom_solve(cbct_plan* p, const void* b, const float* x0, float* z, const cbct_solver_params& prm,
                 double* resid, cudaStream_t st);
void fdk_run(cbct_plan* p, const void* proj, float* vol, const float* filter, uint32_t flags, float* work,
             cudaStream_t st, cbct_dtype proj_dtype);
void osmom_precon(cbct_plan* p, float* D, cudaStream_t st);
void osmom_step(cbct_plan* p, int s, cbct_dtype bt, const void* b, float* z, float* xold, const float* D, float* r,
                float step, float mom, int nonneg, double* norm2, cudaStream_t st);

// ---------------------------------------------------------- work-list launches
// The fused batch solver (multi.cu) runs every step of many scans as one
// launch per kernel kind whose CTAs work through a list of (scan, tile)
// items.  A schedule is built on the host first: launch records go into
// `host` (128-byte aligned, as the tensor maps inside them need), and `ops`
// holds the work in order, each op issuing its launches on the stream it is
// given and finding its records at `dev` + offset.  The records are then
// uploaded once and the ops captured into one CUDA graph.  Every work-list
// launch has its own item counter after the records; the first op zeroes them.
struct WorkArena {
  std::vector<unsigned char> host;
  unsigned char* dev = nullptr;
  int n_counters = 0;
  std::vector<std::function<void(cudaStream_t)>> ops;
  size_t add(const void* rec, size_t bytes) {
    const size_t off = (host.size() + 127) & ~size_t(127);
    host.resize(off + bytes);
    std::memcpy(host.data() + off, rec, bytes);
    return off;
  }
  size_t counters_offset() const { return (host.size() + 127) & ~size_t(127); }
  int* counter(int i) const { return reinterpret_cast<int*>(dev + counters_offset()) + i; }
  size_t bytes() const { return counters_offset() + sizeof(int) * (size_t)std::max(n_counters, 1); }
};

// Resident CTAs per SM of `func` at `threads` x `smem`, times the SMs: the
// grid of a work-list launch (cached per kernel and size).
int resident_grid(const void* func, int threads, size_t smem);

// A scan whose own launch would fill the GPU for this many waves of resident
// CTAs keeps its one-scan launch in the fused schedule: its last partial wave
// is a small share of it, and the one-scan kernel reads its arguments from the
// constant bank instead of holding a work-list record's fields in registers
// (measured: the work-list kernels run 2-7 % slower per item; at 4 waves a
// partial last wave costs more, at 16 less).
#ifndef CBCT_MULTI_FILL_WAVES
#define CBCT_MULTI_FILL_WAVES 16
#endif
constexpr int kMultiFillWaves = CBCT_MULTI_FILL_WAVES;

// One scan's part of a work-list forward residual launch: r_s = w (A_s vol - b_s),
// the one-scan call forward_launch_ex(p, s, CBCT_F32, vol, out, b, NULL, 1, 1,
// apply_offset, 0, norm2_out, st, b_dtype).
struct MultiFwdJob {
  cbct_plan* p;
  int s;
  const float* vol;
  float* out;
  const void* b;
  cbct_dtype b_dtype;
  int apply_offset;
  double* norm2_out;
};
// Adds the launches of `jobs` to the schedule: the scans whose plans use the
// TMA slab, row-pair or row-quad kernel are grouped by kernel and box width,
// one work-list launch per group; the others get their one-scan launch.
void forward_multi(WorkArena& A, const std::vector<MultiFwdJob>& jobs);

// One scan's part of a work-list back-projection over subset s of p:
// kind 0 = preconditioner (vol = 1/max(A^T proj, 1e-6)), kind 1 = OS-MOM
// update of (vol = z, xold) with precon aux, step, mom, nonneg.
struct MultiBpJob {
  cbct_plan* p;
  int s;
  const float* proj;
  float* vol;
  float* xold;
  const float* aux;
  float step, mom;
  int nonneg;
};
void backproject_multi(WorkArena& A, int kind, const std::vector<MultiBpJob>& jobs);

// multi.cu: the fused batch solver (cbct_batch_osmom_fused)
void batch_osmom_fused(const cbct_batch_item* items, int n, cudaStream_t st);
// solver.cu: the plan's solver workspace of at least `elems` floats (grown on
// demand, kept), and a fill of n floats with v.
float* solver_workspace(cbct_plan* p, size_t elems);
void fill_launch(float* x, size_t n, float v, cudaStream_t st);

// host helpers (abi.cu)
void default_filter(int W, float* out);
void subset_partition(int n_views, const int* view_bin, int n_subsets, int* order,
                      int* sizes, int* n_out);

}  // namespace cbct
