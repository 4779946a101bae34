/* cbct.h -- C ABI of the B200 cone-beam projector and ordered-subset core.
 *
 * This is the drop-in boundary for gt-tomography's circular-orbit cone-beam
 * hot path.  Every entry point replaces one reference function or operator
 * method (cited below by file:line within the gt-tomography project).  No C++
 * types or exceptions cross this boundary: arguments are plain pointers and
 * sizes, results are cbct_status codes.
 *
 * Layouts (identical to the reference's cuNDArray<float> arrays):
 *   volume       (nx, ny, nz)   x fastest:  index = (k*ny + j)*nx + i
 *   projections  (W, H, P)      u fastest:  index = (p*H + v)*W + u
 *   offsets      (P, 2)         per view (offset_x, offset_y) in mm
 * Views are held in subset-contiguous order: subset s owns views
 * [first_s, first_s + size_s) where first_s is the sum of the sizes before it
 * (the order CBSubsetOperator::setup leaves behind, CBSubsetOperator.cpp:100-115).
 *
 * Device pointers are CUDA global-memory pointers of the current device.
 * All device work is enqueued on the caller's stream (0 = legacy default
 * stream); no entry point synchronises the device unless documented.
 */
#ifndef CBCT_H_
#define CBCT_H_

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CBCT_API __attribute__((visibility("default")))
#else
#define CBCT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
  CBCT_OK = 0,
  CBCT_ERR_INVALID_ARGUMENT = 1, /* bad pointer, rank or size (conebeam_projection.cu:547-561) */
  CBCT_ERR_CUDA = 2,             /* a CUDA runtime call failed (CHECK_FOR_CUDA_ERROR in the reference) */
  CBCT_ERR_OUT_OF_MEMORY = 3,
  CBCT_ERR_UNSUPPORTED = 4,      /* geometry or dtype outside what this build implements */
  CBCT_ERR_DEVICE_CHECK = 5,     /* a kernel's own range check recorded a violation */
  CBCT_ERR_TIMEOUT = 6,          /* a bounded device-side wait expired */
  CBCT_ERR_BUDGET = 7,           /* request exceeds the memory budget (serving loop) */
  CBCT_ERR_CANCELLED = 8,
  CBCT_ERR_INTERNAL = 9
} cbct_status;

typedef enum { CBCT_F32 = 0, CBCT_F16 = 1, CBCT_BF16 = 2 } cbct_dtype;

/* Geometry in the units of CBCT_geometry (xray/CBCT_acquisition.h:24-120)
 * plus the image grid of the operator setup (is_dims_in_mm). */
typedef struct {
  float SAD;               /* source-to-axis distance, mm */
  float SDD;               /* source-to-detector distance, mm */
  float fov_u, fov_v;      /* detector size in mm (CBCT_geometry::get_FOV) */
  int32_t width, height;   /* detector pixels W, H */
  int32_t nx, ny, nz;      /* volume voxels */
  float lx, ly, lz;        /* volume size in mm (is_dims_in_mm) */
  float samples_per_pixel; /* rays take (int)(spp*nx) samples; reference default 1.5
                              (cuConebeamProjectionOperator.cpp:18) */
} cbct_geometry;

typedef struct cbct_plan cbct_plan;

/* Flags of cbct_backproject. */
#define CBCT_BP_OFFSET_WEIGHT 0x1u /* multiply the input by the sin^2 Wang weight first
                                      (offset_correct_kernel, conebeam_projection.cu:233-262) */
#define CBCT_BP_FDK_WEIGHT 0x2u    /* FDK 1/U^2 distance weight (conebeam_projection.cu:1009-1024) */

/* Flags of cbct_fdk_filter / cbct_fdk. */
#define CBCT_FDK_COSINE 0x1u   /* cosine pre-weight (hoCuConebeamProjectionOperator.cpp:64-102) */
#define CBCT_FDK_PARKER 0x2u   /* Parker short-scan weight (conebeam_projection.cu:151-194) */
#define CBCT_FDK_OFFSET 0x4u   /* sin^2 offset weight after filtering (conebeam_projection.cu:1516-1517) */
#define CBCT_FDK_RAMP 0x8u     /* the row filter itself (conebeam_projection.cu:1504-1511) */

/* ----------------------------------------------------------------------------
 * Status and diagnostics
 * ------------------------------------------------------------------------- */
CBCT_API const char* cbct_status_string(cbct_status s);
/* Message of the last failing call on this host thread ("" if none). */
CBCT_API const char* cbct_last_error(void);
/* Library version string. */
CBCT_API const char* cbct_version(void);

/* ----------------------------------------------------------------------------
 * Host-side setup helpers (pure host code; no device work)
 * ------------------------------------------------------------------------- */

/* Subset assignment of CBSubsetOperator<ARRAY>::setup (CBSubsetOperator.cpp:52-115):
 * views with view_bin[i] >= 0 are dealt round-robin to n_subsets subsets in index
 * order, each subset is sorted by bin, and order_out receives the concatenation.
 * view_bin may be NULL (one bin holding every view).  *n_out = views placed. */
CBCT_API cbct_status cbct_subset_partition(int32_t n_views, const int32_t* view_bin, int32_t n_subsets,
                                  int32_t* order_out, int32_t* subset_sizes_out, int32_t* n_out);

/* Default FDK frequency filter, length W+1, normalised to sum W+1
 * (hoCuConebeamProjectionOperator::compute_default_frequency_filter, .cpp:26-62). */
CBCT_API cbct_status cbct_default_frequency_filter(int32_t W, float* out);

/* Cosine weights (W x H) of hoCuConebeamProjectionOperator::compute_cosine_weights (.cpp:64-102). */
CBCT_API cbct_status cbct_cosine_weights(const cbct_geometry* g, float* out);

/* Short-scan test (span <= pi + 3*delta) of hoCuConebeamProjectionOperator.h:57-65
 * and cuConebeamProjectionOperator.cpp:166-174.  Angles must already start at 0. */
CBCT_API cbct_status cbct_is_short_scan(const cbct_geometry* g, const float* angles_deg, int32_t n,
                               int32_t* short_scan_out);

/* Offset-correction override rule (|mean offset_x| > 0.1*fov_u) of
 * cuConebeamProjectionOperator.cpp:176-181 / hoCuConebeamProjectionOperator.h:72-76. */
CBCT_API cbct_status cbct_offset_override(const cbct_geometry* g, const float* offsets_xy, int32_t n,
                                 int32_t* use_offset_correction_out);

/* ----------------------------------------------------------------------------
 * Plans: geometry resident on the device
 * ------------------------------------------------------------------------- */

/* Creates a plan for n_views views held in subset-contiguous order.
 * angles_deg / offsets_xy are host arrays (n_views and 2*n_views floats).
 * subset_sizes (n_subsets ints, summing to n_views) may be NULL for one subset.
 * offset_correction (n_subsets ints, 0/1) selects the sin^2 input weight of
 * cbct_backproject per subset (use_offset_correction_ of each
 * cuConebeamProjectionOperator); NULL = all off.
 * Replaces cuConebeamProjectionOperator::setup (.cpp:148-206) and the per-call
 * thrust uploads of conebeam_projection.cu:600-601,1225-1226.  Allocates device
 * memory; must not be called during stream capture. */
CBCT_API cbct_status cbct_plan_create(const cbct_geometry* g, const float* angles_deg,
                             const float* offsets_xy, int32_t n_views,
                             const int32_t* subset_sizes, int32_t n_subsets,
                             const int32_t* offset_correction, cbct_plan** plan_out);
CBCT_API cbct_status cbct_plan_destroy(cbct_plan* plan);

/* Number of views in subset s (s = -1: all views) and index of its first view. */
CBCT_API cbct_status cbct_plan_subset(const cbct_plan* plan, int32_t s, int32_t* first_out,
                             int32_t* count_out);

/* Name of the forward-projector variant the plan selected ("tma-quad", "tma-pair", "tma-slab",
 * "tma-fan" or "gather"). */
CBCT_API const char* cbct_plan_forward_variant(const cbct_plan* plan);

/* Autotuner (no reference counterpart): runs every forward projector (slab,
 * column-fan, gather, row-pair, row-quad) and back-projector (TMA-staged,
 * global loads) the plan can use on its largest subset, keeps the fastest of
 * each for the plan, and writes the timings (ms per launch; -1 where a variant
 * is unavailable) to times_ms_out[7] = {fwd slab, fwd fan, fwd gather, bp TMA,
 * bp global, fwd row-pair, fwd row-quad}.  Synchronises `stream`; allocates
 * and frees two scratch buffers. */
CBCT_API cbct_status cbct_plan_autotune(cbct_plan* plan, float* times_ms_out, void* stream);

/* Plan options (no reference counterpart; diagnostics of this library).
 * CBCT_OPT_DEBUG_CHECKS: kernels record index-range violations and unconsumed
 *   samples in the plan's flag word instead of only clamping.
 * CBCT_OPT_FORCE_GATHER: use the global-gather forward projector. */
#define CBCT_OPT_DEBUG_CHECKS 1
#define CBCT_OPT_FORCE_GATHER 2
/* CBCT_OPT_FORWARD_KERNEL: 0 = automatic (the row-quad kernel where adjacent
 * detector rows stay within 0.66 z texel of each other, else the row-pair
 * kernel where they stay within one texel, else the per-ray slab kernel, each
 * where its boxes fit, else gather), 1 = slab, 2 = gather, 3 = the column-fan
 * kernel (e/d interpolation shared by the rays of a detector column; slower on
 * B200 at the sizes measured so far), 4 = the row-pair kernel (one thread
 * marches two vertically adjacent rays of a column and shares their in-plane
 * interpolation), 5 = the row-quad kernel (four rows per thread).  Slab, fan,
 * row-pair and row-quad results are bitwise equal. */
#define CBCT_OPT_FORWARD_KERNEL 3
/* CBCT_OPT_WAIT_LIMIT: polls (>= 0) a TMA-staged projector kernel spends
 * waiting for its next shared-memory stage before it gives up (default
 * 4194304).  A CTA that gives up records the event in the plan's flag word,
 * waits with the default limit for the loads it still has in flight, leaves
 * its rays or voxels unfinished and exits; the calling entry point (or
 * cbct_plan_check) then reports CBCT_ERR_TIMEOUT.  0 makes every such wait
 * give up at once, which is how the failure path is tested. */
#define CBCT_OPT_WAIT_LIMIT 4
/* CBCT_OPT_STATUS_CHECK: 1 (default) = cbct_osmom_solve, cbct_ossart_solve,
 * cbct_fdk and cbct_fdk_ex synchronise their stream on return and report the
 * plan's flag words as a status (CBCT_ERR_TIMEOUT, CBCT_ERR_DEVICE_CHECK),
 * except while the stream is being captured into a CUDA graph; 0 = they stay
 * asynchronous and the caller checks with cbct_plan_check. */
#define CBCT_OPT_STATUS_CHECK 5
CBCT_API cbct_status cbct_plan_set_option(cbct_plan* plan, int32_t option, int32_t value);

/* On-chip ceiling of the projectors' inner operation (no reference
 * counterpart; a measurement of this library): FP32 software interpolation
 * from a shared-memory box at the projectors' access pattern and arithmetic,
 * with nothing else in the loop, over four waves of resident thread blocks.
 * kind 3 = trilinear (the forward projectors' ray sample), 2 = bilinear (the
 * back-projector's voxel-view update); groups = loop trips per thread (8
 * samples per trip for kind 3, 16 for kind 2).  rate_out = interpolations per
 * second (CUDA events, warm-up launch first).  Synchronises `stream`. */
CBCT_API cbct_status cbct_microbench_interp(int32_t kind, int32_t groups, double* rate_out, void* stream);

/* Reads (and optionally clears) the plan's device flag words:
 * flags_out[0] = range-check violations and footprints that did not fit their
 * shared-memory box, flags_out[1] = expired bounded waits.
 * Synchronises the device. */
CBCT_API cbct_status cbct_plan_read_flags(cbct_plan* plan, int32_t* flags_out, int32_t reset);

/* Device-side status of the plan's work (no reference counterpart: the
 * reference's kernels have no device-side failure path).  Synchronises
 * `stream`, reads and clears the plan's flag words and returns
 * CBCT_ERR_TIMEOUT when a kernel's bounded wait expired, CBCT_ERR_DEVICE_CHECK
 * when a kernel recorded a range violation or a footprint that did not fit its
 * box (results of the calls since the last check are then not to be trusted),
 * else CBCT_OK.  The asynchronous operators (cbct_forward, cbct_backproject,
 * cbct_forward_residual, cbct_fdk_filter ...) leave the check to the caller;
 * the host-array operators, the batch executor and the serving loop run it
 * themselves. */
CBCT_API cbct_status cbct_plan_check(cbct_plan* plan, void* stream);

/* ----------------------------------------------------------------------------
 * Operators
 * ------------------------------------------------------------------------- */

/* mult_M: forward projection of vol into the projections of subset s
 * (s = -1: every view).  proj points at the subset's first projection.
 * vol_dtype selects the volume storage type (CBCT_F32, CBCT_F16, CBCT_BF16);
 * interpolation and accumulation are FP32; proj is float.
 * Replaces conebeam_forwards_projection (conebeam_projection.cu:530-635) as
 * called by cuConebeamProjectionOperator::mult_M (.cpp:38-80). */
CBCT_API cbct_status cbct_forward(cbct_plan* plan, int32_t s, cbct_dtype vol_dtype, const void* vol,
                         float* proj, int32_t accumulate, void* stream);

/* mult_MH: back-projection of the subset's projections into vol.
 * flags: CBCT_BP_OFFSET_WEIGHT (weighted copy of the input, the input itself is
 * not modified), CBCT_BP_FDK_WEIGHT.
 * Replaces conebeam_backwards_projection (conebeam_projection.cu:1172-1299) as
 * called by cuConebeamProjectionOperator::mult_MH (.cpp:82-116).  With
 * use_plan_offset = 1 the plan's per-subset offset_correction flag is OR-ed in. */
CBCT_API cbct_status cbct_backproject(cbct_plan* plan, int32_t s, const float* proj, float* vol,
                             uint32_t flags, int32_t use_plan_offset, int32_t accumulate,
                             void* stream);

/* Wang offset weight in place on the subset's projections.
 * variant 0: sin^2 with zeroing (offset_correct_kernel, conebeam_projection.cu:233-262);
 * variant 1: sin (offset_correct_kernel_sqrt, :303-331; apply_offset_correct, :369-404). */
CBCT_API cbct_status cbct_offset_correct(cbct_plan* plan, int32_t s, float* proj, int32_t variant,
                                void* stream);

/* FDK pre-processing of the subset's projections, proj_in -> proj_out (may alias):
 * [cosine] -> [Parker] -> [ramp filter] -> [sin^2 offset], per the flags.
 * filter: host array of W+1 floats, or NULL for the default filter.
 * Replaces the per-batch FBP block of conebeam_projection.cu:1483-1521 (with
 * cb_fft/cb_ifft :87-139); the filter is a hand-written shared-memory FFT. */
CBCT_API cbct_status cbct_fdk_filter(cbct_plan* plan, int32_t s, const float* proj_in, float* proj_out,
                            const float* filter, uint32_t flags, void* stream);

/* Whole FDK of hoCuConebeamProjectionOperator::mult_MH with filtered
 * back-projection (hoCuConebeamProjectionOperator.cpp:235-254): every view of
 * the plan is one bin; FDK pre-processing as cbct_fdk_filter with
 * flags | CBCT_FDK_RAMP | CBCT_FDK_COSINE, 1/U^2-weighted back-projection,
 * then vol *= 2/P.  work: device scratch of at least W*H*P floats (the
 * filtered projections), or NULL to use a plan-owned buffer. */
CBCT_API cbct_status cbct_fdk(cbct_plan* plan, const float* proj, float* vol, const float* filter,
                     uint32_t flags, float* work, void* stream);

/* cbct_fdk_filter and cbct_fdk for projections stored as proj_dtype
 * (CBCT_F32, CBCT_F16 or CBCT_BF16); the filter computes in FP32 and writes
 * FP32.  cbct_fdk_ex with a 16-bit proj needs work (or the plan buffer); with
 * CBCT_F32 it behaves as cbct_fdk. */
CBCT_API cbct_status cbct_fdk_filter_ex(cbct_plan* plan, int32_t s, cbct_dtype proj_dtype, const void* proj_in,
                                        float* proj_out, const float* filter, uint32_t flags, void* stream);
CBCT_API cbct_status cbct_fdk_ex(cbct_plan* plan, cbct_dtype proj_dtype, const void* proj, float* vol,
                                 const float* filter, uint32_t flags, float* work, void* stream);

/* Bins (CBCT_binning, xray/CBCT_binning.h:18-172): view_bin gives the bin of
 * every plan view (n_views ints in [0, n_bins)); within each subset the views
 * of a bin must be contiguous, the order CBSubsetOperator::setup produces
 * (each subset sorted by bin, CBSubsetOperator.cpp:86-87).  Volumes then hold
 * n_bins images (bin-major, nx*ny*nz floats each): cbct_forward projects each
 * bin's views from that bin's image, cbct_backproject writes each bin's image
 * from its own views (a bin without views in the call is cleared unless
 * accumulating), as cuConebeamProjectionOperator does per bin (.cpp:49-116),
 * and cbct_osmom_solve reconstructs all bins (fp32, without a residual trace).
 * n_bins <= 1 or view_bin = NULL returns to one bin. */
CBCT_API cbct_status cbct_plan_set_bins(cbct_plan* plan, int32_t n_bins, const int32_t* view_bin);

/* ----------------------------------------------------------------------------
 * Voxel masks
 * Masks are uint8 arrays of nx*ny*nz voxels (1 = keep), the layout of the
 * reference's cuNDArray<bool>.
 * ------------------------------------------------------------------------- */

/* Space carver over the views of subset s (s = -1: all views):
 * conebeam_spacecarver (conebeam_projection.cu:1043-1167, kernel :822-921).
 * combine = 0 writes the mask; combine = 1 ANDs it into `mask`, as
 * CBSubsetOperator::calculate_mask combines its subsets (CBSubsetOperator.cpp:179-190). */
CBCT_API cbct_status cbct_spacecarver(cbct_plan* plan, int32_t s, const float* proj, float limit, uint8_t* mask,
                                      int32_t combine, void* stream);

/* vol *= mask (apply_mask, conebeam_projection.cu:1651-1657). */
CBCT_API cbct_status cbct_apply_mask(float* vol, const uint8_t* mask, size_t n, void* stream);

/* Sets (or clears, with NULL) the mask the plan's back-projections apply to
 * their output (cuConebeamProjectionOperator::set_mask and the apply_mask at
 * .cpp:113-114).  The caller keeps the mask alive while the plan uses it.
 * Applies to cbct_backproject without CBCT_BP_FDK_WEIGHT and to the solvers.
 * An accumulating back-projection is masked as a whole, the caller's earlier
 * contents included (vol = mask * (vol + A^T p)), as the reference's
 * apply_mask on the operator's output is. */
CBCT_API cbct_status cbct_plan_set_mask(cbct_plan* plan, const uint8_t* mask);

/* Projection weights of CBSubsetWeightOperator (xray/CBSubsetWeightOperator.h:11-63):
 * a device array of W*H*n_views floats in subset-contiguous order (NULL clears).
 * With weights set, cbct_forward returns w * (A x), cbct_backproject back-projects
 * w * input, and the fused residual and the solvers weight the same way.  The
 * caller keeps the array alive while the plan uses it. */
CBCT_API cbct_status cbct_plan_set_projection_weights(cbct_plan* plan, const float* weights);

/* ----------------------------------------------------------------------------
 * Solver building blocks
 * ------------------------------------------------------------------------- */

/* Fused residual forward projection used by the ordered-subset solvers:
 *   r = w_off(u) * (A_s vol - b_s) * scale          (weight when apply_offset)
 * and, when norm2_out is not NULL, norm2_out[0] = sum (A_s vol - b_s)^2 in FP64
 * (the VERBOSE residual norm of osMOMSolverD.h:147-149).
 * Replaces mult_M + "-= subsets[s]" + the offset-weighted copy inside mult_MH
 * (osMOMSolverD.h:144-145, cuConebeamProjectionOperator.cpp:101-102). */
CBCT_API cbct_status cbct_forward_residual(cbct_plan* plan, int32_t s, cbct_dtype vol_dtype,
                                  const void* vol, const float* b, float* r, float scale,
                                  int32_t apply_offset, double* norm2_out, void* stream);

/* The OS-MOM preconditioner (osMOMSolverD.h:115-120): precon_out =
 * 1 / max(A^T (W A 1), 1e-6) over every subset of the plan, W being each
 * subset's offset weight as its mult_MH applies it (the ones image is
 * projected and back-projected subset by subset, as the reference's
 * all-subset mult_M / mult_MH do).  Uses the plan's solver workspace
 * (allocated on first use, so the first call must not be captured). */
CBCT_API cbct_status cbct_osmom_precon(cbct_plan* plan, float* precon_out, void* stream);

/* One OS-MOM subset step (osMOMSolverD.h:142-175 without regularisers) as the
 * two kernels cbct_osmom_solve runs per subset:
 *   r = w_off (A_s z - b_s) into r_work (W*H*|s| floats), and
 *   norm2_out[0] = ||A_s z - b_s||^2 in FP64 when norm2_out is not NULL;
 *   then, fused into the back-projection of r:
 *   zt = z - step * precon * A_s^T r ; x = nonneg ? max(zt,0) : zt ;
 *   z = x (1+mom) - mom xold ; xold = x.
 * b_s: the subset's measured projections, of type b_dtype.  step is
 * beta / (1 + gamma i) * n_subsets and mom = (told - 1) / t, the solver's
 * values (:142, :155-157, :171-173).  A caller that keeps its own loop (the
 * reference driver's osMOMSolverD) gets the solver's arithmetic per step. */
CBCT_API cbct_status cbct_osmom_step(cbct_plan* plan, int32_t s, cbct_dtype b_dtype, const void* b_s, float* z,
                                     float* xold, const float* precon, float* r_work, float step, float mom,
                                     int32_t nonneg, double* norm2_out, void* stream);

/* One OS-MOM update (osMOMSolverD.h:155-175 without regularisers):
 *   zt = z - step * precon * g ; x = nonneg ? max(zt,0) : zt
 *   z  = x*(1+mom) - mom*xold ; xold = x                                  */
CBCT_API cbct_status cbct_osmom_update(float* z, float* xold, const float* precon, const float* g,
                              size_t n, float step, float mom, int32_t nonneg, void* stream);

/* One primal-dual step of the TV regulariser inside the OS-MOM denoise
 * (osMOMSolverD.h:214-224 with a cuTVPrimalDualOperator of weight 1 after the
 * solver's normalisation): P (3*nx*ny*nz floats) receives the periodic forward
 * differences of x times `scale` (= sigma / (1 + sigma alpha)), each gradient
 * vector projected onto the unit ball (cuTVPrimalDualOperator.cu:9-37); then
 * x = ((x - tau g) + tau_lambda (s / D)) / ((1 / D) tau_lambda + 1) with g the
 * negative divergence of P (:40-62) and tau_lambda = tau / lambda
 * (updateG, osMOMSolverD.h:233-247). */
CBCT_API cbct_status cbct_tv_step(float* x, float* P, const float* s, const float* D, int32_t nx, int32_t ny,
                                  int32_t nz, float scale, float tau, float tau_lambda, void* stream);

/* FP64 reductions: kind 0 = dot(a,b), 1 = nrm2(a)^2 (sum of squares),
 * 2 = asum(a).  out_dev: one double in device memory.  The per-block partial
 * sums use a buffer taken from the device's stream-ordered memory pool on
 * `stream` and returned in stream order (cudaMallocAsync / cudaFreeAsync), so
 * calls on different streams or host threads never share it. */
CBCT_API cbct_status cbct_reduce_f64(int32_t kind, const float* a, const float* b, size_t n,
                            double* out_dev, void* stream);

/* The same FP64 reduction for callers that cannot allocate device memory.
 * No counterpart in the reference: it exists for code that must not call
 * cudaMalloc while it runs, such as a latency-bound caller sharing the GPU
 * with other work (cudaMalloc may wait for the whole device to go idle) or a
 * host whose device memory is owned by another allocator (a framework's
 * caching allocator) that forbids side allocations.  cbct_reduce_f64 takes its
 * partial-sum buffer from the stream-ordered pool on every call; this entry
 * point allocates nothing and calls no allocating routine.
 * Scratch: the per-block partial sums live in a static device array of 1024
 * doubles (8 KiB) that every GPU which loads the library holds until the
 * process exits.  A call needs min(592, ceil(n/256)) of them: the reduction's
 * grid is capped at 592 blocks, so every n fits (a build whose launch shape
 * needed more than 1024 would reject the call with CBCT_ERR_INVALID_ARGUMENT).
 * Set-up: the first call on each device looks up the array's device address
 * (with that device current); make that first call before any stream capture.
 * The looked-up address is kept for the life of the library, which assumes
 * the device is not reset (cudaDeviceReset) in between.
 * All calls share the array: each call writes every partial it reads, so an
 * earlier call's leftovers never reach a result, but calls that overlap on the
 * GPU (different streams with no ordering between them) race on it. */
CBCT_API cbct_status cbct_reduce_f64_noalloc(int32_t kind, const float* a, const float* b, size_t n,
                                             double* out_dev, void* stream);

/* ----------------------------------------------------------------------------
 * Solvers (device-resident loops)
 * ------------------------------------------------------------------------- */

typedef struct {
  int32_t iterations;      /* default 10 (osMOMSolverD.h:23) */
  float beta;              /* default 1 */
  float gamma;             /* default 0 */
  int32_t non_negativity;  /* clamp x at 0 after each update */
  int32_t use_graph;       /* capture one iteration in a CUDA graph and replay it */
  cbct_dtype storage;      /* storage type of the forward projector's volume input */
  int32_t refine_every;    /* mixed precision: FP32 forward every n iterations (0 = never) */
  cbct_dtype proj_storage; /* storage type of the measured projections b (OS-MOM); the residual stays FP32 */
  /* OS-MOM total-variation regularisation (osMOMSolverD with a cuTVPrimalDualOperator:
   * denoise and updateG of osMOMSolverD.h:205-247, operators/cuTVPrimalDualOperator.cu;
   * the updateG that osMOMSolverD<cuNDArray<float>> runs): tv_weight > 0 turns
   * it on (the operator's weight), tv_alpha is its alpha, tau the solver's tau
   * (reference default 1e-3), reg_steps its primal-dual steps per subset step
   * (reference default 1).  Regularised solves run eagerly (use_graph ignored). */
  float tv_weight;
  float tv_alpha;
  float tau;
  int32_t reg_steps;
} cbct_solver_params;

/* osMOMSolverD<cuNDArray<float>>::solve without regularisers
 * (solvers/osMOMSolverD.h:82-196) on the plan's subsets.
 * b: measured projections (subset-contiguous) of type params->proj_storage,
 * x0: initial image or NULL,
 * z_out: result (the momentum point z, as the reference returns).
 * resid_norm2_out: NULL or device array of iterations*n_subsets doubles that
 * receives ||A_s x - b_s||^2 of every subset step. */
CBCT_API cbct_status cbct_osmom_solve(cbct_plan* plan, const void* b, const float* x0, float* z_out,
                             const cbct_solver_params* params, double* resid_norm2_out,
                             void* stream);

/* osSARTSolver<cuNDArray<float>>::solve (solvers/osSARTSolver.h:33-126):
 * cost_out: NULL or device array of `iterations` doubles, ||A x - b||^2 after
 * each iteration (the "Function value" print of :110-116). */
CBCT_API cbct_status cbct_ossart_solve(cbct_plan* plan, const float* b, const float* x0, float* x_out,
                              const cbct_solver_params* params, double* cost_out, void* stream);

/* ----------------------------------------------------------------------------
 * Batched reconstruction of many independent scans
 * ------------------------------------------------------------------------- */

typedef struct {
  cbct_plan* plan;              /* the scan's geometry and subsets */
  const void* b;                /* measured projections (subset-contiguous, type params.proj_storage), device */
  const float* x0;              /* initial image or NULL */
  float* z_out;                 /* result, device */
  cbct_solver_params params;    /* use_graph is forced on */
  double* resid_norm2_out;      /* NULL or device array of iterations*n_subsets doubles */
} cbct_batch_item;

/* Runs n independent osMOMSolverD reconstructions (cbct_osmom_solve semantics)
 * concurrently on up to n_streams internal streams.  Items are ordered largest
 * first; an item whose forward launches fill the GPU four times or more runs
 * on the first stream after the other such items, the others go to the
 * least-loaded of the remaining streams; each item replays its own plan's
 * captured CUDA graph.  Items must not share plans or output buffers.
 * Every kernel of an item reads only that item's buffers, so each result is
 * bitwise identical to the item solved alone.  The work starts after all work
 * already enqueued on `stream` and the call returns once every item has
 * finished (later work on `stream` is ordered after it).
 * No counterpart in the reference (its drivers reconstruct one scan per process). */
CBCT_API cbct_status cbct_batch_osmom(const cbct_batch_item* items, int32_t n, int32_t n_streams, void* stream);

/* The same reconstructions advanced in lockstep through work-list launches,
 * the items split into two groups of about equal work whose schedules run
 * side by side: step k of a group runs subset k mod S_i of iteration k / S_i
 * of every item of the group that has one.  A step is one persistent forward launch per projector kind and box
 * width and one persistent back-projection (OS-MOM update fused) per box width
 * over all those items; resident CTAs take (scan, tile) items from a counter
 * until the list is empty.  The whole schedule, preconditioner included, is
 * captured and replayed as one CUDA graph.  Items may differ in volume,
 * detector, views, subsets and iterations.  Each result is bitwise identical
 * to cbct_osmom_solve of the item alone.  Requires params.storage = CBCT_F32,
 * no bins and no regulariser (CBCT_ERR_UNSUPPORTED otherwise).  Items must not
 * share plans or outputs; ordering as cbct_batch_osmom.
 * No counterpart in the reference. */
CBCT_API cbct_status cbct_batch_osmom_fused(const cbct_batch_item* items, int32_t n, void* stream);

/* ----------------------------------------------------------------------------
 * Host-array operators streamed in batches of views
 *
 * hoCuConebeamProjectionOperator::mult_M / mult_MH (hoCuConebeamProjectionOperator.cpp:104-265)
 * over the reference's host-array projectors (conebeam_projection.cu:640-819 and
 * :1300-1649).  The plan's subsets [s_first, s_first + n_batches) are the batches of
 * one bin; view_index (n_views ints, plan order) gives each plan view's position in
 * the host projection array proj_host (W*H*P_acquisition floats, acquisition
 * order).  The bin's volume (nx*ny*nz floats, host) stays on the device while
 * the projections pass through two device batch buffers, the copy engine moving
 * one batch while the kernels run on another.  The work starts after the work
 * enqueued on `stream`; the calls return once the host outputs are written.
 * Host arrays should be page-locked for the copies to overlap the kernels.
 * ------------------------------------------------------------------------- */

/* mult_M of one bin: proj_host[view_index[v]] = A_v vol_host for every view v of
 * the batches; offset_sqrt = 1 applies the sqrt offset weight to each projected
 * batch (mult_M without FBP, hoCuConebeamProjectionOperator.cpp:168-169). */
CBCT_API cbct_status cbct_host_forward(cbct_plan* plan, int32_t s_first, int32_t n_batches, const float* vol_host,
                                       float* proj_host, const int32_t* view_index, int32_t offset_sqrt,
                                       void* stream);

/* mult_MH of one bin: vol_host = scale * ((accumulate ? vol_host : 0) + A^T p).
 * fbp = 1: each batch is FDK-filtered first (cosine, ramp with `filter` or the
 * default, plus fdk_flags: CBCT_FDK_PARKER, CBCT_FDK_OFFSET) and back-projected
 * with the 1/U^2 weight, and scale is the bin's 2/P; fbp = 0: the sqrt offset
 * weight when offset_sqrt = 1, plain back-projection, scale 1 as the reference. */
CBCT_API cbct_status cbct_host_backproject(cbct_plan* plan, int32_t s_first, int32_t n_batches,
                                           const float* proj_host, float* vol_host, const int32_t* view_index,
                                           int32_t fbp, const float* filter, uint32_t fdk_flags,
                                           int32_t offset_sqrt, float scale, int32_t accumulate, void* stream);

/* ----------------------------------------------------------------------------
 * Serving loop: continuous batching of FDK and OS-MOM reconstructions
 *
 * No counterpart in the reference (its drivers reconstruct one scan per
 * process).  A server owns max_inflight request slots, each a host worker
 * with its own CUDA stream, and a stream-ordered device memory pool.  A
 * submitted request waits until a slot is idle and its device footprint
 * (cbct_server_request_bytes) fits into what the admitted requests leave of
 * the budget; the oldest waiting request that fits is admitted first, and a
 * request passed over 8 times blocks younger ones until it fits.  An admitted
 * request builds its plan (set-up rules of CBSubsetOperator::setup and
 * hoCuConebeamProjectionOperator::setup), copies its projections host ->
 * device into subset order, reconstructs, copies the volume device -> host
 * and releases its memory.  Requests on different slots overlap on the GPU;
 * no kernel of one request reads another's memory, so each result is bitwise
 * identical to the same request served alone.
 * ------------------------------------------------------------------------- */

typedef struct cbct_server cbct_server;

typedef struct {
  size_t hbm_budget_bytes;   /* device memory the admitted requests may hold together */
  int32_t max_inflight;      /* request slots (streams and host workers), >= 1 */
  int32_t device;            /* CUDA device ordinal */
} cbct_server_config;

enum { CBCT_REQ_FDK = 0, CBCT_REQ_OSMOM = 1 };

typedef struct {
  int32_t kind;                /* CBCT_REQ_FDK or CBCT_REQ_OSMOM */
  cbct_geometry geometry;
  const float* angles_deg;     /* host, n_views, acquisition order (copied at submit) */
  const float* offsets_xy;     /* host, 2*n_views, or NULL for zero offsets (copied at submit) */
  int32_t n_views;
  int32_t n_subsets;           /* OS-MOM: round-robin subsets of CBSubsetOperator::setup */
  cbct_dtype storage;          /* device storage of the measured projections (FP32 arithmetic;
                                  volumes stay FP32) */
  const void* proj_host;       /* host, W*H*n_views values of type `storage`, acquisition order;
                                  must stay valid until the request completes */
  float* vol_host;             /* host, nx*ny*nz floats, written when the request completes */
  cbct_solver_params params;   /* OS-MOM; proj_storage is set from `storage`, storage to CBCT_F32 */
  const float* filter;         /* FDK: host array of W+1 floats, or NULL for the default (copied) */
  uint32_t fdk_flags;          /* FDK: CBCT_FDK_OFFSET / CBCT_FDK_PARKER in addition to the rules */
  int32_t offset_correction;   /* -1: the reference's override rule (per subset for OS-MOM); 0 off; 1 on */
} cbct_request;

typedef struct {
  cbct_status status;          /* the request's outcome */
  int32_t slot;                /* slot that ran it */
  double t_submit, t_admit, t_done;  /* seconds on the server's clock */
  size_t bytes_reserved;       /* admission footprint */
  size_t bytes_peak;           /* peak of the device buffers the request held */
  char message[256];           /* error message when status != CBCT_OK */
} cbct_request_info;

CBCT_API cbct_status cbct_server_create(const cbct_server_config* cfg, cbct_server** server_out);

/* Device bytes the request will hold while it runs (its admission footprint). */
CBCT_API cbct_status cbct_server_request_bytes(const cbct_request* req, size_t* bytes_out);

/* Queues a request; returns at once.  CBCT_ERR_BUDGET when its footprint
 * exceeds the whole budget. */
CBCT_API cbct_status cbct_server_submit(cbct_server* server, const cbct_request* req, uint64_t* ticket_out);

/* Waits up to timeout_s seconds (< 0: no limit) for a request.  Returns
 * CBCT_OK once it has completed (info->status is its outcome; the ticket is
 * then released) and CBCT_ERR_TIMEOUT if it has not. */
CBCT_API cbct_status cbct_server_wait(cbct_server* server, uint64_t ticket, double timeout_s,
                                      cbct_request_info* info_out);

/* Seconds on the server's clock (steady, zero at creation). */
CBCT_API cbct_status cbct_server_now(cbct_server* server, double* t_out);

/* Serves every queued request, then releases the slots and the pool. */
CBCT_API cbct_status cbct_server_destroy(cbct_server* server);

/* ----------------------------------------------------------------------------
 * Synthetic phantoms (seeded ellipsoids; used by the benchmarks and tests)
 * Ellipsoid record (10 floats): cx cy cz ax ay az phi theta psi density,
 * rotation R = Rz(phi) Ry(theta) Rx(psi).
 * ------------------------------------------------------------------------- */
CBCT_API cbct_status cbct_phantom_voxelize(const cbct_geometry* g, const float* ellipsoids_dev,
                                  int32_t n_ellipsoids, int32_t supersample, float* vol,
                                  void* stream);
/* Exact line integrals of the box-truncated phantom along every ray of subset s. */
CBCT_API cbct_status cbct_phantom_project(cbct_plan* plan, int32_t s, const float* ellipsoids_dev,
                                 int32_t n_ellipsoids, float* proj, void* stream);

/* Element-wise conversion of n floats to a 16-bit storage type (dst_dtype). */
CBCT_API cbct_status cbct_convert(const float* src, void* dst, size_t n, cbct_dtype dst_dtype,
                         void* stream);

#ifdef __cplusplus
}
#endif

#endif /* CBCT_H_ */
