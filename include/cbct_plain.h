/* cbct_plain.h -- the plain FP32 one-scan-at-a-time GPU path (measurement baseline).
 *
 * A restatement of gt-tomography's own CUDA path as it runs today, re-hosted on
 * sm_100a: texture objects with hardware linear filtering (normalised
 * coordinates, border 0, 9-bit interpolation weights) in place of the removed
 * texture references (xray/conebeam_projection.cu:35-42), one thread per ray
 * or voxel, a whole-volume / whole-subset cudaArray copy, per-call uploads and
 * allocations on every call, element-wise solver passes and a host-synchronised
 * residual norm per subset step (osMOMSolverD.h:139-181 in OUTPUT_VERBOSE mode,
 * as cuCBOS_reconstruct.cpp runs it), compiled with --use_fast_math like the
 * reference (CMakeLists.txt:52).  It is the denominator of the recon/s
 * comparison and the stand-in for "the reference's CUDA projector outputs".
 * Not the product path: the product entry points are in cbct.h.
 *
 * Arguments follow cbct.h: device pointers, host angle/offset arrays, views of
 * one call, layouts (W,H,P) and (nx,ny,nz).  Every call synchronises the device.
 */
#ifndef CBCT_PLAIN_H_
#define CBCT_PLAIN_H_

#include "cbct.h"

#ifdef __cplusplus
extern "C" {
#endif

/* conebeam_forwards_projection (conebeam_projection.cu:530-635). */
CBCT_API cbct_status cbct_plain_forward(const cbct_geometry* g, const float* angles_deg, const float* offsets_xy,
                                        int32_t n_views, const float* vol, float* proj, int32_t accumulate);

/* conebeam_backwards_projection (conebeam_projection.cu:1172-1299) as called by
 * cuConebeamProjectionOperator::mult_MH (.cpp:82-116): with offset correction
 * the input is copied and the copy weighted (sin^2) first. */
CBCT_API cbct_status cbct_plain_backproject(const cbct_geometry* g, const float* angles_deg,
                                            const float* offsets_xy, int32_t n_views, const float* proj, float* vol,
                                            int32_t offset_correction, int32_t accumulate);

/* osMOMSolverD::solve without regularisers over n_subsets subsets of
 * subset-contiguous views, with the reference's call structure.  resid_norm2
 * (host array of iterations*n_subsets doubles, nullable) receives the
 * per-subset-step ||A_s x - b_s||^2 the reference prints. */
CBCT_API cbct_status cbct_plain_osmom_solve(const cbct_geometry* g, const float* angles_deg,
                                            const float* offsets_xy, int32_t n_views, const int32_t* subset_sizes,
                                            int32_t n_subsets, const int32_t* offset_correction, const float* b,
                                            float* z_out, int32_t iterations, int32_t non_negativity,
                                            double* resid_norm2);

/* hoCuConebeamProjectionOperator::mult_MH with filtered back-projection
 * (hoCuConebeamProjectionOperator.cpp:235-254 over conebeam_backwards_projection<true>,
 * conebeam_projection.cu:1300-1649): HOST projections (W,H,P) in, HOST volume
 * out, views_per_batch views per batch (the operator's default is 20), cuFFT
 * for the row filter as in the reference (loaded on first use), no Parker
 * weights (full-scan orbits only).  filter: W+1 floats or NULL (default).
 * Angles are used as given (start them at 0 as the operator's setup does). */
CBCT_API cbct_status cbct_plain_fdk(const cbct_geometry* g, const float* angles_deg, const float* offsets_xy,
                                    int32_t n_views, const float* proj_host, float* vol_host, const float* filter,
                                    int32_t offset_correction, int32_t views_per_batch);

/* Device-only times of the reference's two kernels (conebeam_forwards_projection_kernel,
 * conebeam_projection.cu:412-528, and conebeam_backwards_projection_kernel<false>, :922-1037)
 * on the same views: the volume and the projections are copied into their
 * texture arrays once, then each kernel is launched reps times between CUDA
 * events on the legacy stream.  proj_out (W*H*n floats) and vol_out receive the
 * kernels' results; ms_out[0] = forward, ms_out[1] = back-projection, ms per launch. */
CBCT_API cbct_status cbct_plain_kernel_times(const cbct_geometry* g, const float* angles_deg,
                                             const float* offsets_xy, int32_t n_views, const float* vol,
                                             const float* proj, float* proj_out, float* vol_out, int32_t reps,
                                             float* ms_out);

#ifdef __cplusplus
}
#endif

#endif /* CBCT_PLAIN_H_ */
