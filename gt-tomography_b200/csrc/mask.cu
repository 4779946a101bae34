// mask.cu -- space carver and voxel masks.
//
// conebeam_spacecarver_kernel (xray/conebeam_projection.cu:822-921): for each
// voxel centre, with its z coordinate negated as the reference does (:852), the
// projection of every view of the call is point-sampled (texel floor(u*W),
// border 0; projections_mask_tex at :41-42 uses point filtering).  Views whose
// sample is nonzero and below `limit` are counted; the voxel stays in the mask
// when fewer than 3 views were counted.  apply_mask (:1651-1657) multiplies an
// image by the mask.
#include "device_common.cuh"

namespace cbct {

namespace {

__global__ void spacecarver_kernel(const float* __restrict__ proj, const ViewParams* __restrict__ views, int P,
                                   GridConst gc, float limit, unsigned char* __restrict__ mask, int combine) {
  const size_t n = (size_t)gc.nx * gc.ny * gc.nz;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    const int i = int(idx % gc.nx), j = int((idx / gc.nx) % gc.ny), k = int(idx / ((size_t)gc.nx * gc.ny));
    const float x = fmaf(float(i) + 0.5f, gc.vx, -gc.hx);
    const float y = fmaf(float(j) + 0.5f, gc.vy, -gc.hy);
    const float z = -fmaf(float(k) + 0.5f, gc.vz, -gc.hz);
    int count = 0;
    for (int p = 0; p < P; ++p) {
      const ViewParams& vp = views[p];
      const float xr = fmaf(vp.cs, x, vp.sn * y);
      const float yr = fmaf(-vp.sn, x, vp.cs * y);
      const float dy = yr + gc.SAD;
      const float ex = gc.SDD * __fdiv_rn(xr, dy) - vp.ox;
      const float ez = gc.SDD * __fdiv_rn(z, dy) - vp.oy;
      const float un = ex / gc.fov_u + 0.5f, vn = ez / gc.fov_v + 0.5f;
      const int iu = int(floorf(un * float(gc.W))), iv = int(floorf(vn * float(gc.H)));
      float t = 0.f;
      if ((unsigned)iu < (unsigned)gc.W && (unsigned)iv < (unsigned)gc.H)
        t = __ldg(proj + ((size_t)p * gc.H + iv) * gc.W + iu);
      if (t < limit && t != 0.f) ++count;
    }
    const unsigned char m = count < 3 ? 1 : 0;
    mask[idx] = combine ? (unsigned char)(mask[idx] & m) : m;
  }
}

__global__ void apply_mask_kernel(float* __restrict__ vol, const unsigned char* __restrict__ mask, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    vol[i] = vol[i] * float(mask[i]);
}

__global__ void mul_kernel(float* out, const float* in, const float* __restrict__ w, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = in[i] * w[i];
}

}  // namespace

void mul_launch(float* out, const float* in, const float* w, size_t n, cudaStream_t st) {
  if (n == 0) return;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  mul_kernel<<<blocks, 256, 0, st>>>(out, in, w, n);
  check_launch("mul_kernel");
}

void spacecarver_launch(cbct_plan* p, int s, const float* proj, float limit, unsigned char* mask, int combine,
                        cudaStream_t st) {
  const size_t n = (size_t)p->g.nx * p->g.ny * p->g.nz;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  spacecarver_kernel<<<blocks, 256, 0, st>>>(proj, p->d_views + p->first[s], p->count[s], p->gc, limit, mask, combine);
  check_launch("spacecarver_kernel");
}

void apply_mask_launch(float* vol, const unsigned char* mask, size_t n, cudaStream_t st) {
  if (n == 0) return;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  apply_mask_kernel<<<blocks, 256, 0, st>>>(vol, mask, n);
  check_launch("apply_mask_kernel");
}

}  // namespace cbct
