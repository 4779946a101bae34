// device_common.cuh -- device helpers shared by the cone-beam kernels.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstdint>

#include "cbct_internal.h"

namespace cbct {

// ------------------------------------------------------------ storage types
template <class V> __device__ __forceinline__ float ld_f(const V* p);
template <> __device__ __forceinline__ float ld_f<float>(const float* p) { return __ldg(p); }
template <> __device__ __forceinline__ float ld_f<__half>(const __half* p) {
  return __half2float(__ldg(p));
}
template <> __device__ __forceinline__ float ld_f<__nv_bfloat16>(const __nv_bfloat16* p) {
  return __bfloat162float(__ldg(p));
}
// Element i of an array whose storage type is chosen at run time (cbct_dtype).
__device__ __forceinline__ float ld_any(const void* p, size_t i, int dtype) {
  if (dtype == CBCT_F16) return ld_f(static_cast<const __half*>(p) + i);
  if (dtype == CBCT_BF16) return ld_f(static_cast<const __nv_bfloat16*>(p) + i);
  return ld_f(static_cast<const float*>(p) + i);
}

template <class V> __device__ __forceinline__ float sm_f(V v);
template <> __device__ __forceinline__ float sm_f<float>(float v) { return v; }
template <> __device__ __forceinline__ float sm_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float sm_f<__nv_bfloat16>(__nv_bfloat16 v) {
  return __bfloat162float(v);
}

// ------------------------------------------------------------ geometry
// Ray of pixel (u,v): texel-space start c0, texel-space step dc, and the
// ray-sum scale delta (conebeam_projection.cu:441-500).  span = a2 - a1.
struct Ray {
  float c0x, c0y, c0z;
  float dcx, dcy, dcz;
  float delta;
  float a1, a2;
};

__device__ __forceinline__ Ray make_ray(const ViewParams& vp, const GridConst& gc, int u, int v) {
  Ray r;
  const float dx = fmaf(float(u), vp.Eux, vp.D0x);
  const float dy = fmaf(float(u), vp.Euy, vp.D0y);
  const float dz = fmaf(float(v), vp.Evz, vp.D0z);
  // Box clip in world coordinates (conebeam_projection.cu:478-484).
  const float tx1 = __fdiv_rn(gc.hx - vp.Sx, dx), tx2 = __fdiv_rn(-gc.hx - vp.Sx, dx);
  const float ty1 = __fdiv_rn(gc.hy - vp.Sy, dy), ty2 = __fdiv_rn(-gc.hy - vp.Sy, dy);
  const float tz1 = __fdiv_rn(gc.hz, dz), tz2 = __fdiv_rn(-gc.hz, dz);
  const float a1 = fmaxf(fmaxf(fmaxf(fminf(tx1, tx2), fminf(ty1, ty2)), fminf(tz1, tz2)), 0.f);
  const float a2 = fminf(fminf(fminf(fmaxf(tx1, tx2), fmaxf(ty1, ty2)), fmaxf(tz1, tz2)), 1.f);
  const float span = a2 - a1;
  const float len = sqrtf(fmaf(dx, dx, fmaf(dy, dy, dz * dz)));
  r.delta = fabsf(span) * len * gc.invN;
  const float f = span * gc.invN;
  // texel coordinate = world * k + b ; start point S + a1*d
  r.c0x = fmaf(fmaf(a1, dx, vp.Sx), gc.kx, gc.bx);
  r.c0y = fmaf(fmaf(a1, dy, vp.Sy), gc.ky, gc.by);
  r.c0z = fmaf(a1 * dz, gc.kz, gc.bz);
  r.dcx = dx * f * gc.kx;
  r.dcy = dy * f * gc.ky;
  r.dcz = dz * f * gc.kz;
  r.a1 = a1;
  r.a2 = a2;
  return r;
}

// ------------------------------------------------------------ rounding
// floor(x) for |x| < 2^22 on the FMA pipe instead of the conversion unit:
// x + 1.5 * 2^23 rounded toward -infinity is floor(x) + 1.5 * 2^23 (the sum's
// last place is 1), and subtracting the constant again is exact.  The result
// equals floorf(x).
constexpr float kRoundC = 12582912.f;      // 1.5 * 2^23
constexpr int kRoundBits = 0x4B400000;     // its bit pattern
__device__ __forceinline__ float floor_small(float x) { return __fadd_rd(x, kRoundC) - kRoundC; }
// The integer v (|v| < 2^22) held by a float s = v + 1.5 * 2^23: its low mantissa bits.
__device__ __forceinline__ int int_of_biased(float s) { return __float_as_int(s) - kRoundBits; }

// Bounds-checked trilinear fetch from global memory at texel coordinates
// (border texels read as 0, as cudaAddressModeBorder does).
template <class V>
__device__ __forceinline__ float fetch3_global(const V* __restrict__ vol, int nx, int ny, int nz,
                                               float cx, float cy, float cz) {
  const float fx = floorf(cx), fy = floorf(cy), fz = floorf(cz);
  const float ax = cx - fx, ay = cy - fy, az = cz - fz;
  const int ix = int(fx), iy = int(fy), iz = int(fz);
  const bool vx0 = (unsigned)ix < (unsigned)nx, vx1 = (unsigned)(ix + 1) < (unsigned)nx;
  const bool vy0 = (unsigned)iy < (unsigned)ny, vy1 = (unsigned)(iy + 1) < (unsigned)ny;
  const bool vz0 = (unsigned)iz < (unsigned)nz, vz1 = (unsigned)(iz + 1) < (unsigned)nz;
  const int x0 = min(max(ix, 0), nx - 1), x1 = min(max(ix + 1, 0), nx - 1);
  const int y0 = min(max(iy, 0), ny - 1), y1 = min(max(iy + 1, 0), ny - 1);
  const int z0 = min(max(iz, 0), nz - 1), z1 = min(max(iz + 1, 0), nz - 1);
  const size_t sxy = (size_t)nx * ny;
  const size_t r00 = (size_t)z0 * sxy + (size_t)y0 * nx, r10 = (size_t)z0 * sxy + (size_t)y1 * nx;
  const size_t r01 = (size_t)z1 * sxy + (size_t)y0 * nx, r11 = (size_t)z1 * sxy + (size_t)y1 * nx;
  const float v000 = (vx0 && vy0 && vz0) ? ld_f(vol + r00 + x0) : 0.f;
  const float v100 = (vx1 && vy0 && vz0) ? ld_f(vol + r00 + x1) : 0.f;
  const float v010 = (vx0 && vy1 && vz0) ? ld_f(vol + r10 + x0) : 0.f;
  const float v110 = (vx1 && vy1 && vz0) ? ld_f(vol + r10 + x1) : 0.f;
  const float v001 = (vx0 && vy0 && vz1) ? ld_f(vol + r01 + x0) : 0.f;
  const float v101 = (vx1 && vy0 && vz1) ? ld_f(vol + r01 + x1) : 0.f;
  const float v011 = (vx0 && vy1 && vz1) ? ld_f(vol + r11 + x0) : 0.f;
  const float v111 = (vx1 && vy1 && vz1) ? ld_f(vol + r11 + x1) : 0.f;
  const float c00 = fmaf(ax, v100 - v000, v000), c10 = fmaf(ax, v110 - v010, v010);
  const float c01 = fmaf(ax, v101 - v001, v001), c11 = fmaf(ax, v111 - v011, v011);
  const float c0 = fmaf(ay, c10 - c00, c00), c1 = fmaf(ay, c11 - c01, c01);
  return fmaf(az, c1 - c0, c0);
}

// Wang offset weight of detector column u (sin^2 variant with zeroing,
// offset_correct_kernel, conebeam_projection.cu:233-262).  o = offset_x.
__device__ __forceinline__ float offset_weight_full(float fov_u, int W, int u, float o) {
  const float sg = o / fabsf(o);  // NaN for o == 0: no weight (comparisons fail)
  const float t = (fov_u * (float(u) / float(W) - 0.5f) + o) * sg;
  const float omega = fov_u * 0.5f - fabsf(o);
  float w = 1.f;
  if (fabsf(t) <= omega) {
    const float s = sinf(3.14159265358979f * (t + omega) / (4.f * omega));
    w = s * s;
  }
  if (t < -omega) w = 0.f;
  return w;
}

// sqrt variant (offset_correct_kernel_sqrt, conebeam_projection.cu:303-331).
__device__ __forceinline__ float offset_weight_sqrt(float fov_u, int W, int u, float o) {
  const float sg = o / fabsf(o);
  const float t = (fov_u * ((float(u) + 0.5f) / float(W) - 0.5f) + o) * sg;
  const float omega = fov_u * 0.5f - fabsf(o);
  float w = 1.f;
  if (fabsf(t) <= fabsf(omega)) w = sinf(3.14159265358979f * (t + omega) / (4.f * omega));
  return w;
}

// ------------------------------------------------------------ mbarrier + TMA
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count)
               : "memory");
}

// Retires an mbarrier with no pending arrivals or copies, so that the CTA of
// a work-list kernel may initialise it again for its next item.
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Scans per work-list launch (their first-item indices are kept in shared
// memory by every CTA).
constexpr int kMultiMaxRecs = 64;

// Index of the last entry of base[0..n) (ascending) that is <= t.
__device__ __forceinline__ int find_rec(const int* base, int n, int t) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (base[mid] <= t) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// Orders this thread's later TMA reads of a tensor map that sits in global
// memory (written by a host copy before the launch) after its generic-proxy
// contents.
__device__ __forceinline__ void tensormap_acquire(const void* map) {
  asm volatile("fence.proxy.tensormap::generic.acquire.sys [%0], 128;" ::"l"(map) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(bytes)
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Bounded wait: gives up after `limit` polls (each try_wait itself blocks for a
// hardware-defined interval) and returns false.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, uint32_t limit) {
  for (uint32_t i = 0; i < limit; ++i) {
    if (mbar_try_wait(bar, parity)) return true;
    if (i > 64) __nanosleep(128);
  }
  return false;
}

// 3-D tiled TMA load (no multicast) into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int x, int y, int z,
                                            uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
      : "memory");
}

// 1-D bulk copy global -> shared (no multicast), completing on bar.  Both
// addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

// ------------------------------------------------------------ reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide FP64 sum in a fixed order (deterministic); result valid in thread 0.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* sh /* NT/32 doubles */) {
  v = warp_sum(v);
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) sh[w] = v;
  __syncthreads();
  double r = 0;
  if (threadIdx.x < 32) {
    r = (l < NT / 32) ? sh[l] : 0.0;
    r = warp_sum(r);
  }
  return r;
}

}  // namespace cbct
