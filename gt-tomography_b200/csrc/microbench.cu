// microbench.cu -- the on-chip ceiling of the projectors' inner operation.
//
// The forward projector's work is FP32 software trilinear interpolation from a
// shared-memory box (8 taps, 7 lerps per ray sample); the back-projector's is
// bilinear interpolation from a shared-memory detector box (4 taps, 3 lerps
// per voxel-view).  Both are bound on chip (shared-memory wavefronts and FP32
// issue), not by HBM, so their roofline is the rate of that operation alone.
// These kernels measure it: every thread of a full grid interpolates from a
// shared-memory box at the projectors' access pattern (lanes of a warp half a
// texel apart across the box's fast axis, samples 0.67 texel apart along a
// ray, the same floor / index / paired-lerp arithmetic), with nothing else in
// the loop: no TMA, no slab changes, no clipping, no epilogue.  A projector
// timed against this rate shows how much of its time goes to the operation it
// cannot avoid; a projector that shares taps between rays (the row-pair and
// row-quad kernels) can exceed it.
#include <algorithm>
#include <string>

#include "device_common.cuh"

namespace cbct {

namespace {

constexpr int kMbThreads = 256;
constexpr int kMbGroup = 8;          // samples per group; positions restart along the ray after each

__device__ __forceinline__ float2 lerp2f(float2 a, float2 b, float2 t) {
  return __ffma2_rn(t, make_float2(b.x - a.x, b.y - a.y), a);
}

// Trilinear: a 40 x 10 x 24 box (the forward projectors' box shape).  Thread
// (tx, ty) = (tid % 16, tid / 16), a ray of a 16 x 16 tile, starts at
// e = 2 + 0.53 tx, z = 2 + 0.61 ty, d = 0.3 + 0.011 tx (the rays of a tile
// cross the slab rows together); per sample d advances 0.67, e 0.031,
// z 0.017.  Bounds (checked by hand for the sizes below): d <= 0.47 + 7 * 0.67
// = 5.16, e < 28 + 0.22, z < 19 + 0.12, so the highest tap index is
// 29 + 6 * 40 + 20 * 400 = 8269 < 9600.
__global__ void __launch_bounds__(kMbThreads) trilinear_peak_kernel(float* __restrict__ out, int groups) {
  constexpr int BX = 40, BY = 10, BZ = 24, BXY = BX * BY;
  __shared__ float box[BX * BY * BZ];
  for (int i = threadIdx.x; i < BX * BY * BZ; i += kMbThreads) box[i] = float((i * 37) % 101) * 0.01f;
  __syncthreads();
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float ce = 2.f + 0.53f * float(tx), cz = 2.f + 0.61f * float(ty);
  const float cd = 0.3f + 0.011f * float(tx);
  const float de = 0.031f, dd = 0.67f, dz = 0.017f;
  float acc = 0.f;
  for (int g = 0; g < groups; ++g) {
    float v[kMbGroup];
#pragma unroll
    for (int k = 0; k < kMbGroup; ++k) {
      const float2 p = __ffma2_rn(make_float2(float(k), float(k)), make_float2(de, dd), make_float2(ce, cd));
      const float z = fmaf(float(k), dz, cz);
      const float fe = floor_small(p.x), fd = floor_small(p.y), fz = floor_small(z);
      const float2 a = __fadd2_rn(p, make_float2(-fe, -fd));
      const float az = z - fz;
      const int idx = int_of_biased(fmaf(fz, float(BXY), fmaf(fd, float(BX), fe)) + kRoundC);
      const float* q = box + idx;
      const float2 a0 = make_float2(q[0], q[BX]), b0 = make_float2(q[1], q[BX + 1]);
      const float2 a1 = make_float2(q[BXY], q[BXY + BX]), b1 = make_float2(q[BXY + 1], q[BXY + BX + 1]);
      const float2 te = make_float2(a.x, a.x);
      const float2 e0 = lerp2f(a0, b0, te), e1 = lerp2f(a1, b1, te);
      const float2 d2 = lerp2f(make_float2(e0.x, e1.x), make_float2(e0.y, e1.y), make_float2(a.y, a.y));
      v[k] = fmaf(az, d2.y - d2.x, d2.x);
    }
#pragma unroll
    for (int k = 0; k < kMbGroup; ++k) acc += v[k];
    ce += float(kMbGroup) * de;
    if (ce >= 28.f) ce -= 24.f;
    cz += float(kMbGroup) * dz;
    if (cz >= 19.f) cz -= 16.f;
  }
  out[(size_t)blockIdx.x * kMbThreads + threadIdx.x] = acc;
}

// Bilinear: a 72 x 40 detector box (the back-projector's box at the benchmark
// geometry).  Warps hold 8 x 4 voxel columns as the back-projector's do: lane
// (l % 8, l / 8) of warp w takes detector column cu = 3 + 0.55 (l % 8) + 4.4 (w & 1)
// and row cv = 2 + 0.55 (l / 8) + 2.2 (w >> 1); per voxel of its z-run the row
// advances 0.61, per group (one "view") the column 0.29 and the run restarts.
// Bounds: cu starts at most at 11.25 and wraps to stay in [3, 60), so the
// right tap column is at most 60; cv <= 2 + 1.65 + 6.6 + 15 * 0.61 = 19.4, so
// the lower tap row is at most 20; highest tap index 60 + 20 * 72 = 1500 < 72 * 40.
__global__ void __launch_bounds__(kMbThreads) bilinear_peak_kernel(float* __restrict__ out, int groups) {
  constexpr int BU = 72, BV = 40, ZR = 16;
  __shared__ float box[BU * BV];
  for (int i = threadIdx.x; i < BU * BV; i += kMbThreads) box[i] = float((i * 53) % 97) * 0.01f;
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float cu = 3.f + 0.55f * float(lane & 7) + 4.4f * float(warp & 1);
  const float cv0 = 2.f + 0.55f * float(lane >> 3) + 2.2f * float(warp >> 1);
  const float dv = 0.61f, du = 0.29f;
  float acc[ZR];
#pragma unroll
  for (int q = 0; q < ZR; ++q) acc[q] = 0.f;
  for (int g = 0; g < groups; ++g) {
    const float fu = floor_small(cu);
    const float au = cu - fu;
    const float2 tu = make_float2(au, au);
    const float fubc = fu + kRoundC;
    float cv = cv0;
#pragma unroll
    for (int q = 0; q < ZR; ++q) {
      const float fv = floor_small(cv);
      const float av = cv - fv;
      const int idx = int_of_biased(fmaf(fv, float(BU), fubc));
      const float* t = box + idx;
      const float2 r0 = make_float2(t[0], t[BU]);
      const float2 r1 = make_float2(t[1], t[BU + 1]);
      const float2 h = __ffma2_rn(tu, r1, __ffma2_rn(make_float2(-au, -au), r0, r0));
      acc[q] += fmaf(av, h.y - h.x, h.x);
      cv += dv;
    }
    cu += du;
    if (cu >= 60.f) cu -= 56.f;
  }
  float s = 0.f;
#pragma unroll
  for (int q = 0; q < ZR; ++q) s += acc[q];
  out[(size_t)blockIdx.x * kMbThreads + threadIdx.x] = s;
}

}  // namespace

// Runs the kernel `kind` (3 = trilinear, 2 = bilinear) over four waves of
// resident CTAs of 256 threads with `groups` groups each, once to warm up and
// `reps` times between CUDA events; returns interpolations per second.
double microbench_interp(int kind, int groups, int reps, cudaStream_t st) {
  int dev = 0, sms = 0, per_sm = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  CBCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  if (kind == 3)
    CBCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trilinear_peak_kernel, kMbThreads, 0));
  else
    CBCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bilinear_peak_kernel, kMbThreads, 0));
  const int blocks = std::max(1, sms * per_sm * 4);
  float* out = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  const size_t n = (size_t)blocks * kMbThreads;
  CBCT_CUDA(cudaMallocAsync(reinterpret_cast<void**>(&out), n * sizeof(float), st));
  float ms = 0.f;
  cudaError_t err = cudaEventCreate(&e0);
  if (err == cudaSuccess) err = cudaEventCreate(&e1);
  auto launch = [&] {
    if (kind == 3) trilinear_peak_kernel<<<blocks, kMbThreads, 0, st>>>(out, groups);
    else bilinear_peak_kernel<<<blocks, kMbThreads, 0, st>>>(out, groups);
  };
  if (err == cudaSuccess) {
    launch();
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaEventRecord(e0, st);
  for (int r = 0; r < reps && err == cudaSuccess; ++r) {
    launch();
    err = cudaGetLastError();
  }
  if (err == cudaSuccess) err = cudaEventRecord(e1, st);
  if (err == cudaSuccess) err = cudaEventSynchronize(e1);
  if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
  cudaFreeAsync(out, st);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (err != cudaSuccess) throw Error(CBCT_ERR_CUDA, std::string("microbench: ") + cudaGetErrorString(err));
  const double per = kind == 3 ? double(kMbGroup) : double(16);
  return double(n) * groups * per * reps / (double(ms) * 1e-3);
}

}  // namespace cbct
