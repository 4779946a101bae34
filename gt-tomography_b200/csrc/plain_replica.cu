// plain_replica.cu -- the plain FP32 one-scan-at-a-time GPU path (baseline).
//
// Built with --use_fast_math (see build.py), like the reference
// (CMakeLists.txt:52).  The kernels restate xray/conebeam_projection.cu with
// texture objects in place of the texture references CUDA 12 removed:
//   forward  :412-528 (tex3D, normalised coords, linear filter, border 0)
//   backward :922-1037 (tex2DLayered)
//   offset   :233-262 (sin^2 weight)
// and the host functions keep the reference's per-call structure: a cudaArray
// of the whole volume / subset is allocated and filled on every call, angles
// and offsets are uploaded on every call (thrust device_vector at :600-601,
// :1225-1226), the grid is 1-D with 256 threads (setup_grid :48-75).  The
// OS-MOM loop restates osMOMSolverD.h:82-196 with one pass per Gadgetron array
// operation, a fresh device image per subset step (:153) and in denoise (:209),
// and host-synchronised norms (:147-149, :206).
#include <cuda_runtime.h>
#include <cufft.h>
#include <dlfcn.h>
#include <math_constants.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/cbct_plain.h"
#include "cbct_internal.h"

namespace cbct {
namespace plain {

void check(cudaError_t e, const char* what) {
  if (e != cudaSuccess) throw Error(CBCT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

// setup_grid (conebeam_projection.cu:48-75): 256 threads, 1-D grid, 2-D when too long.
void setup_grid(size_t n, dim3* block, dim3* grid) {
  *block = dim3(256);
  size_t gx = (n + 255) / 256;
  unsigned gy = 1;
  if (gx > 65535) {
    gx = (unsigned)std::floor(std::sqrt(double(n) / 256.0));
    const size_t per = 256 * gx;
    gy = (unsigned)((n + per - 1) / per);
  }
  *grid = dim3((unsigned)gx, gy);
}

__device__ __forceinline__ size_t gidx() {
  return (size_t)blockIdx.y * gridDim.x * blockDim.x + (size_t)blockIdx.x * blockDim.x + threadIdx.x;
}

__global__ void fwd_kernel(float* __restrict__ projections, const float* __restrict__ angles,
                           const float2* __restrict__ offsets, float3 L, int W, int H, float2 ps_mm, int P,
                           float SDD, float SAD, int N, bool accumulate, cudaTextureObject_t tex) {
  const size_t idx = gidx();
  if (idx >= (size_t)W * H * P) return;
  const int u = int(idx % W), v = int((idx / W) % H), p = int(idx / ((size_t)W * H));
  float s, c;
  sincosf(angles[p] * (CUDART_PI_F / 180.0f), &s, &c);
  // start = R (0,-SAD,0); rows of R are (c,-s,0), (s,c,0), (0,0,1)
  float3 sp = make_float3(s * SAD, -c * SAD, 0.f);
  const float pcx = ((u + 0.5f) / float(W) - 0.5f) * ps_mm.x + offsets[p].x;
  const float pcy = ((v + 0.5f) / float(H) - 0.5f) * ps_mm.y + offsets[p].y;
  const float ADD = SDD - SAD;
  const float3 ep = make_float3(c * pcx - s * ADD, s * pcx + c * ADD, pcy);
  float3 dir = make_float3(ep.x - sp.x, ep.y - sp.y, ep.z - sp.z);
  const float vx = (L.x / 2 - sp.x) / dir.x, vy = (L.y / 2 - sp.y) / dir.y, vz = (L.z / 2 - sp.z) / dir.z;
  const float wx = (-L.x / 2 - sp.x) / dir.x, wy = (-L.y / 2 - sp.y) / dir.y, wz = (-L.z / 2 - sp.z) / dir.z;
  const float a1 = fmaxf(fmaxf(fmaxf(fminf(wx, vx), fminf(wy, vy)), fminf(wz, vz)), 0.0f);
  const float aend = fminf(fminf(fminf(fmaxf(wx, vx), fmaxf(wy, vy)), fmaxf(wz, vz)), 1.0f);
  sp.x += a1 * dir.x; sp.y += a1 * dir.y; sp.z += a1 * dir.z;
  const float dx = (aend - a1) * dir.x, dy = (aend - a1) * dir.y, dz = (aend - a1) * dir.z;
  const float sampling_distance = sqrtf(dx * dx + dy * dy + dz * dz) / N;
  sp.x = sp.x / L.x + 0.5f; sp.y = sp.y / L.y + 0.5f; sp.z = sp.z / L.z + 0.5f;
  const float f = (aend - a1) / float(N);
  dir.x = dir.x / L.x * f; dir.y = dir.y / L.y * f; dir.z = dir.z / L.z * f;
  float result = 0.0f;
  for (int k = 0; k < N; ++k)
    result += tex3D<float>(tex, sp.x + dir.x * float(k), sp.y + dir.y * float(k), sp.z + dir.z * float(k));
  projections[idx] = accumulate ? projections[idx] + result * sampling_distance : result * sampling_distance;
}

// FBP: the 1/U^2 weight of conebeam_projection.cu:1008-1026 (filtered back-projection).
template <bool FBP>
__global__ void bp_kernel(float* __restrict__ image, const float* __restrict__ angles,
                          const float2* __restrict__ offsets, int nx, int ny, int nz, float3 L, float2 ps_mm, int P,
                          float SDD, float SAD, bool accumulate, cudaTextureObject_t tex) {
  const size_t idx = gidx();
  if (idx >= (size_t)nx * ny * nz) return;
  const int i = int(idx % nx), j = int((idx / nx) % ny), k = int(idx / ((size_t)nx * ny));
  const float px = ((i + 0.5f) / nx - 0.5f) * L.x;
  const float py = ((j + 0.5f) / ny - 0.5f) * L.y;
  const float pz = ((k + 0.5f) / nz - 0.5f) * L.z;
  const float incoming = accumulate ? image[idx] : 0.0f;
  float result = 0.0f;
  for (int p = 0; p < P; ++p) {
    float s, c;
    sincosf(-(angles[p] * (CUDART_PI_F / 180.0f)), &s, &c);
    const float qx = c * px - s * py, qy = s * px + c * py;   // R(-angle) pos
    float3 d = make_float3(qx, qy + SAD, pz);
    d.x /= d.y; d.z /= d.y; d.y = 1.0f;
    const float ex = SDD * d.x - offsets[p].x, ez = SDD * d.z - offsets[p].y;
    const float uu = ex / ps_mm.x + 0.5f, vv = ez / ps_mm.y + 0.5f;
    float weight = 1.0f;
    if (FBP) {
      const float beta = angles[p] * (CUDART_PI_F / 180.0f);
      const float r = hypotf(px, py), phi = atan2f(py, px);
      const float U = (SAD + r * sinf(beta - phi)) / SAD;
      weight = 1.0f / (U * U);
    }
    result += weight * tex2DLayered<float>(tex, uu, vv, p);
  }
  image[idx] = incoming + result;
}

__global__ void offset_kernel(float* __restrict__ projections, const float2* __restrict__ offsets, int W, int H,
                              int P, float2 ps_mm) {
  const size_t idx = gidx();
  if (idx >= (size_t)W * H * P) return;
  const int u = int(idx % W), p = int(idx / ((size_t)W * H));
  const float o = offsets[p].x;
  const float t = (ps_mm.x * (float(u) / float(W) - 0.5f) + o) * o / fabsf(o);
  const float omega = ps_mm.x / 2.0f - fabsf(o);
  if (fabsf(t) <= omega) {
    const float sw = sinf(CUDART_PI_F * (t + omega) / (4.0f * omega));
    projections[idx] *= sw * sw;
  }
  if (t < -omega) projections[idx] *= 0;
}

// Gadgetron array operations, one pass each.
__global__ void ew_sub(float* a, const float* b, size_t n) { size_t i = gidx(); if (i < n) a[i] -= b[i]; }
__global__ void ew_mul(float* a, const float* b, size_t n) { size_t i = gidx(); if (i < n) a[i] *= b[i]; }
__global__ void ew_scale(float* a, float s, size_t n) { size_t i = gidx(); if (i < n) a[i] *= s; }
__global__ void ew_axpy(float a, const float* x, float* y, size_t n) { size_t i = gidx(); if (i < n) y[i] += a * x[i]; }
__global__ void ew_fill(float* a, float v, size_t n) { size_t i = gidx(); if (i < n) a[i] = v; }
__global__ void ew_clamp_min(float* a, float v, size_t n) { size_t i = gidx(); if (i < n) a[i] = fmaxf(a[i], v); }
__global__ void ew_reciprocal(float* a, size_t n) { size_t i = gidx(); if (i < n) a[i] = 1.0f / a[i]; }
__global__ void red_sq(const float* a, size_t n, double* out) {
  __shared__ double sh[256];
  double acc = 0;
  for (size_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) acc += double(a[i]) * a[i];
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}
__global__ void red_abs(const float* a, size_t n, double* out) {
  __shared__ double sh[256];
  double acc = 0;
  for (size_t i = blockIdx.x * 256 + threadIdx.x; i < n; i += (size_t)gridDim.x * 256) acc += fabs(double(a[i]));
  sh[threadIdx.x] = acc;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (threadIdx.x < s) sh[threadIdx.x] += sh[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[blockIdx.x] = sh[0];
}

// FDK pre-processing passes of conebeam_projection.cu:1483-1521, one kernel
// per Gadgetron array operation.
__global__ void ew_mul_bcast(float* a, const float* w, size_t n, size_t m) {   // a *= w (broadcast)
  size_t i = gidx();
  if (i < n) a[i] *= w[i % m];
}
__global__ void ew_cmul_bcast(float2* a, const float* f, size_t n, size_t m) {  // complex *= real filter
  size_t i = gidx();
  if (i < n) {
    const float w = f[i % m];
    a[i].x *= w;
    a[i].y *= w;
  }
}
__global__ void pad_rows(const float* in, float* out, int W, size_t n_out) {    // centred pad to 2W
  size_t i = gidx();
  if (i >= n_out) return;
  const size_t r = i / (2 * W);
  const int x = int(i % (2 * W)) - W / 2;
  out[i] = (x >= 0 && x < W) ? in[r * W + x] : 0.0f;
}
__global__ void crop_rows(const float* in, float* out, int W, size_t n_out) {   // crop at W/2 (:1510)
  size_t i = gidx();
  if (i >= n_out) return;
  const size_t r = i / W;
  out[i] = in[r * 2 * W + (i % W) + W / 2];
}

template <class K, class... A>
void launch_ew(K k, size_t n, A... a) {
  dim3 b, g;
  setup_grid(n, &b, &g);
  k<<<g, b>>>(a...);
  check(cudaGetLastError(), "plain element-wise kernel");
}

// Host-synchronised reduction (the value comes back to the host, as cuBLAS nrm2/asum do).
double reduce_host(bool squares, const float* a, size_t n) {
  const int blocks = 592;
  double* d = nullptr;
  check(cudaMalloc(&d, blocks * sizeof(double)), "cudaMalloc");
  if (squares) red_sq<<<blocks, 256>>>(a, n, d);
  else red_abs<<<blocks, 256>>>(a, n, d);
  std::vector<double> h(blocks);
  check(cudaMemcpy(h.data(), d, blocks * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
  cudaFree(d);
  double s = 0;
  for (double v : h) s += v;
  return s;
}

struct Uploads {
  float* angles = nullptr;
  float2* offsets = nullptr;
  Uploads(const float* a, const float* o, int n) {
    check(cudaMalloc(&angles, sizeof(float) * n), "cudaMalloc");
    check(cudaMalloc(&offsets, sizeof(float2) * n), "cudaMalloc");
    check(cudaMemcpy(angles, a, sizeof(float) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
    check(cudaMemcpy(offsets, o, sizeof(float2) * n, cudaMemcpyHostToDevice), "cudaMemcpy");
  }
  ~Uploads() {
    cudaFree(angles);
    cudaFree(offsets);
  }
};

void forward(const cbct_geometry& g, const float* angles, const float* offsets, int P, const float* vol,
             float* proj, bool accumulate) {
  if (P == 0) return;
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  cudaExtent ext = make_cudaExtent(g.nx, g.ny, g.nz);
  cudaArray_t arr = nullptr;
  check(cudaMalloc3DArray(&arr, &ch, ext), "cudaMalloc3DArray");
  cudaMemcpy3DParms cp = {};
  cp.srcPtr = make_cudaPitchedPtr((void*)vol, g.nx * sizeof(float), g.nx, g.ny);
  cp.dstArray = arr;
  cp.extent = ext;
  cp.kind = cudaMemcpyDeviceToDevice;
  check(cudaMemcpy3D(&cp), "cudaMemcpy3D");
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  cudaTextureObject_t tex = 0;
  check(cudaCreateTextureObject(&tex, &rd, &td, nullptr), "cudaCreateTextureObject");
  {
    Uploads up(angles, offsets, P);
    dim3 b, gr;
    setup_grid((size_t)g.width * g.height * P, &b, &gr);
    const int N = (int)(g.samples_per_pixel * float(g.nx));
    fwd_kernel<<<gr, b>>>(proj, up.angles, up.offsets, make_float3(g.lx, g.ly, g.lz), g.width, g.height,
                          make_float2(g.fov_u, g.fov_v), P, g.SDD, g.SAD, N, accumulate, tex);
    check(cudaGetLastError(), "plain fwd_kernel");
    check(cudaDeviceSynchronize(), "plain fwd_kernel");
  }
  cudaDestroyTextureObject(tex);
  cudaFreeArray(arr);
}

void backproject(const cbct_geometry& g, const float* angles, const float* offsets, int P, const float* proj,
                 float* vol, bool offset_correction, bool accumulate) {
  if (P == 0) return;
  Uploads up(angles, offsets, P);
  const size_t np = (size_t)g.width * g.height * P;
  const float* src = proj;
  float* copy = nullptr;
  if (offset_correction) {
    check(cudaMalloc(&copy, np * sizeof(float)), "cudaMalloc");
    check(cudaMemcpy(copy, proj, np * sizeof(float), cudaMemcpyDeviceToDevice), "cudaMemcpy");
    launch_ew(offset_kernel, np, copy, (const float2*)up.offsets, g.width, g.height, P,
              make_float2(g.fov_u, g.fov_v));
    src = copy;
  }
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  cudaExtent ext = make_cudaExtent(g.width, g.height, P);
  cudaArray_t arr = nullptr;
  check(cudaMalloc3DArray(&arr, &ch, ext, cudaArrayLayered), "cudaMalloc3DArray(layered)");
  cudaMemcpy3DParms cp = {};
  cp.srcPtr = make_cudaPitchedPtr((void*)src, g.width * sizeof(float), g.width, g.height);
  cp.dstArray = arr;
  cp.extent = ext;
  cp.kind = cudaMemcpyDeviceToDevice;
  check(cudaMemcpy3D(&cp), "cudaMemcpy3D");
  cudaResourceDesc rd = {};
  rd.resType = cudaResourceTypeArray;
  rd.res.array.array = arr;
  cudaTextureDesc td = {};
  td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
  td.filterMode = cudaFilterModeLinear;
  td.readMode = cudaReadModeElementType;
  td.normalizedCoords = 1;
  cudaTextureObject_t tex = 0;
  check(cudaCreateTextureObject(&tex, &rd, &td, nullptr), "cudaCreateTextureObject");
  dim3 b, gr;
  setup_grid((size_t)g.nx * g.ny * g.nz, &b, &gr);
  bp_kernel<false><<<gr, b>>>(vol, up.angles, up.offsets, g.nx, g.ny, g.nz, make_float3(g.lx, g.ly, g.lz),
                       make_float2(g.fov_u, g.fov_v), P, g.SDD, g.SAD, accumulate, tex);
  check(cudaGetLastError(), "plain bp_kernel");
  check(cudaDeviceSynchronize(), "plain bp_kernel");
  cudaDestroyTextureObject(tex);
  cudaFreeArray(arr);
  if (copy) cudaFree(copy);
}

// Device-only timing of the two reference kernels on already-built textures:
// the cudaArray copies, uploads and texture objects are made once, outside the
// timed launches, so the times are the kernels' own (what the reference's
// structure costs in the kernels alone, apart from its per-call host work).
void kernel_times(const cbct_geometry& g, const float* angles, const float* offsets, int P, const float* vol,
                  const float* proj, float* proj_out, float* vol_out, int reps, float* ms) {
  Uploads up(angles, offsets, P);
  cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
  cudaArray_t varr = nullptr, parr = nullptr;
  cudaTextureObject_t vtex = 0, ptex = 0;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto release = [&] {
    if (vtex) cudaDestroyTextureObject(vtex);
    if (ptex) cudaDestroyTextureObject(ptex);
    if (varr) cudaFreeArray(varr);
    if (parr) cudaFreeArray(parr);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
  };
  try {
    cudaTextureDesc td = {};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 1;
    cudaExtent vext = make_cudaExtent(g.nx, g.ny, g.nz);
    check(cudaMalloc3DArray(&varr, &ch, vext), "cudaMalloc3DArray");
    cudaMemcpy3DParms cp = {};
    cp.srcPtr = make_cudaPitchedPtr((void*)vol, g.nx * sizeof(float), g.nx, g.ny);
    cp.dstArray = varr;
    cp.extent = vext;
    cp.kind = cudaMemcpyDeviceToDevice;
    check(cudaMemcpy3D(&cp), "cudaMemcpy3D");
    cudaResourceDesc rd = {};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = varr;
    check(cudaCreateTextureObject(&vtex, &rd, &td, nullptr), "cudaCreateTextureObject");
    cudaExtent pext = make_cudaExtent(g.width, g.height, P);
    check(cudaMalloc3DArray(&parr, &ch, pext, cudaArrayLayered), "cudaMalloc3DArray(layered)");
    cudaMemcpy3DParms cq = {};
    cq.srcPtr = make_cudaPitchedPtr((void*)proj, g.width * sizeof(float), g.width, g.height);
    cq.dstArray = parr;
    cq.extent = pext;
    cq.kind = cudaMemcpyDeviceToDevice;
    check(cudaMemcpy3D(&cq), "cudaMemcpy3D");
    rd.res.array.array = parr;
    check(cudaCreateTextureObject(&ptex, &rd, &td, nullptr), "cudaCreateTextureObject");
    check(cudaEventCreate(&e0), "cudaEventCreate");
    check(cudaEventCreate(&e1), "cudaEventCreate");
    dim3 fb, fg, bb, bg;
    setup_grid((size_t)g.width * g.height * P, &fb, &fg);
    setup_grid((size_t)g.nx * g.ny * g.nz, &bb, &bg);
    const int N = (int)(g.samples_per_pixel * float(g.nx));
    const float3 L = make_float3(g.lx, g.ly, g.lz);
    const float2 ps = make_float2(g.fov_u, g.fov_v);
    auto fwd = [&] {
      fwd_kernel<<<fg, fb>>>(proj_out, up.angles, up.offsets, L, g.width, g.height, ps, P, g.SDD, g.SAD, N, false, vtex);
    };
    auto bp = [&] {
      bp_kernel<false><<<bg, bb>>>(vol_out, up.angles, up.offsets, g.nx, g.ny, g.nz, L, ps, P, g.SDD, g.SAD, false,
                                   ptex);
    };
    for (int which = 0; which < 2; ++which) {
      if (which == 0) fwd(); else bp();                  // warm-up launch
      check(cudaGetLastError(), "plain kernel");
      check(cudaDeviceSynchronize(), "plain kernel");
      check(cudaEventRecord(e0, 0), "cudaEventRecord");
      for (int r = 0; r < reps; ++r) {
        if (which == 0) fwd(); else bp();
      }
      check(cudaEventRecord(e1, 0), "cudaEventRecord");
      check(cudaEventSynchronize(e1), "cudaEventSynchronize");
      float t = 0.f;
      check(cudaEventElapsedTime(&t, e0, e1), "cudaEventElapsedTime");
      ms[which] = t / float(reps);
    }
  } catch (...) {
    release();
    throw;
  }
  release();
}

void osmom(const cbct_geometry& g, const float* angles, const float* offsets, int P, const int* sizes, int S,
           const int* offcorr, const float* b, float* z_out, int iters, bool nonneg, double* resid) {
  const size_t nv = (size_t)g.nx * g.ny * g.nz, plane = (size_t)g.width * g.height, np = plane * P;
  std::vector<int> first(S, 0);
  for (int s = 1; s < S; ++s) first[s] = first[s - 1] + sizes[s - 1];
  auto M = [&](int s, const float* x, float* out) {
    forward(g, angles + first[s], offsets + 2 * first[s], sizes[s], x, out, false);
  };
  auto MH = [&](int s, const float* in, float* x, bool acc) {
    backproject(g, angles + first[s], offsets + 2 * first[s], sizes[s], in, x, offcorr[s] != 0, acc);
  };
  float *z = nullptr, *x = nullptr, *xold = nullptr, *precon = nullptr, *tmp_proj = nullptr;
  check(cudaMalloc(&z, nv * 4), "cudaMalloc");
  check(cudaMalloc(&x, nv * 4), "cudaMalloc");
  check(cudaMalloc(&xold, nv * 4), "cudaMalloc");
  check(cudaMalloc(&precon, nv * 4), "cudaMalloc");
  check(cudaMalloc(&tmp_proj, np * 4), "cudaMalloc");
  check(cudaMemset(z, 0, nv * 4), "cudaMemset");                               // clear(z) (:100-104)
  check(cudaMemcpy(x, z, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");       // x = z
  check(cudaMemcpy(xold, z, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");    // xold = z
  // precon: fill(1), mult_M (all subsets), mult_MH (all subsets), clamp_min, reciprocal (:115-120)
  launch_ew(ew_fill, nv, precon, 1.0f, nv);
  for (int s = 0; s < S; ++s) M(s, precon, tmp_proj + plane * first[s]);
  for (int s = 0; s < S; ++s) MH(s, tmp_proj + plane * first[s], precon, s > 0);
  launch_ew(ew_clamp_min, nv, precon, 1e-6f, nv);
  launch_ew(ew_reciprocal, nv, precon, nv);
  float t = 1, told = 1;
  int step = 0;
  for (int it = 0; it < iters; ++it) {
    for (int s = 0; s < S; ++s, ++step) {
      t = 0.5f * (1 + std::sqrt(1 + 4 * t * t));
      float* ts = tmp_proj + plane * first[s];
      const size_t ns = plane * sizes[s];
      M(s, x, ts);
      launch_ew(ew_sub, ns, ts, b + plane * first[s], ns);                     // -= subsets[s]
      const double n2 = reduce_host(true, ts, ns);                             // VERBOSE nrm2 (:147-149)
      if (resid) resid[step] = n2;
      float* tmp_image = nullptr;                                              // ARRAY_TYPE tmp_image (:153)
      check(cudaMalloc(&tmp_image, nv * 4), "cudaMalloc");
      MH(s, ts, tmp_image, false);
      launch_ew(ew_mul, nv, tmp_image, (const float*)precon, nv);
      launch_ew(ew_axpy, nv, -1.0f * S, (const float*)tmp_image, z, nv);
      cudaFree(tmp_image);
      // denoise (:205-213): asum(precon) on the host path, a fresh g, then x = z
      (void)reduce_host(false, precon, nv);
      float* gbuf = nullptr;
      check(cudaMalloc(&gbuf, nv * 4), "cudaMalloc");
      cudaFree(gbuf);
      check(cudaMemcpy(x, z, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");
      if (nonneg) launch_ew(ew_clamp_min, nv, x, 0.0f, nv);
      check(cudaMemcpy(z, x, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");  // *z = *x
      launch_ew(ew_scale, nv, z, 1 + (told - 1) / t, nv);
      launch_ew(ew_axpy, nv, -(told - 1) / t, (const float*)xold, z, nv);
      std::swap(x, xold);
      check(cudaMemcpy(x, z, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");  // *x = *z
      told = t;
    }
  }
  check(cudaMemcpy(z_out, z, nv * 4, cudaMemcpyDeviceToDevice), "cudaMemcpy");
  check(cudaDeviceSynchronize(), "plain osmom");
  cudaFree(z);
  cudaFree(x);
  cudaFree(xold);
  cudaFree(precon);
  cudaFree(tmp_proj);
}

// cuFFT, as the reference's cb_fft/cb_ifft call it (conebeam_projection.cu:87-139).
// Only this baseline uses it; it is opened on first use so that the library
// itself has no link-time dependency on cuFFT.
struct Cufft {
  decltype(&cufftPlanMany) plan_many = nullptr;
  decltype(&cufftExecR2C) exec_r2c = nullptr;
  decltype(&cufftExecC2R) exec_c2r = nullptr;
  decltype(&cufftDestroy) destroy = nullptr;
};

const Cufft& cufft() {
  static Cufft api;
  static std::once_flag once;
  static std::string err;
  std::call_once(once, [] {
    void* h = dlopen("libcufft.so.11", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libcufft.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) {
      err = "plain FDK path: cannot open libcufft";
      return;
    }
    api.plan_many = reinterpret_cast<decltype(api.plan_many)>(dlsym(h, "cufftPlanMany"));
    api.exec_r2c = reinterpret_cast<decltype(api.exec_r2c)>(dlsym(h, "cufftExecR2C"));
    api.exec_c2r = reinterpret_cast<decltype(api.exec_c2r)>(dlsym(h, "cufftExecC2R"));
    api.destroy = reinterpret_cast<decltype(api.destroy)>(dlsym(h, "cufftDestroy"));
    if (!api.plan_many || !api.exec_r2c || !api.exec_c2r || !api.destroy) err = "plain FDK path: cuFFT symbols missing";
  });
  if (!err.empty()) throw Error(CBCT_ERR_UNSUPPORTED, err);
  return api;
}

void cufft_check(cufftResult r, const char* what) {
  if (r != CUFFT_SUCCESS) throw Error(CBCT_ERR_CUDA, std::string(what) + " failed (cufftResult " + std::to_string(int(r)) + ")");
}

// hoCuConebeamProjectionOperator::mult_MH with FBP (hoCuConebeamProjectionOperator.cpp:235-254)
// over conebeam_backwards_projection<true> (conebeam_projection.cu:1300-1649):
// cosine weights computed on the host per operator (.cpp:64-102), batches of
// views uploaded from host memory on two alternating streams, per batch the
// cosine multiply, centred pad to 2W, cuFFT R2C (plan made and destroyed per
// call), filter multiply, C2R, /2W, crop, offset weight, a layered cudaArray
// copy and the 1/U^2-weighted texture back-projection; the volume comes back
// to the host and is scaled by 2/P there.
void fdk(const cbct_geometry& g, const float* angles, const float* offsets, int P, const float* proj_host,
         float* vol_host, const float* filter, bool offset_correction, int per_batch) {
  const Cufft& F = cufft();
  const int W = g.width, H = g.height;
  const size_t plane = (size_t)W * H, nv = (size_t)g.nx * g.ny * g.nz;
  std::vector<float> cw(plane), filt(W + 1);
  const double SAD = g.SAD, SDD = g.SDD;
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) {
      const double xx = (double(x) / W - 0.5) * g.fov_u, yy = (double(y) / H - 0.5) * g.fov_v;
      const double s = SAD * xx / SDD, v = SAD * yy / SDD;
      cw[(size_t)y * W + x] = float(SAD / std::sqrt(SAD * SAD + s * s + v * v));
    }
  if (filter) std::copy(filter, filter + W + 1, filt.begin());
  else default_filter(W, filt.data());
  float *d_cw = nullptr, *d_filter = nullptr, *image = nullptr, *buf = nullptr, *buf2 = nullptr;
  check(cudaMalloc(&d_cw, plane * 4), "cudaMalloc");
  check(cudaMemcpy(d_cw, cw.data(), plane * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
  check(cudaMalloc(&d_filter, (W + 1) * 4), "cudaMalloc");
  check(cudaMemcpy(d_filter, filt.data(), (W + 1) * 4, cudaMemcpyHostToDevice), "cudaMemcpy");
  check(cudaMalloc(&image, nv * 4), "cudaMalloc");
  const int B = std::max(1, std::min(per_batch, P));
  const int nb = (P + B - 1) / B;
  check(cudaMalloc(&buf, plane * B * 4), "cudaMalloc");
  check(cudaMalloc(&buf2, plane * B * 4), "cudaMalloc");
  cudaStream_t main_st, indy_st;
  check(cudaStreamCreate(&main_st), "cudaStreamCreate");
  check(cudaStreamCreate(&indy_st), "cudaStreamCreate");
  {
    Uploads up(angles, offsets, P);
    check(cudaMemcpyAsync(buf, proj_host, plane * B * 4, cudaMemcpyHostToDevice, main_st), "cudaMemcpyAsync");
    for (int batch = 0; batch < nb; ++batch) {
      const int from = batch * B, n = std::min(P, from + B) - from;
      const size_t nproj = plane * n, npad = 2 * plane * n, nspec = (size_t)(W + 1) * H * n;
      launch_ew(ew_mul_bcast, nproj, buf, (const float*)d_cw, nproj, plane);
      float* padded = nullptr;
      float2* spec = nullptr;
      check(cudaMalloc(&padded, npad * 4), "cudaMalloc");
      launch_ew(pad_rows, npad, (const float*)buf, padded, W, npad);
      check(cudaMalloc(&spec, nspec * 8), "cudaMalloc");
      int len = 2 * W;
      cufftHandle pl;
      cufft_check(F.plan_many(&pl, 1, &len, nullptr, 1, 2 * W, nullptr, 1, W + 1, CUFFT_R2C, H * n), "cufftPlanMany");
      cufft_check(F.exec_r2c(pl, padded, reinterpret_cast<cufftComplex*>(spec)), "cufftExecR2C");
      cufft_check(F.destroy(pl), "cufftDestroy");
      launch_ew(ew_cmul_bcast, nspec, spec, (const float*)d_filter, nspec, (size_t)(W + 1));
      cufft_check(F.plan_many(&pl, 1, &len, nullptr, 1, W + 1, nullptr, 1, 2 * W, CUFFT_C2R, H * n), "cufftPlanMany");
      cufft_check(F.exec_c2r(pl, reinterpret_cast<cufftComplex*>(spec), padded), "cufftExecC2R");
      cufft_check(F.destroy(pl), "cufftDestroy");
      launch_ew(ew_scale, npad, padded, 1.0f / float(2 * W), npad);
      launch_ew(crop_rows, nproj, (const float*)padded, buf, W, nproj);
      cudaFree(spec);
      cudaFree(padded);
      if (offset_correction)
        launch_ew(offset_kernel, nproj, buf, (const float2*)up.offsets + from, W, H, n, make_float2(g.fov_u, g.fov_v));
      cudaChannelFormatDesc ch = cudaCreateChannelDesc<float>();
      cudaExtent ext = make_cudaExtent(W, H, n);
      cudaArray_t arr = nullptr;
      check(cudaMalloc3DArray(&arr, &ch, ext, cudaArrayLayered), "cudaMalloc3DArray(layered)");
      cudaMemcpy3DParms cp = {};
      cp.srcPtr = make_cudaPitchedPtr((void*)buf, W * sizeof(float), W, H);
      cp.dstArray = arr;
      cp.extent = ext;
      cp.kind = cudaMemcpyDeviceToDevice;
      check(cudaMemcpy3DAsync(&cp, main_st), "cudaMemcpy3DAsync");
      cudaResourceDesc rd = {};
      rd.resType = cudaResourceTypeArray;
      rd.res.array.array = arr;
      cudaTextureDesc td = {};
      td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeBorder;
      td.filterMode = cudaFilterModeLinear;
      td.readMode = cudaReadModeElementType;
      td.normalizedCoords = 1;
      cudaTextureObject_t tex = 0;
      check(cudaCreateTextureObject(&tex, &rd, &td, nullptr), "cudaCreateTextureObject");
      if (batch + 1 < nb) {
        const int nf = std::min(P, from + 2 * B) - (from + B);
        check(cudaMemcpyAsync(buf2, proj_host + plane * (from + B), plane * nf * 4, cudaMemcpyHostToDevice, indy_st),
              "cudaMemcpyAsync");
      }
      dim3 b, gr;
      setup_grid(nv, &b, &gr);
      bp_kernel<true><<<gr, b, 0, main_st>>>(image, up.angles + from, up.offsets + from, g.nx, g.ny, g.nz,
                                             make_float3(g.lx, g.ly, g.lz), make_float2(g.fov_u, g.fov_v), n,
                                             g.SDD, g.SAD, batch > 0, tex);
      check(cudaGetLastError(), "plain bp_kernel<FBP>");
      cudaDestroyTextureObject(tex);
      cudaFreeArray(arr);
      std::swap(buf, buf2);
      std::swap(main_st, indy_st);
    }
    check(cudaMemcpy(vol_host, image, nv * 4, cudaMemcpyDeviceToHost), "cudaMemcpy");
  }
  const float sc = 2.0f / float(P);  // image_3d *= 2/P on the host array (.cpp:253)
  for (size_t i = 0; i < nv; ++i) vol_host[i] *= sc;
  cudaFree(buf);
  cudaFree(buf2);
  cudaFree(image);
  cudaFree(d_cw);
  cudaFree(d_filter);
  cudaStreamDestroy(main_st);
  cudaStreamDestroy(indy_st);
}

}  // namespace plain
}  // namespace cbct

using namespace cbct::plain;
using cbct::guard;

extern "C" {

cbct_status cbct_plain_forward(const cbct_geometry* g, const float* angles, const float* offsets, int32_t n,
                               const float* vol, float* proj, int32_t accumulate) {
  return guard([&] {
    if (!g || !angles || !offsets || !vol || !proj || n < 0) throw cbct::Error(CBCT_ERR_INVALID_ARGUMENT, "bad args");
    forward(*g, angles, offsets, n, vol, proj, accumulate != 0);
  });
}

cbct_status cbct_plain_backproject(const cbct_geometry* g, const float* angles, const float* offsets, int32_t n,
                                   const float* proj, float* vol, int32_t offset_correction, int32_t accumulate) {
  return guard([&] {
    if (!g || !angles || !offsets || !vol || !proj || n < 0) throw cbct::Error(CBCT_ERR_INVALID_ARGUMENT, "bad args");
    backproject(*g, angles, offsets, n, proj, vol, offset_correction != 0, accumulate != 0);
  });
}

cbct_status cbct_plain_osmom_solve(const cbct_geometry* g, const float* angles, const float* offsets, int32_t n,
                                   const int32_t* sizes, int32_t S, const int32_t* offcorr, const float* b,
                                   float* z_out, int32_t iterations, int32_t nonneg, double* resid) {
  return guard([&] {
    if (!g || !angles || !offsets || !sizes || !offcorr || !b || !z_out || S < 1)
      throw cbct::Error(CBCT_ERR_INVALID_ARGUMENT, "bad args");
    osmom(*g, angles, offsets, n, sizes, S, offcorr, b, z_out, iterations, nonneg != 0, resid);
  });
}

cbct_status cbct_plain_kernel_times(const cbct_geometry* g, const float* angles, const float* offsets, int32_t n,
                                    const float* vol, const float* proj, float* proj_out, float* vol_out, int32_t reps,
                                    float* ms_out) {
  return guard([&] {
    if (!g || !angles || !offsets || !vol || !proj || !proj_out || !vol_out || !ms_out || n < 1 || reps < 1)
      throw cbct::Error(CBCT_ERR_INVALID_ARGUMENT, "bad args");
    kernel_times(*g, angles, offsets, n, vol, proj, proj_out, vol_out, reps, ms_out);
  });
}

cbct_status cbct_plain_fdk(const cbct_geometry* g, const float* angles, const float* offsets, int32_t n,
                           const float* proj_host, float* vol_host, const float* filter, int32_t offset_correction,
                           int32_t views_per_batch) {
  return guard([&] {
    if (!g || !angles || !offsets || !proj_host || !vol_host || n < 1 || views_per_batch < 1)
      throw cbct::Error(CBCT_ERR_INVALID_ARGUMENT, "bad args");
    fdk(*g, angles, offsets, n, proj_host, vol_host, filter, offset_correction != 0, views_per_batch);
  });
}

}  // extern "C"
