// tv.cu -- the total-variation regulariser of the OS-MOM solver.
//
// The reference regularises osMOMSolverD by a few primal-dual steps per subset
// step (denoise, solvers/osMOMSolverD.h:205-231): the regulariser's
// primalDual (cuTVPrimalDualOperator, operators/cuTVPrimalDualOperator.cu:9-96:
// forward differences with periodic neighbours, scaled and projected onto the
// unit ball, then their negative divergence) followed by the resolvent of the
// preconditioned data term (updateG of osMOMSolverD.h:233-247, the version
// osMOMSolverD<cuNDArray<float>> runs in cuCBOS_reconstruct; the thrust functor
// of solvers/cuOSMOMSolverD.cu:8-27 divides by D tau/lambda + 1 instead of
// (tau/lambda)/D + 1 and belongs to a subclass the drivers do not use).  Here
// the primal kernel writes the projected gradient field and one fused kernel
// takes its divergence and applies updateG, so a primal-dual step reads the
// image twice and writes it once.
#include "cbct_internal.h"

namespace cbct {
namespace {

// Threads run along x; grid-y walks the (j, k) rows, so no voxel index is
// divided out of a linear index.
constexpr int kTvThreads = 256;

// P_a = d_a / max(1, |d|), d_a = (x[c + e_a] - x[c]) * scale, neighbours
// periodic, scale = (w sigma) / (1 + sigma alpha).
__global__ void __launch_bounds__(kTvThreads) tv_primal_kernel(const float* __restrict__ x, float* __restrict__ P,
                                                               int nx, int ny, int nz, float scale) {
  const size_t n = (size_t)nx * ny * nz, sxy = (size_t)nx * ny;
  for (int row = blockIdx.y; row < ny * nz; row += gridDim.y) {
    const int j = row % ny, k = row / ny;
    const int jp = j + 1 == ny ? 0 : j + 1, kp = k + 1 == nz ? 0 : k + 1;
    const size_t r0 = (size_t)k * sxy + (size_t)j * nx;
    const size_t ry = (size_t)k * sxy + (size_t)jp * nx, rz = (size_t)kp * sxy + (size_t)j * nx;
    for (int i = blockIdx.x * kTvThreads + threadIdx.x; i < nx; i += gridDim.x * kTvThreads) {
      const int ip = i + 1 == nx ? 0 : i + 1;
      const float v = x[r0 + i];
      const float d0 = (x[r0 + ip] - v) * scale;
      const float d1 = (x[ry + i] - v) * scale;
      const float d2 = (x[rz + i] - v) * scale;
      // d / max(1, |d|): only gradients longer than 1 are scaled
      const float n2 = d0 * d0 + d1 * d1 + d2 * d2;
      const float inv = n2 > 1.f ? 1.f / sqrtf(n2) : 1.f;
      P[r0 + i] = d0 * inv;
      P[n + r0 + i] = d1 * inv;
      P[2 * n + r0 + i] = d2 * inv;
    }
  }
}

// g = w * sum_a (P_a[c - e_a] - P_a[c]) (periodic), then updateG:
// x = ((x - tau g) + (tau / lambda) (s / D)) / ((1 / D) (tau / lambda) + 1).
__global__ void __launch_bounds__(kTvThreads) tv_update_kernel(const float* __restrict__ P, float* __restrict__ x,
                                                               const float* __restrict__ s,
                                                               const float* __restrict__ D, int nx, int ny, int nz,
                                                               float w, float tau, float tau_lambda) {
  const size_t n = (size_t)nx * ny * nz, sxy = (size_t)nx * ny;
  for (int row = blockIdx.y; row < ny * nz; row += gridDim.y) {
    const int j = row % ny, k = row / ny;
    const int jm = j == 0 ? ny - 1 : j - 1, km = k == 0 ? nz - 1 : k - 1;
    const size_t r0 = (size_t)k * sxy + (size_t)j * nx;
    const size_t ry = (size_t)k * sxy + (size_t)jm * nx, rz = (size_t)km * sxy + (size_t)j * nx;
    for (int i = blockIdx.x * kTvThreads + threadIdx.x; i < nx; i += gridDim.x * kTvThreads) {
      const int im = i == 0 ? nx - 1 : i - 1;
      const size_t c = r0 + i;
      float r = 0.f;
      r += P[r0 + im] - P[c];
      r += P[n + ry + i] - P[n + c];
      r += P[2 * n + rz + i] - P[2 * n + c];
      // ((x - tau g) + tl s / D) / (tl / D + 1) = ((x - tau g) D + tl s) / (tl + D)
      const float g = r * w;
      const float d = D[c];
      x[c] = fmaf(x[c] - tau * g, d, tau_lambda * s[c]) / (tau_lambda + d);
    }
  }
}

dim3 tv_grid(int nx, int ny, int nz) {
  const int gx = (nx + kTvThreads - 1) / kTvThreads;
  return dim3(gx, (unsigned)std::min(ny * nz, 65535));
}

}  // namespace

void tv_primal_launch(const float* x, float* P, int nx, int ny, int nz, float scale, cudaStream_t st) {
  const size_t n = (size_t)nx * ny * nz;
  if (n == 0) return;
  tv_primal_kernel<<<tv_grid(nx, ny, nz), kTvThreads, 0, st>>>(x, P, nx, ny, nz, scale);
  check_launch("tv_primal_kernel");
}

void tv_update_launch(const float* P, float* x, const float* s, const float* D, int nx, int ny, int nz, float w,
                      float tau, float tau_lambda, cudaStream_t st) {
  const size_t n = (size_t)nx * ny * nz;
  if (n == 0) return;
  tv_update_kernel<<<tv_grid(nx, ny, nz), kTvThreads, 0, st>>>(P, x, s, D, nx, ny, nz, w, tau, tau_lambda);
  check_launch("tv_update_kernel");
}

}  // namespace cbct
