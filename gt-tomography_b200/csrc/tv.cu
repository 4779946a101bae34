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

__device__ __forceinline__ void voxel_of(size_t idx, int nx, int ny, int& i, int& j, int& k) {
  i = int(idx % nx);
  j = int((idx / nx) % ny);
  k = int(idx / ((size_t)nx * ny));
}

// P_a = d_a / max(1, |d|), d_a = (x[c + e_a] - x[c]) * scale, neighbours
// periodic, scale = (w sigma) / (1 + sigma alpha).
__global__ void tv_primal_kernel(const float* __restrict__ x, float* __restrict__ P, int nx, int ny, int nz,
                                 float scale) {
  const size_t n = (size_t)nx * ny * nz;
  const size_t sxy = (size_t)nx * ny;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    voxel_of(idx, nx, ny, i, j, k);
    const float v = x[idx];
    const int ip = i + 1 == nx ? 0 : i + 1, jp = j + 1 == ny ? 0 : j + 1, kp = k + 1 == nz ? 0 : k + 1;
    const float d0 = (x[(size_t)k * sxy + (size_t)j * nx + ip] - v) * scale;
    const float d1 = (x[(size_t)k * sxy + (size_t)jp * nx + i] - v) * scale;
    const float d2 = (x[(size_t)kp * sxy + (size_t)j * nx + i] - v) * scale;
    const float m = fmaxf(1.f, sqrtf(d0 * d0 + d1 * d1 + d2 * d2));
    P[idx] = d0 / m;
    P[n + idx] = d1 / m;
    P[2 * n + idx] = d2 / m;
  }
}

// g = w * sum_a (P_a[c - e_a] - P_a[c]) (periodic), then updateG:
// x = ((x - tau g) + (tau / lambda) (s / D)) / ((1 / D) (tau / lambda) + 1).
__global__ void tv_update_kernel(const float* __restrict__ P, float* __restrict__ x, const float* __restrict__ s,
                                 const float* __restrict__ D, int nx, int ny, int nz, float w, float tau,
                                 float tau_lambda) {
  const size_t n = (size_t)nx * ny * nz;
  const size_t sxy = (size_t)nx * ny;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n; idx += (size_t)gridDim.x * blockDim.x) {
    int i, j, k;
    voxel_of(idx, nx, ny, i, j, k);
    const int im = i == 0 ? nx - 1 : i - 1, jm = j == 0 ? ny - 1 : j - 1, km = k == 0 ? nz - 1 : k - 1;
    const size_t row = (size_t)k * sxy + (size_t)j * nx;
    float r = 0.f;
    r += P[row + im] - P[idx];
    r += P[n + (size_t)k * sxy + (size_t)jm * nx + i] - P[n + idx];
    r += P[2 * n + (size_t)km * sxy + (size_t)j * nx + i] - P[2 * n + idx];
    const float g = r * w;
    const float d = D[idx];
    const float num = (x[idx] - tau * g) + tau_lambda * (s[idx] / d);
    x[idx] = num / ((1.f / d) * tau_lambda + 1.f);
  }
}

int tv_blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

void tv_primal_launch(const float* x, float* P, int nx, int ny, int nz, float scale, cudaStream_t st) {
  const size_t n = (size_t)nx * ny * nz;
  if (n == 0) return;
  tv_primal_kernel<<<tv_blocks(n), 256, 0, st>>>(x, P, nx, ny, nz, scale);
  check_launch("tv_primal_kernel");
}

void tv_update_launch(const float* P, float* x, const float* s, const float* D, int nx, int ny, int nz, float w,
                      float tau, float tau_lambda, cudaStream_t st) {
  const size_t n = (size_t)nx * ny * nz;
  if (n == 0) return;
  tv_update_kernel<<<tv_blocks(n), 256, 0, st>>>(P, x, s, D, nx, ny, nz, w, tau, tau_lambda);
  check_launch("tv_update_kernel");
}

}  // namespace cbct
