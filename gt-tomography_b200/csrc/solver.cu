// solver.cu -- FP64 reductions, the fused OS-MOM update, and the
// device-resident osMOMSolverD / osSARTSolver / FDK drivers.
//
// osMOMSolverD<ARRAY>::solve (solvers/osMOMSolverD.h:82-196), no regularisers:
//   D = 1/max(A^T A 1, 1e-6)                                       (:115-120)
//   per iteration i, subset s:  t = (1+sqrt(1+4t^2))/2              (:142)
//     r = A_s x - b_s                                                (:144-145)
//     z -= beta/(1+gamma i) * S * D .* A_s^T r                       (:155-157)
//     x = z ; [x = max(x,0)] ; z = x (1+m) - m xold, m = (told-1)/t (:167-173)
//     xold = x ; x = z ; told = t                                    (:174-177)
//   returns z (:195).  x == z holds at the start of every subset step, so the
//   state is (z, xold).  Here the step is two kernels: the residual forward
//   projection (offset weight and the VERBOSE norm fused in) and the
//   back-projection with the update fused into its epilogue.
//
// osSARTSolver<ARRAY>::solve (solvers/osSARTSolver.h:33-126):
//   Wp = 1/max(A 1, 1e-6), V_s = 1/max(A_s^T 1, 1e-6)                (:59-81)
//   r = -(A_s x - b_s) .* Wp_s ; x += beta/(1+gamma i) V_s .* A_s^T r  (:91-101)
//   clamp, reverse the subset order each iteration, cost ||A x - b||^2 (:104-116).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "device_common.cuh"

namespace cbct {

void fill_launch(float* x, size_t n, float v, cudaStream_t st);
void convert_launch(const float* src, void* dst, size_t n, cbct_dtype dt, cudaStream_t st);
void backproject_recip_launch(cbct_plan* p, int s, const float* proj, float* out, cudaStream_t st);
void backproject_mom_launch(cbct_plan* p, int s, const float* proj, float* z, float* xold,
                            const float* precon, float step, float mom, int nonneg, cudaStream_t st);
void backproject_sart_launch(cbct_plan* p, int s, const float* proj, float* x, const float* V,
                             float step, int nonneg, cudaStream_t st);
void backproject_step_launch(cbct_plan* p, int s, const float* proj, const float* z, float* out,
                             const float* precon, float step, cudaStream_t st);

namespace {

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 148 * 4;

__global__ void __launch_bounds__(kRedThreads) reduce_kernel(int kind, const float* __restrict__ a,
                                                             const float* __restrict__ b, size_t n,
                                                             double* __restrict__ partials) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (size_t i = blockIdx.x * (size_t)kRedThreads + threadIdx.x; i < n; i += (size_t)gridDim.x * kRedThreads) {
    const double x = a[i];
    if (kind == 0) acc += x * double(b[i]);
    else if (kind == 1) acc += x * x;
    else acc += fabs(x);
  }
  const double s = block_sum<kRedThreads>(acc, sh);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// Sums n partials in a fixed order (deterministic) into out[0].
__global__ void __launch_bounds__(kRedThreads) finalize_kernel(const double* __restrict__ partials, int n,
                                                               double* __restrict__ out) {
  __shared__ double sh[kRedThreads / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kRedThreads) acc += partials[i];
  const double s = block_sum<kRedThreads>(acc, sh);
  if (threadIdx.x == 0) out[0] = s;
}

__global__ void osmom_update_kernel(float* __restrict__ z, float* __restrict__ xold,
                                    const float* __restrict__ precon, const float* __restrict__ g,
                                    size_t n, float step, float mom, int nonneg) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float zt = fmaf(-step, precon[i] * (g ? g[i] : 0.f), z[i]);  // g = NULL: no gradient
    const float xc = nonneg ? fmaxf(zt, 0.f) : zt;
    z[i] = fmaf(-mom, xold[i], xc * (1.f + mom));
    xold[i] = xc;
  }
}

// x = 1 / max(x, 1e-6): the preconditioner of osMOMSolverD.h:115-120 when
// its back-projection is accumulated over several launches.
__global__ void recip_kernel(float* __restrict__ x, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    x[i] = 1.f / fmaxf(x[i], 1e-6f);
}

__global__ void fill_kernel(float* __restrict__ x, size_t n, float v) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) x[i] = v;
}

template <class T>
__global__ void convert_kernel(const float* __restrict__ src, T* __restrict__ dst, size_t n);
template <>
__global__ void convert_kernel<__half>(const float* __restrict__ src, __half* __restrict__ dst, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __float2half_rn(src[i]);
}
template <>
__global__ void convert_kernel<__nv_bfloat16>(const float* __restrict__ src, __nv_bfloat16* __restrict__ dst,
                                              size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = __float2bfloat16_rn(src[i]);
}

int ew_blocks(size_t n) { return (int)std::min<size_t>((n + 255) / 256, 148 * 16); }

}  // namespace

void reduce_launch(int kind, const float* a, const float* b, size_t n, double* partials, size_t n_partials,
                   double* out, cudaStream_t st) {
  const int blocks = (int)std::min<size_t>(std::min<size_t>(kRedBlocks, n_partials),
                                           std::max<size_t>((n + kRedThreads - 1) / kRedThreads, 1));
  reduce_kernel<<<blocks, kRedThreads, 0, st>>>(kind, a, b, n, partials);
  check_launch("reduce_kernel");
  finalize_partials(partials, blocks, out, st);
}

void finalize_partials(const double* partials, int n, double* out, cudaStream_t st) {
  finalize_kernel<<<1, kRedThreads, 0, st>>>(partials, n, out);
  check_launch("finalize_kernel");
}

// ------------------------------------------------------------------ allocation-free reduction
// Scratch of cbct_reduce_f64_noalloc: the per-block partial sums of the
// reduction live in this file-scope device array instead of device memory
// obtained from cudaMalloc.  It holds kNoAllocMaxPartials doubles (8 KiB), and
// every GPU that loads the library keeps it until the process exits.  All calls
// share it: a call writes every partial it later reads, so contents left by an
// earlier call never reach a result, but two calls that overlap on the GPU
// (different streams, no ordering between them) race on it.
constexpr int kNoAllocMaxPartials = 1024;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocMaxPartials];
// The reduction's grid is capped at kRedBlocks (592) blocks, one partial each,
// so no input size needs more partials than the array holds; the size check
// in reduce_noalloc_launch is a guard for a future change of the launch shape.
static_assert(kRedBlocks <= kNoAllocMaxPartials, "the static scratch must hold one partial per reduction block");

// The array's name is only a host-side stand-in in host code; its device
// address is looked up once per device, with that device current, by the first
// call made on that device.  The cached address assumes the device's primary
// context lives as long as the library (no cudaDeviceReset in between, which
// would give the array a new address).
static double* noalloc_partials_address() {
  static std::mutex mu;
  static std::vector<double*> by_device;
  int dev = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  std::lock_guard<std::mutex> lock(mu);
  if ((int)by_device.size() <= dev) by_device.resize(dev + 1, nullptr);
  if (by_device[dev] == nullptr) {
    void* ptr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_partials);
    if (e != cudaSuccess)
      throw Error(CBCT_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_partials): ") + cudaGetErrorString(e));
    by_device[dev] = static_cast<double*>(ptr);
  }
  return by_device[dev];
}

void reduce_noalloc_launch(int kind, const float* a, const float* b, size_t n, double* out, cudaStream_t st) {
  // Same launch shape as reduce_launch: one partial per block.
  const size_t needed = std::min<size_t>(kRedBlocks, std::max<size_t>((n + kRedThreads - 1) / kRedThreads, 1));
  if (needed > (size_t)kNoAllocMaxPartials)
    throw Error(CBCT_ERR_INVALID_ARGUMENT, "cbct_reduce_f64_noalloc: the reduction needs " + std::to_string(needed) +
                                               " partial sums but its static scratch holds " +
                                               std::to_string(kNoAllocMaxPartials));
  reduce_launch(kind, a, b, n, noalloc_partials_address(), (size_t)kNoAllocMaxPartials, out, st);
}

void osmom_update_launch(float* z, float* xold, const float* precon, const float* g, size_t n, float step,
                         float mom, int nonneg, cudaStream_t st) {
  if (n == 0) return;
  osmom_update_kernel<<<ew_blocks(n), 256, 0, st>>>(z, xold, precon, g, n, step, mom, nonneg);
  check_launch("osmom_update_kernel");
}

static void recip_launch(float* x, size_t n, cudaStream_t st) {
  if (n == 0) return;
  recip_kernel<<<ew_blocks(n), 256, 0, st>>>(x, n);
  check_launch("recip_kernel");
}

void fill_launch(float* x, size_t n, float v, cudaStream_t st) {
  if (n == 0) return;
  fill_kernel<<<ew_blocks(n), 256, 0, st>>>(x, n, v);
  check_launch("fill_kernel");
}

void convert_launch(const float* src, void* dst, size_t n, cbct_dtype dt, cudaStream_t st) {
  if (n == 0) return;
  if (dt == CBCT_F16) convert_kernel<__half><<<ew_blocks(n), 256, 0, st>>>(src, (__half*)dst, n);
  else if (dt == CBCT_BF16) convert_kernel<__nv_bfloat16><<<ew_blocks(n), 256, 0, st>>>(src, (__nv_bfloat16*)dst, n);
  else throw Error(CBCT_ERR_INVALID_ARGUMENT, "convert: destination must be CBCT_F16 or CBCT_BF16");
  check_launch("convert_kernel");
}

// ------------------------------------------------------------------ workspace
static size_t vol_elems(const cbct_plan* p) { return (size_t)p->g.nx * p->g.ny * p->g.nz; }
static size_t proj_elems(const cbct_plan* p) { return (size_t)p->g.width * p->g.height * p->n_views; }
static size_t plane_elems(const cbct_plan* p) { return (size_t)p->g.width * p->g.height; }

// Workspace layout (floats):
//  OS-MOM : xold | D | r (all views) | 16-bit shadow of z (mixed precision)
//  OS-SART: Wp (all views) | r (all views) | V_0 .. V_{S-1}
static float* workspace(cbct_plan* p, size_t elems) {
  if (p->ws_elems < elems) {
    plan_dealloc(p, p->ws);
    p->ws = nullptr;
    p->ws_elems = 0;
    p->ws = plan_alloc_n<float>(p, elems);
    p->ws_elems = elems;
  }
  return p->ws;
}

float* solver_workspace(cbct_plan* p, size_t elems) { return workspace(p, elems); }

static void run_osmom(cbct_plan* p, const void* b, const float* x0, float* z, const cbct_solver_params& prm,
                      double* resid, float* xold, float* D, float* r, void* shadow, cudaStream_t st) {
  const cbct_dtype bt = prm.proj_storage;
  auto b_of = [&](int s) {
    return static_cast<const char*>(b) + plane_elems(p) * p->first[s] * dtype_size(bt);
  };
  const size_t nv = vol_elems(p);
  const int S = p->n_subsets;
  // Preconditioner: D = 1/max(A^T (W A 1), 1e-6) over every subset, the
  // offset weight W applied per subset as the reference's mult_MH does.
  fill_launch(xold, nv, 1.f, st);
  for (int s = 0; s < S; ++s)
    forward_launch_ex(p, s, CBCT_F32, xold, r + plane_elems(p) * p->first[s], nullptr, nullptr, 1.f, 1,
                      p->offcorr[s], 0, nullptr, st);
  backproject_recip_launch(p, p->n_subsets, r, D, st);
  // z = x0 or 0 ; xold = z
  if (x0) {
    CBCT_CUDA(cudaMemcpyAsync(z, x0, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CBCT_CUDA(cudaMemcpyAsync(xold, x0, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  } else {
    CBCT_CUDA(cudaMemsetAsync(z, 0, nv * sizeof(float), st));
    CBCT_CUDA(cudaMemsetAsync(xold, 0, nv * sizeof(float), st));
  }
  double t = 1.0, told = 1.0;
  int step = 0;
  for (int it = 0; it < prm.iterations; ++it) {
    const bool lowp = prm.storage != CBCT_F32 && shadow != nullptr &&
                      !(prm.refine_every > 0 && (it % prm.refine_every) == prm.refine_every - 1);
    for (int s = 0; s < S; ++s, ++step) {
      t = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * t * t));
      float* rs = r + plane_elems(p) * p->first[s];
      if (lowp) {
        convert_launch(z, shadow, nv, prm.storage, st);
        forward_launch_ex(p, s, prm.storage, shadow, rs, b_of(s), nullptr, 1.f, 1, p->offcorr[s], 0,
                          resid ? resid + step : nullptr, st, bt);
      } else {
        forward_launch_ex(p, s, CBCT_F32, z, rs, b_of(s), nullptr, 1.f, 1, p->offcorr[s], 0,
                          resid ? resid + step : nullptr, st, bt);
      }
      const double stepsz = double(prm.beta) / (1.0 + double(prm.gamma) * it) * S;
      const double mom = (told - 1.0) / t;
      backproject_mom_launch(p, s, rs, z, xold, D, float(stepsz), float(mom), prm.non_negativity, st);
      told = t;
    }
  }
}

// osMOMSolverD with bins (the subset operator of CBSubsetOperator over
// binned cuConebeamProjectionOperators, CBSubsetOperator.cpp:66-135 and
// cuConebeamProjectionOperator.cpp:49-116): z, xold and D hold n_bins volumes;
// a subset's segments project and back-project their own bin's volume, and
// the bins without views in the subset take the momentum step with a zero
// gradient (their mult_MH output is 0).
static void run_osmom_bins(cbct_plan* p, const float* b, const float* x0, float* z, const cbct_solver_params& prm,
                           float* xold, float* D, float* r, cudaStream_t st) {
  const size_t nv = vol_elems(p), pl = plane_elems(p);
  const int S = p->n_subsets, NB = p->n_bins;
  const size_t nall = nv * NB;
  // D = 1/max(A^T (W A 1), 1e-6) per bin; one ones-volume serves every bin.
  fill_launch(xold, nv, 1.f, st);
  for (int s = 0; s < S; ++s)
    for (int k = p->seg_begin[s]; k < p->seg_end[s]; ++k)
      forward_launch_ex(p, k, CBCT_F32, xold, r + pl * p->first[k], nullptr, nullptr, 1.f, 1, p->offcorr[k], 0,
                        nullptr, st);
  CBCT_CUDA(cudaMemsetAsync(D, 0, nall * sizeof(float), st));
  for (int s = 0; s < S; ++s)
    for (int k = p->seg_begin[s]; k < p->seg_end[s]; ++k)
      backproject_launch(p, k, r + pl * p->first[k], D + nv * p->seg_bin[k], 0, 1, 1.f, st);
  recip_launch(D, nall, st);
  if (x0) {
    CBCT_CUDA(cudaMemcpyAsync(z, x0, nall * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CBCT_CUDA(cudaMemcpyAsync(xold, x0, nall * sizeof(float), cudaMemcpyDeviceToDevice, st));
  } else {
    CBCT_CUDA(cudaMemsetAsync(z, 0, nall * sizeof(float), st));
    CBCT_CUDA(cudaMemsetAsync(xold, 0, nall * sizeof(float), st));
  }
  std::vector<int> seg_of_bin(NB);
  double t = 1.0, told = 1.0;
  for (int it = 0; it < prm.iterations; ++it) {
    for (int s = 0; s < S; ++s) {
      t = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * t * t));
      std::fill(seg_of_bin.begin(), seg_of_bin.end(), -1);
      for (int k = p->seg_begin[s]; k < p->seg_end[s]; ++k) {
        seg_of_bin[p->seg_bin[k]] = k;
        forward_launch_ex(p, k, CBCT_F32, z + nv * p->seg_bin[k], r + pl * p->first[k], b + pl * p->first[k], nullptr,
                          1.f, 1, p->offcorr[k], 0, nullptr, st);
      }
      const double stepsz = double(prm.beta) / (1.0 + double(prm.gamma) * it) * S;
      const double mom = (told - 1.0) / t;
      for (int bb = 0; bb < NB; ++bb) {
        const int k = seg_of_bin[bb];
        if (k >= 0)
          backproject_mom_launch(p, k, r + pl * p->first[k], z + nv * bb, xold + nv * bb, D + nv * bb, float(stepsz),
                                 float(mom), prm.non_negativity, st);
        else
          osmom_update_launch(z + nv * bb, xold + nv * bb, D + nv * bb, nullptr, nv, float(stepsz), float(mom),
                              prm.non_negativity, st);
      }
      told = t;
    }
  }
}

// osMOMSolverD with a total-variation regulariser (osMOMSolverD.h:82-196 with
// denoise, :205-247): after the gradient step s = z - step D A^T r, reg_steps
// primal-dual steps move the momentum point toward s under the TV prior
// (cuTVPrimalDualOperator with weight 1 after the solver's normalisation by
// avg_lambda = tv_weight; updateG with avg_lambda), then the clamp and the
// momentum step.  Works on one bin or several (each bin's TV is 3-D).
static void run_osmom_tv(cbct_plan* p, const float* b, const float* x0, float* z, const cbct_solver_params& prm,
                         float* xold, float* D, float* r, float* sbuf, float* P, double* asum_dev, cudaStream_t st) {
  const size_t nv = vol_elems(p), pl = plane_elems(p);
  const int S = p->n_subsets, NB = p->n_bins;
  const size_t nall = nv * NB;
  const int nx = p->g.nx, ny = p->g.ny, nz = p->g.nz;
  std::vector<std::vector<int>> segs(S);
  for (int s = 0; s < S; ++s) {
    if (NB == 1) segs[s].push_back(s);
    else
      for (int k = p->seg_begin[s]; k < p->seg_end[s]; ++k) segs[s].push_back(k);
  }
  auto bin_of = [&](int k) { return NB == 1 ? 0 : p->seg_bin[k]; };
  // D = 1/max(A^T (W A 1), 1e-6), per bin.
  fill_launch(xold, nv, 1.f, st);
  for (int s = 0; s < S; ++s)
    for (int k : segs[s])
      forward_launch_ex(p, k, CBCT_F32, xold, r + pl * p->first[k], nullptr, nullptr, 1.f, 1, p->offcorr[k], 0,
                        nullptr, st);
  CBCT_CUDA(cudaMemsetAsync(D, 0, nall * sizeof(float), st));
  for (int s = 0; s < S; ++s)
    for (int k : segs[s]) backproject_launch(p, k, r + pl * p->first[k], D + nv * bin_of(k), 0, 1, 1.f, st);
  recip_launch(D, nall, st);
  // denoise's gam needs asum(D) on the host (osMOMSolverD.h:206).
  reduce_launch(2, D, nullptr, nall, p->d_partials, p->n_partials, asum_dev, st);
  double asum = 0.0;
  CBCT_CUDA(cudaMemcpyAsync(&asum, asum_dev, sizeof(double), cudaMemcpyDeviceToHost, st));
  CBCT_CUDA(cudaStreamSynchronize(st));
  const float lambda = prm.tv_weight;
  const float gam = 0.35f / lambda / (float(nall) / float(asum));
  if (x0) {
    CBCT_CUDA(cudaMemcpyAsync(z, x0, nall * sizeof(float), cudaMemcpyDeviceToDevice, st));
    CBCT_CUDA(cudaMemcpyAsync(xold, x0, nall * sizeof(float), cudaMemcpyDeviceToDevice, st));
  } else {
    CBCT_CUDA(cudaMemsetAsync(z, 0, nall * sizeof(float), st));
    CBCT_CUDA(cudaMemsetAsync(xold, 0, nall * sizeof(float), st));
  }
  std::vector<int> seg_of_bin(NB);
  double t = 1.0, told = 1.0;
  for (int it = 0; it < prm.iterations; ++it) {
    for (int s = 0; s < S; ++s) {
      t = 0.5 * (1.0 + std::sqrt(1.0 + 4.0 * t * t));
      std::fill(seg_of_bin.begin(), seg_of_bin.end(), -1);
      for (int k : segs[s]) {
        seg_of_bin[bin_of(k)] = k;
        forward_launch_ex(p, k, CBCT_F32, z + nv * bin_of(k), r + pl * p->first[k], b + pl * p->first[k], nullptr,
                          1.f, 1, p->offcorr[k], 0, nullptr, st);
      }
      const double stepsz = double(prm.beta) / (1.0 + double(prm.gamma) * it) * S;
      const double mom = (told - 1.0) / t;
      for (int bb = 0; bb < NB; ++bb) {
        const int k = seg_of_bin[bb];
        if (k >= 0)
          backproject_step_launch(p, k, r + pl * p->first[k], z + nv * bb, sbuf + nv * bb, D + nv * bb,
                                  float(stepsz), st);
        else
          CBCT_CUDA(cudaMemcpyAsync(sbuf + nv * bb, z + nv * bb, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
      }
      // denoise (osMOMSolverD.h:205-231): L = 4, sigma = 1/(tau L^2), tau and
      // sigma rescaled by theta = 1/sqrt(1 + 2 gam tau) after every step.
      float tau = prm.tau, sigma = 1.f / (tau * 4.f * 4.f);
      for (int rs = 0; rs < prm.reg_steps; ++rs) {
        const float scale = (1.f * sigma) / (1.f + sigma * prm.tv_alpha);
        for (int bb = 0; bb < NB; ++bb) {
          tv_primal_launch(z + nv * bb, P, nx, ny, nz, scale, st);
          tv_update_launch(P, z + nv * bb, sbuf + nv * bb, D + nv * bb, nx, ny, nz, 1.f, tau, tau / lambda, st);
        }
        const float theta = 1.f / std::sqrt(1.f + 2.f * gam * tau);
        tau *= theta;
        sigma /= theta;
      }
      // clamp and momentum: the update kernel with no gradient
      osmom_update_launch(z, xold, D, nullptr, nall, 0.f, float(mom), prm.non_negativity, st);
      told = t;
    }
  }
}

static void run_ossart(cbct_plan* p, const float* b, const float* x0, float* x, const cbct_solver_params& prm,
                       double* cost, float* Wp, float* r, float* V, cudaStream_t st) {
  const size_t nv = vol_elems(p);
  const int S = p->n_subsets;
  // Wp = 1/max(A 1, 1e-6): forward of a ones image (x holds it for now).
  fill_launch(x, nv, 1.f, st);
  for (int s = 0; s < S; ++s)
    forward_launch_ex(p, s, CBCT_F32, x, Wp + plane_elems(p) * p->first[s], nullptr, nullptr, 1.f, 2, 0, 0,
                      nullptr, st);
  // V_s = 1/max(A_s^T (W 1), 1e-6)
  fill_launch(r, proj_elems(p), 1.f, st);
  for (int s = 0; s < S; ++s) {
    float* rs = r + plane_elems(p) * p->first[s];
    if (p->d_pweights)  // mult_MH of CBSubsetWeightOperator weights its input
      mul_launch(rs, rs, p->d_pweights + plane_elems(p) * p->first[s], plane_elems(p) * p->count[s], st);
    if (p->offcorr[s]) offset_weight_launch(p, s, rs, rs, 0, st);
    backproject_recip_launch(p, s, rs, V + nv * s, st);
  }
  if (x0) CBCT_CUDA(cudaMemcpyAsync(x, x0, nv * sizeof(float), cudaMemcpyDeviceToDevice, st));
  else CBCT_CUDA(cudaMemsetAsync(x, 0, nv * sizeof(float), st));
  std::vector<int> order(S);
  for (int s = 0; s < S; ++s) order[s] = s;
  for (int it = 0; it < prm.iterations; ++it) {
    for (int is = 0; is < S; ++is) {
      const int s = order[is];
      const size_t o = plane_elems(p) * p->first[s];
      forward_launch_ex(p, s, CBCT_F32, x, r + o, b + o, Wp + o, -1.f, 1, p->offcorr[s], 0, nullptr, st);
      const double a = double(prm.beta) / (1.0 + double(prm.gamma) * it);
      backproject_sart_launch(p, s, r + o, x, V + nv * s, float(a), prm.non_negativity, st);
    }
    std::reverse(order.begin(), order.end());
    if (cost) {
      // ||A x - b||^2 over all views (one partial per forward block, summed in order).
      forward_launch_ex(p, p->n_subsets, CBCT_F32, x, r, b, nullptr, 1.f, 1, 0, 0, cost + it, st);
    }
  }
}

void osmom_precon(cbct_plan* p, float* D, cudaStream_t st) {
  const size_t nv = vol_elems(p), np = proj_elems(p);
  float* ws = workspace(p, nv + np);
  float* ones = ws;
  float* r = ws + nv;
  fill_launch(ones, nv, 1.f, st);
  for (int s = 0; s < p->n_subsets; ++s)
    forward_launch_ex(p, s, CBCT_F32, ones, r + plane_elems(p) * p->first[s], nullptr, nullptr, 1.f, 1,
                      p->offcorr[s], 0, nullptr, st);
  backproject_recip_launch(p, p->n_subsets, r, D, st);
}

void osmom_step(cbct_plan* p, int s, cbct_dtype bt, const void* b, float* z, float* xold, const float* D, float* r,
                float step, float mom, int nonneg, double* norm2, cudaStream_t st) {
  forward_launch_ex(p, s, CBCT_F32, z, r, b, nullptr, 1.f, 1, p->offcorr[s], 0, norm2, st, bt);
  backproject_mom_launch(p, s, r, z, xold, D, step, mom, nonneg, st);
}

struct GraphCache {
  cudaGraphExec_t exec = nullptr;
  std::vector<uint64_t> key;
  cudaStream_t cap = nullptr;
};

void graph_cache_free(cbct_plan* p) {
  ++p->generation;
  GraphCache* g = static_cast<GraphCache*>(p->graph_cache);
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->cap) cudaStreamDestroy(g->cap);
  delete g;
  p->graph_cache = nullptr;
}

template <class F>
static void run_maybe_graph(cbct_plan* p, bool use_graph, const std::vector<uint64_t>& key, cudaStream_t st,
                            F&& body) {
  if (!use_graph) {
    body(st);
    return;
  }
  GraphCache* gc = static_cast<GraphCache*>(p->graph_cache);
  if (!gc) {
    gc = new GraphCache();
    p->graph_cache = gc;
    CBCT_CUDA(cudaStreamCreateWithFlags(&gc->cap, cudaStreamNonBlocking));
  }
  if (!gc->exec || gc->key != key) {
    if (gc->exec) {
      CBCT_CUDA(cudaGraphExecDestroy(gc->exec));
      gc->exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    CBCT_CUDA(cudaStreamBeginCapture(gc->cap, cudaStreamCaptureModeThreadLocal));
    try {
      body(gc->cap);
    } catch (...) {
      cudaStreamEndCapture(gc->cap, &graph);
      if (graph) cudaGraphDestroy(graph);
      throw;
    }
    CBCT_CUDA(cudaStreamEndCapture(gc->cap, &graph));
    cudaError_t e = cudaGraphInstantiate(&gc->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) throw Error(CBCT_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
    gc->key = key;
  }
  CBCT_CUDA(cudaGraphLaunch(gc->exec, st));
}

void osmom_solve(cbct_plan* p, const void* b, const float* x0, float* z, const cbct_solver_params& prm,
                 double* resid, cudaStream_t st) {
  CBCT_REQUIRE(prm.proj_storage == CBCT_F32 || prm.proj_storage == CBCT_F16 || prm.proj_storage == CBCT_BF16,
               "unknown projection storage type");
  if (prm.tv_weight > 0.f) {
    if (prm.storage != CBCT_F32 || prm.proj_storage != CBCT_F32 || resid)
      throw Error(CBCT_ERR_UNSUPPORTED, "regularised OS-MOM: fp32 storage, no residual trace");
    CBCT_REQUIRE(prm.tau > 0.f && prm.reg_steps >= 0, "regularised OS-MOM needs tau > 0 and reg_steps >= 0");
    const size_t nv = vol_elems(p), nall = nv * p->n_bins;
    const size_t need = 3 * nall + proj_elems(p) + 3 * nv + 4;
    float* ws = workspace(p, need);
    float* tail = ws + 3 * nall + proj_elems(p) + 3 * nv;
    double* asum_dev = reinterpret_cast<double*>((reinterpret_cast<uintptr_t>(tail) + 7) & ~uintptr_t(7));
    run_osmom_tv(p, static_cast<const float*>(b), x0, z, prm, ws, ws + nall, ws + 2 * nall,
                 ws + 2 * nall + proj_elems(p), ws + 3 * nall + proj_elems(p), asum_dev, st);
    return;
  }
  if (p->n_bins > 1) {
    if (prm.storage != CBCT_F32 || prm.proj_storage != CBCT_F32 || resid)
      throw Error(CBCT_ERR_UNSUPPORTED, "binned OS-MOM: fp32 storage, no residual trace");
    const size_t nall = vol_elems(p) * p->n_bins;
    float* ws = workspace(p, 2 * nall + proj_elems(p));
    std::vector<uint64_t> key = {3, (uint64_t)b, (uint64_t)x0, (uint64_t)z, (uint64_t)prm.iterations,
                                 (uint64_t)prm.non_negativity, (uint64_t)p->n_bins};
    uint32_t bb, gg;
    std::memcpy(&bb, &prm.beta, 4);
    std::memcpy(&gg, &prm.gamma, 4);
    key.push_back(bb);
    key.push_back(gg);
    const float* bf = static_cast<const float*>(b);
    run_maybe_graph(p, prm.use_graph != 0, key, st, [&](cudaStream_t s) {
      run_osmom_bins(p, bf, x0, z, prm, ws, ws + nall, ws + 2 * nall, s);
    });
    return;
  }
  const size_t nv = vol_elems(p), np = proj_elems(p);
  const bool lowp = prm.storage != CBCT_F32;
  const size_t need = 2 * nv + np + (lowp ? (nv + 1) / 2 + 64 : 0);
  float* ws = workspace(p, need);
  float* xold = ws;
  float* D = ws + nv;
  float* r = ws + 2 * nv;
  void* shadow = lowp ? (void*)(((uintptr_t)(ws + 2 * nv + np) + 255) & ~uintptr_t(255)) : nullptr;
  std::vector<uint64_t> key = {1, (uint64_t)b, (uint64_t)x0, (uint64_t)z, (uint64_t)resid,
                               (uint64_t)prm.iterations, (uint64_t)prm.non_negativity, (uint64_t)prm.storage,
                               (uint64_t)prm.refine_every, (uint64_t)prm.proj_storage};
  uint32_t bb, gg;
  std::memcpy(&bb, &prm.beta, 4);
  std::memcpy(&gg, &prm.gamma, 4);
  key.push_back(bb);
  key.push_back(gg);
  run_maybe_graph(p, prm.use_graph != 0, key, st, [&](cudaStream_t s) {
    run_osmom(p, b, x0, z, prm, resid, xold, D, r, shadow, s);
  });
}

void ossart_solve(cbct_plan* p, const float* b, const float* x0, float* x, const cbct_solver_params& prm,
                  double* cost, cudaStream_t st) {
  const size_t nv = vol_elems(p), np = proj_elems(p);
  const size_t need = 2 * np + nv * p->n_subsets;
  float* ws = workspace(p, need);
  float* Wp = ws;
  float* r = ws + np;
  float* V = ws + 2 * np;
  std::vector<uint64_t> key = {2, (uint64_t)b, (uint64_t)x0, (uint64_t)x, (uint64_t)cost,
                               (uint64_t)prm.iterations, (uint64_t)prm.non_negativity};
  uint32_t bb, gg;
  std::memcpy(&bb, &prm.beta, 4);
  std::memcpy(&gg, &prm.gamma, 4);
  key.push_back(bb);
  key.push_back(gg);
  run_maybe_graph(p, prm.use_graph != 0, key, st, [&](cudaStream_t s) {
    run_ossart(p, b, x0, x, prm, cost, Wp, r, V, s);
  });
}

void fdk_run(cbct_plan* p, const void* proj, float* vol, const float* filter, uint32_t flags, float* work,
             cudaStream_t st, cbct_dtype proj_dtype) {
  const size_t np = proj_elems(p);
  if (!work) {
    if (p->fdk_work_elems < np) {
      plan_dealloc(p, p->d_fdk_work);
      p->d_fdk_work = nullptr;
      p->fdk_work_elems = 0;
      p->d_fdk_work = plan_alloc_n<float>(p, np);
      p->fdk_work_elems = np;
    }
    work = p->d_fdk_work;
  }
  const uint32_t f = flags | CBCT_FDK_RAMP | CBCT_FDK_COSINE;
  fdk_filter_launch(p, p->n_subsets, proj, work, filter, f, st, proj_dtype);
  backproject_launch(p, p->n_subsets, work, vol, 1, 0, 2.f / float(p->n_views), st);
}

}  // namespace cbct
