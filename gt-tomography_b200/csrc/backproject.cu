// backproject.cu -- voxel-driven cone-beam back-projection (mult_MH) for sm_100a.
//
// Semantics: conebeam_backwards_projection_kernel<FBP> (xray/conebeam_projection.cu:922-1037):
// each voxel centre is rotated into the view frame, projected from the source
// onto the (offset) detector and the projection is sampled bilinearly with
// border 0; samples are summed over the views of the call.  With FBP the FDK
// distance weight 1/U^2, U = (SAD + r sin(beta - phi))/SAD, multiplies each
// sample (:1009-1024).  No ray-length weight: the pair is unmatched, as in
// the reference.
//
// Layout of the work: a thread owns one (x, y) column and a run of kZB voxels
// along z.  For one view, the detector column u and the 1/distance factor are
// the same for the whole run, and the detector row is affine in z, so the
// per-view geometry is computed once per run.  Threads of a warp hold 32
// consecutive x voxels, so their taps fall on neighbouring detector pixels.
//
// Epilogues fuse what the reference runs as separate element-wise passes:
//  kStore : vol = scale * ((accumulate ? vol : 0) + sum)          (mult_MH, FDK 2/P)
//  kRecip : vol = 1 / max(sum, 1e-6)                                (precon, osMOMSolverD.h:115-120)
//  kMom   : OS-MOM update of z and xold                              (osMOMSolverD.h:155-175)
//  kSart  : x = x + step * V * sum, optional clamp                   (osSARTSolver.h:99-104)
#include "device_common.cuh"

namespace cbct {

namespace {

constexpr int kBX = 32, kBY = 4, kZB = 8;
constexpr int kMaxViewsSmem = 1024;

enum { kStore = 0, kRecip = 1, kMom = 2, kSart = 3 };

struct BpEpi {
  float* vol;            // kStore / kRecip output, kSart: x (in/out), kMom: z (in/out)
  float* xold;           // kMom
  const float* aux;      // kMom: precon D; kSart: V_s
  float scale;           // kStore: output scale; kMom/kSart: step
  float mom;             // kMom: (told-1)/t
  int nonneg;
  int accumulate;
};

template <int EPI, bool FDK>
__global__ void __launch_bounds__(kBX * kBY) bp_kernel(const float* __restrict__ proj,
                                                       const ViewParams* __restrict__ views,
                                                       int n_views, GridConst gc, BpEpi e) {
  extern __shared__ ViewParams sv[];
  const int tid = threadIdx.y * kBX + threadIdx.x;
  for (int i = tid; i < n_views; i += kBX * kBY) sv[i] = views[i];
  __syncthreads();

  const int i = blockIdx.x * kBX + threadIdx.x;
  const int j = blockIdx.y * kBY + threadIdx.y;
  const int k0 = blockIdx.z * kZB;
  if (i >= gc.nx || j >= gc.ny) return;

  const float x = fmaf(float(i) + 0.5f, gc.vx, -gc.hx);
  const float y = fmaf(float(j) + 0.5f, gc.vy, -gc.hy);
  const float z0 = fmaf(float(k0) + 0.5f, gc.vz, -gc.hz);
  const size_t plane = (size_t)gc.W * gc.H;

  float acc[kZB];
#pragma unroll
  for (int q = 0; q < kZB; ++q) acc[q] = 0.f;

  for (int p = 0; p < n_views; ++p) {
    const ViewParams& vp = sv[p];
    const float xr = fmaf(vp.cs, x, vp.sn * y);        // Rz(-theta) * pos
    const float yr = fmaf(-vp.sn, x, vp.cs * y);
    const float dist = yr + gc.SAD;
    const float inv = __fdiv_rn(1.f, dist);
    const float cu = fmaf(fmaf(gc.SDD * xr, inv, -vp.ox), gc.ku, gc.bu);
    const float A = gc.SDD * inv * gc.kv;               // detector rows per mm of z
    const float B = fmaf(-vp.oy, gc.kv, gc.bv);
    float w = 1.f;
    if (FDK) {
      // U = (SAD + r sin(beta - phi))/SAD = 1 - yr/SAD
      const float U = 1.f - yr / gc.SAD;
      w = 1.f / (U * U);
    }
    const float fu = floorf(cu);
    const float au = cu - fu;
    const int iu = int(fu);
    const bool u0ok = (unsigned)iu < (unsigned)gc.W, u1ok = (unsigned)(iu + 1) < (unsigned)gc.W;
    const int cu0 = min(max(iu, 0), gc.W - 1), cu1 = min(max(iu + 1, 0), gc.W - 1);
    const float* pv = proj + (size_t)p * plane;
    const float dz = A * gc.vz;
    float cv = fmaf(A, z0, B);
#pragma unroll
    for (int q = 0; q < kZB; ++q) {
      const float fv = floorf(cv);
      const float av = cv - fv;
      const int iv = int(fv);
      const bool v0ok = (unsigned)iv < (unsigned)gc.H, v1ok = (unsigned)(iv + 1) < (unsigned)gc.H;
      const float* r0 = pv + (size_t)min(max(iv, 0), gc.H - 1) * gc.W;
      const float* r1 = pv + (size_t)min(max(iv + 1, 0), gc.H - 1) * gc.W;
      const float p00 = (u0ok && v0ok) ? __ldg(r0 + cu0) : 0.f;
      const float p10 = (u1ok && v0ok) ? __ldg(r0 + cu1) : 0.f;
      const float p01 = (u0ok && v1ok) ? __ldg(r1 + cu0) : 0.f;
      const float p11 = (u1ok && v1ok) ? __ldg(r1 + cu1) : 0.f;
      const float a = fmaf(au, p10 - p00, p00);
      const float b = fmaf(au, p11 - p01, p01);
      const float s = fmaf(av, b - a, a);
      acc[q] = FDK ? fmaf(w, s, acc[q]) : acc[q] + s;
      cv += dz;
    }
  }

  const size_t base = ((size_t)k0 * gc.ny + j) * gc.nx + i;
  const size_t sz = (size_t)gc.nx * gc.ny;
#pragma unroll
  for (int q = 0; q < kZB; ++q) {
    if (k0 + q >= gc.nz) break;
    const size_t idx = base + q * sz;
    const float g = acc[q];
    if (EPI == kStore) {
      e.vol[idx] = e.scale * ((e.accumulate ? e.vol[idx] : 0.f) + g);
    } else if (EPI == kRecip) {
      e.vol[idx] = 1.f / fmaxf(g, 1e-6f);
    } else if (EPI == kMom) {
      const float zt = fmaf(-e.scale, e.aux[idx] * g, e.vol[idx]);
      const float xc = e.nonneg ? fmaxf(zt, 0.f) : zt;
      e.vol[idx] = fmaf(-e.mom, e.xold[idx], xc * (1.f + e.mom));
      e.xold[idx] = xc;
    } else {  // kSart
      float xn = fmaf(e.scale, e.aux[idx] * g, e.vol[idx]);
      if (e.nonneg) xn = fmaxf(xn, 0.f);
      e.vol[idx] = xn;
    }
  }
}

template <int EPI, bool FDK>
void launch_bp(cbct_plan* p, int s, const float* proj, const BpEpi& e, cudaStream_t st) {
  const int first = p->first[s], cnt = p->count[s];
  if (cnt > kMaxViewsSmem) throw Error(CBCT_ERR_UNSUPPORTED, "more than 1024 views in one back-projection");
  dim3 block(kBX, kBY);
  dim3 grid((p->g.nx + kBX - 1) / kBX, (p->g.ny + kBY - 1) / kBY, (p->g.nz + kZB - 1) / kZB);
  const size_t smem = sizeof(ViewParams) * (size_t)std::max(cnt, 1);
  auto k = bp_kernel<EPI, FDK>;
  ensure_smem_attr((const void*)k, smem);
  k<<<grid, block, smem, st>>>(proj, p->d_views + first, cnt, p->gc, e);
  check_launch("bp_kernel");
}

}  // namespace

void backproject_prepare(cbct_plan* p) {
  const size_t smem = sizeof(ViewParams) * (size_t)std::min(p->n_views, kMaxViewsSmem);
  ensure_smem_attr((const void*)bp_kernel<kStore, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kStore, true>, smem);
  ensure_smem_attr((const void*)bp_kernel<kRecip, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kMom, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kSart, false>, smem);
}

void backproject_launch(cbct_plan* p, int s, const float* proj, float* vol, int fdk_weight,
                        int accumulate, float out_scale, cudaStream_t st) {
  BpEpi e{};
  e.vol = vol;
  e.scale = out_scale;
  e.accumulate = accumulate;
  if (fdk_weight) launch_bp<kStore, true>(p, s, proj, e, st);
  else launch_bp<kStore, false>(p, s, proj, e, st);
}

void backproject_recip_launch(cbct_plan* p, int s, const float* proj, float* out, cudaStream_t st) {
  BpEpi e{};
  e.vol = out;
  launch_bp<kRecip, false>(p, s, proj, e, st);
}

void backproject_mom_launch(cbct_plan* p, int s, const float* proj, float* z, float* xold,
                            const float* precon, float step, float mom, int nonneg, cudaStream_t st) {
  BpEpi e{};
  e.vol = z;
  e.xold = xold;
  e.aux = precon;
  e.scale = step;
  e.mom = mom;
  e.nonneg = nonneg;
  launch_bp<kMom, false>(p, s, proj, e, st);
}

void backproject_sart_launch(cbct_plan* p, int s, const float* proj, float* x, const float* V,
                             float step, int nonneg, cudaStream_t st) {
  BpEpi e{};
  e.vol = x;
  e.aux = V;
  e.scale = step;
  e.nonneg = nonneg;
  launch_bp<kSart, false>(p, s, proj, e, st);
}

}  // namespace cbct
