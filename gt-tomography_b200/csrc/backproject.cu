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
//  kStep  : s = z - step * D * sum, into a separate image            (osMOMSolverD.h:151-157 before denoise)
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <utility>

#include "device_common.cuh"

namespace cbct {

namespace {

constexpr int kBX = 32, kBY = 4, kZB = 8;
constexpr int kMaxViewsSmem = 1024;

enum { kStore = 0, kRecip = 1, kMom = 2, kSart = 3, kStep = 4 };

struct BpEpi {
  const unsigned char* mask;  // voxel mask applied to the back-projection (nullable)
  float* vol;            // kStore / kRecip output, kSart: x (in/out), kMom: z (in/out)
  float* xold;           // kMom; kStep: z (input)
  const float* aux;      // kMom: precon D; kSart: V_s
  float scale;           // kStore: output scale; kMom/kSart: step
  float mom;             // kMom: (told-1)/t
  int nonneg;
  int accumulate;
};

// With a mask, the operator's output is multiplied by it (apply_mask after
// mult_MH, cuConebeamProjectionOperator.cpp:113-114), so the masked value of an
// accumulating call is mask * (incoming + sum).
// The epilogue of one voxel in two halves: the operands it reads (mask,
// incoming volume, xold or z, preconditioner or V) are loaded first, so that a
// thread can have the loads of several voxels in flight before any store.
struct BpOps {
  float m, v, x, a;
};

template <int EPI>
__device__ __forceinline__ BpOps bp_load(const BpEpi& e, size_t idx) {
  BpOps o;
  o.m = e.mask ? float(e.mask[idx]) : 1.f;
  o.v = (EPI == kMom || EPI == kSart || (EPI == kStore && e.accumulate)) ? e.vol[idx] : 0.f;
  o.x = (EPI == kMom || EPI == kStep) ? e.xold[idx] : 0.f;
  o.a = (EPI == kMom || EPI == kStep || EPI == kSart) ? e.aux[idx] : 0.f;
  return o;
}

template <int EPI>
__device__ __forceinline__ void bp_finish(const BpEpi& e, size_t idx, float g, const BpOps& o) {
  if (EPI == kStore) {
    e.vol[idx] = e.scale * (((e.accumulate ? o.v : 0.f) + g) * o.m);
    return;
  }
  g *= o.m;
  if (EPI == kRecip) {
    e.vol[idx] = 1.f / fmaxf(g, 1e-6f);
  } else if (EPI == kMom) {
    const float zt = fmaf(-e.scale, o.a * g, o.v);
    const float xc = e.nonneg ? fmaxf(zt, 0.f) : zt;
    e.vol[idx] = fmaf(-e.mom, o.x, xc * (1.f + e.mom));
    e.xold[idx] = xc;
  } else if (EPI == kStep) {
    e.vol[idx] = fmaf(-e.scale, o.a * g, o.x);
  } else {  // kSart
    float xn = fmaf(e.scale, o.a * g, o.v);
    if (e.nonneg) xn = fmaxf(xn, 0.f);
    e.vol[idx] = xn;
  }
}

template <int EPI>
__device__ __forceinline__ void bp_store(const BpEpi& e, size_t idx, float g) {
  bp_finish<EPI>(e, idx, g, bp_load<EPI>(e, idx));
}

// 1: the view loop of the TMA back-projector passes one barrier per view (the
// wait check rides on the barrier that frees the stage); 0 (shipped): two,
// the wait checked before the stage is read (measured the same: 0.514 vs
// 0.516 ms per C2 subset, 814.5 vs 815.0 GUPS for the solve).
#ifndef CBCT_BP_ONE_BARRIER
#define CBCT_BP_ONE_BARRIER 0
#endif

// Voxels of a thread's z-run whose epilogue operands are loaded together.
#ifndef CBCT_BP_EPI_CHUNK
#define CBCT_BP_EPI_CHUNK 4
#endif

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
    bp_store<EPI>(e, base + q * sz, acc[q]);
  }
}

// ------------------------------------------------------------------ TMA-staged
// A CTA owns a kTX x kTY x kZT voxel block; each warp holds an 8 x 4 patch of
// columns so that its lanes read a narrow range of detector words.  For each view the block's footprint
// on the detector (the bounding box of its eight projected corners, a convex
// image of a convex block) is staged into shared memory by a 3-D TMA load
// whose out-of-detector texels arrive as zeros, so the bilinear taps need no
// bounds checks.  Views are pipelined over two stages.
#ifndef CBCT_BP_ZRUN
#define CBCT_BP_ZRUN 16
#endif
constexpr int kZT = CBCT_BP_ZRUN;
constexpr int kTX = 16, kTY = 8;     // columns per CTA of the TMA back-projector

struct BpView {
  float cs, sn, ox, oy;
};

// Detector box widths (u, fp32 elements) the TMA back-projector is compiled
// for; a plan takes the smallest that holds its footprints.  Rows of a box
// sit BU floats apart, so BU mod 32 is the bank offset between the two rows a
// bilinear tap reads.
#ifdef CBCT_BP_WIDTHS_16
constexpr int kBpWidths[] = {48, 80, 112, 144};      // row offset 16 banks
#else
constexpr int kBpWidths[] = {40, 56, 72, 104, 136};  // row offset 8 or 24 banks
#endif
constexpr int kNBpWidths = int(sizeof(kBpWidths) / sizeof(int));

// Calls f(std::integral_constant<int, W>) for the compiled width W == w;
// false when w is not one of them.
template <int I = 0, class F>
bool with_bp_width(int w, F&& f) {
  if constexpr (I < kNBpWidths) {
    if (w == kBpWidths[I]) {
      f(std::integral_constant<int, kBpWidths[I]>{});
      return true;
    }
    return with_bp_width<I + 1>(w, std::forward<F>(f));
  } else {
    return false;
  }
}

// One CTA's work: the kTX x kTY x kZT voxel block (bi, bj, bk) over the views
// of the call.  Shared by the one-scan kernel (block = blockIdx) and the
// work-list kernel over many scans (block = the item's); base_ptr is the
// 128-byte aligned dynamic shared memory, bars/abort_flag the CTA's statics.
template <int EPI, bool FDK, int BU>
__device__ __forceinline__ void bp_tma_body(const CUtensorMap* map, const ViewParams* __restrict__ views,
                                            int n_views, const GridConst& gc, const BpEpi& e, int BV, int* flags,
                                            int bi, int bj, int bk, unsigned char* base_ptr, uint64_t* bars,
                                            int& abort_flag) {
  const uint32_t box_bytes = uint32_t(BU * BV * 4);
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  BpView* tv = reinterpret_cast<BpView*>(base_ptr + 2 * stage_stride);
  int2* org = reinterpret_cast<int2*>(tv + n_views);     // per view: (u origin, v origin)
  int2* ext = org + n_views;                             // per view: (max u, max v) for checks
  const int tid = threadIdx.x;
  const int nthr = kTX * kTY;
  const int i0 = bi * kTX, j0 = bj * kTY, k0 = bk * kZT;

  for (int q = tid; q < n_views; q += nthr) {
    const ViewParams& vp = views[q];
    tv[q] = BpView{vp.cs, vp.sn, vp.ox, vp.oy};
    org[q] = make_int2(INT_MAX, INT_MAX);
    ext[q] = make_int2(INT_MIN, INT_MIN);
  }
  if (tid == 0) {
    abort_flag = 0;
    mbar_init(&bars[0], 1);
    mbar_init(&bars[1], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // Footprints: 8 corners of the block (voxel centres) per view.
  const int ie = min(i0 + kTX, gc.nx) - 1, je = min(j0 + kTY, gc.ny) - 1, ke = min(k0 + kZT, gc.nz) - 1;
  for (int q = tid; q < n_views * 8; q += nthr) {
    const int pv = q >> 3, c = q & 7;
    const BpView w = tv[pv];
    const float x = fmaf(float((c & 1) ? ie : i0) + 0.5f, gc.vx, -gc.hx);
    const float y = fmaf(float((c & 2) ? je : j0) + 0.5f, gc.vy, -gc.hy);
    const float z = fmaf(float((c & 4) ? ke : k0) + 0.5f, gc.vz, -gc.hz);
    const float xr = fmaf(w.cs, x, w.sn * y);
    const float yr = fmaf(-w.sn, x, w.cs * y);
    const float inv = __frcp_rn(yr + gc.SAD);
    const float cu = fmaf(fmaf(gc.SDD * xr, inv, -w.ox), gc.ku, gc.bu);
    const float cv = fmaf(fmaf(gc.SDD * z, inv, -w.oy), gc.kv, gc.bv);
    const int fu = int(floorf(fminf(fmaxf(cu, -1.0e5f), 1.0e5f)));
    const int fv = int(floorf(fminf(fmaxf(cv, -1.0e5f), 1.0e5f)));
    atomicMin(&org[pv].x, fu);
    atomicMin(&org[pv].y, fv);
    atomicMax(&ext[pv].x, fu);
    atomicMax(&ext[pv].y, fv);
  }
  __syncthreads();
  for (int q = tid; q < n_views; q += nthr) {
    int2 o = org[q];
    o.x = (o.x - 1) & ~3;      // 16-byte aligned x start
    o.y = o.y - 1;
    if (ext[q].x + 2 - o.x >= BU || ext[q].y + 2 - o.y >= BV) atomicAdd(&flags[0], 1);
    org[q] = o;
  }
  __syncthreads();
  auto issue = [&](int pv) {
    uint64_t* bar = &bars[pv & 1];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(base_ptr + (pv & 1) * stage_stride, map, org[pv].x, org[pv].y, pv, bar);
  };
  if (tid == 0) {
    for (int pv = 0; pv < min(2, n_views); ++pv) issue(pv);
  }

  const int warp = tid >> 5, lane = tid & 31;
  const int i = i0 + (warp & 1) * 8 + (lane & 7), j = j0 + (warp >> 1) * 4 + (lane >> 3);
  const float x = fmaf(float(min(i, gc.nx - 1)) + 0.5f, gc.vx, -gc.hx);
  const float y = fmaf(float(min(j, gc.ny - 1)) + 0.5f, gc.vy, -gc.hy);
  const float z0 = fmaf(float(k0) + 0.5f, gc.vz, -gc.hz);
  const unsigned maxidx = unsigned(BU * (BV - 1) - 2);
  float acc[kZT];
#pragma unroll
  for (int q = 0; q < kZT; ++q) acc[q] = 0.f;
  int done = 0;
  for (int pv = 0; pv < n_views; ++pv) {
    const bool ok = mbar_wait_bounded(&bars[pv & 1], (pv >> 1) & 1, gc.wait_limit);
#if !CBCT_BP_ONE_BARRIER
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); abort_flag = 1; }
      break;
    }
    done = pv + 1;
#endif
    const BpView w = tv[pv];
    const int2 o = org[pv];
    const float* sp = reinterpret_cast<const float*>(base_ptr + (pv & 1) * stage_stride);
    const float xr = fmaf(w.cs, x, w.sn * y);
    const float yr = fmaf(-w.sn, x, w.cs * y);
    const float inv = __frcp_rn(yr + gc.SAD);
    const float cu = fmaf(fmaf(gc.SDD * xr, inv, -w.ox), gc.ku, gc.bu) - float(o.x);
    const float A = gc.SDD * inv * gc.kv;
    float cv = fmaf(fmaf(A, z0, -w.oy * gc.kv), 1.f, gc.bv) - float(o.y);
    const float dz = A * gc.vz;
    float wt = 1.f;
    if (FDK) {
      const float U = 1.f - yr / gc.SAD;
      wt = 1.f / (U * U);
    }
    // Floors and the box index on the FMA pipe (exact for |cv| < 2^22; the
    // index is clamped into the box below whatever it is).
    const float fu = floor_small(cu);
    const float au = cu - fu;
    const float2 tu = make_float2(au, au);
    const float fubc = fu + kRoundC;
#pragma unroll
    for (int q = 0; q < kZT; ++q) {
      const float fv = floor_small(cv);
      const float av = cv - fv;
      const int idx0 = int_of_biased(fmaf(fv, float(BU), fubc));
      const unsigned idx = min((unsigned)idx0, maxidx);
      const float* t = sp + idx;
      const float2 r0 = make_float2(t[0], t[BU]);        // (u0,v0) (u0,v1)
      const float2 r1 = make_float2(t[1], t[BU + 1]);    // (u1,v0) (u1,v1)
      const float2 h = __ffma2_rn(tu, r1, __ffma2_rn(make_float2(-au, -au), r0, r0));
      const float smp = fmaf(av, h.y - h.x, h.x);
      acc[q] = FDK ? fmaf(wt, smp, acc[q]) : acc[q] + smp;
      cv += dz;
    }
#if CBCT_BP_ONE_BARRIER
    // One barrier per view: every thread is done with the stage before it is
    // refilled, and a wait that gave up anywhere ends the loop (the taps read
    // after such a wait stay inside the box; the block's sums are discarded
    // with the error status).
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); abort_flag = 1; }
      break;
    }
    done = pv + 1;
#else
    __syncthreads();
#endif
    if (tid == 0 && pv + 2 < n_views) {
      fence_proxy_async();
      issue(pv + 2);
    }
  }
  if (abort_flag && tid == 0) {
    for (int pv = done; pv < min(done + 2, n_views); ++pv)
      if (!mbar_wait_bounded(&bars[pv & 1], (pv >> 1) & 1, kWaitLimit)) abort_flag = 2;
  }
  if (i >= gc.nx || j >= gc.ny) return;
  const size_t base = ((size_t)k0 * gc.ny + j) * gc.nx + i;
  const size_t sz = (size_t)gc.nx * gc.ny;
  const int nq = min(kZT, gc.nz - k0);
  constexpr int C = CBCT_BP_EPI_CHUNK;
  static_assert(kZT % C == 0, "epilogue chunks tile the z-run");
#pragma unroll
  for (int c0 = 0; c0 < kZT; c0 += C) {
    BpOps ops[C];
#pragma unroll
    for (int q = 0; q < C; ++q)
      if (c0 + q < nq) ops[q] = bp_load<EPI>(e, base + (c0 + q) * sz);
#pragma unroll
    for (int q = 0; q < C; ++q)
      if (c0 + q < nq) bp_finish<EPI>(e, base + (c0 + q) * sz, acc[c0 + q], ops[q]);
  }
}

template <int EPI, bool FDK, int BU>
__global__ void __launch_bounds__(kTX * kTY) bp_tma_kernel(const __grid_constant__ CUtensorMap map,
                                                           const ViewParams* __restrict__ views, int n_views,
                                                           GridConst gc, BpEpi e, int BV, int* flags) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ uint64_t bars[2];
  __shared__ int abort_flag;
  unsigned char* base_ptr =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  bp_tma_body<EPI, FDK, BU>(&map, views, n_views, gc, e, BV, flags, blockIdx.x, blockIdx.y, blockIdx.z, base_ptr,
                            bars, abort_flag);
}

// One scan's entry in the work list of bp_tma_multi_kernel: the arguments of
// its one-scan launch and where its CTAs start in the list.
struct alignas(128) BpScanRec {
  CUtensorMap map;             // the subset's projections (W, H, views), box BU x BV
  const ViewParams* views;
  int* flags;
  GridConst gc;
  BpEpi e;
  int n_views, BV;
  int tx, ty;                  // CTA grid of the scan (x, y; z follows)
  int base;                    // work-list index of the scan's first CTA
};

// Work-list (persistent) back-projector over many scans of one box width:
// resident CTAs take work-list items (one voxel block of one scan) from an
// atomic counter until the list is empty; the item runs the one-scan kernel's
// body, so every voxel gets the same arithmetic as in a launch of its own.
// Items are numbered scan by scan, CTA-grid order (x fastest) inside a scan.
template <int EPI, bool FDK, int BU>
__global__ void __launch_bounds__(kTX * kTY) bp_tma_multi_kernel(const BpScanRec* __restrict__ recs, int n_recs,
                                                                 int total, int* __restrict__ counter) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ uint64_t bars[2];
  __shared__ int abort_flag;
  __shared__ int item;
  __shared__ int base[kMultiMaxRecs];
  unsigned char* base_ptr =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  for (int i = threadIdx.x; i < n_recs; i += blockDim.x) base[i] = recs[i].base;
  int last = -1;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(counter, 1);
    __syncthreads();
    const int t = item;
    if (t >= total) break;
    // Broadcast: the compiler may then keep the record's fields uniform.
    const int lo = __shfl_sync(0xffffffffu, find_rec(base, n_recs, t), 0);
    const BpScanRec& R = recs[lo];
    int l = t - base[lo];
    const int bi = l % R.tx;
    l /= R.tx;
    const int bj = l % R.ty, bk = l / R.ty;
    if (threadIdx.x == 0 && lo != last) {   // the thread that issues the TMA loads
      tensormap_acquire(&R.map);
      last = lo;
    }
    bp_tma_body<EPI, FDK, BU>(&R.map, R.views, R.n_views, R.gc, R.e, R.BV, R.flags, bi, bj, bk, base_ptr, bars,
                              abort_flag);
    __syncthreads();
    // A wait that gave up is counted in the scan's flag word and its loads
    // drained; only a CTA whose drain also gave up (a copy may still land in
    // its shared memory) stops taking items.
    const bool ok = abort_flag != 2;
    if (threadIdx.x == 0) {
      mbar_inval(&bars[0]);
      mbar_inval(&bars[1]);
    }
    if (!ok) break;
  }
}

size_t bp_tma_smem(const cbct_plan* p, int n_views) {
  const size_t stage = ((size_t)p->bp_box.bx * p->bp_box.by * 4 + 127) & ~size_t(127);
  return 128 + 2 * stage + (size_t)n_views * (sizeof(BpView) + 2 * sizeof(int2));
}

// Tensor map of cnt projections (W x H, fp32) with the plan's detector box.
CUtensorMap make_bp_map(const cbct_plan* p, const float* proj, int cnt) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  cuuint64_t dims[3] = {(cuuint64_t)p->g.width, (cuuint64_t)p->g.height, (cuuint64_t)cnt};
  cuuint64_t strides[2] = {(cuuint64_t)p->g.width * 4, (cuuint64_t)p->g.width * p->g.height * 4};
  cuuint32_t box[3] = {(cuuint32_t)p->bp_box.bx, (cuuint32_t)p->bp_box.by, 1};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult res = tensor_map_encoder()(&m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float*>(proj), dims,
                                      strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (res != CUDA_SUCCESS) throw Error(CBCT_ERR_CUDA, "cuTensorMapEncodeTiled (projections) failed");
  return m;
}

template <int EPI, bool FDK, int BU>
void launch_bp_tma(cbct_plan* p, int first, int cnt, const float* proj, const BpEpi& e, cudaStream_t st) {
  const CUtensorMap m = make_bp_map(p, proj, cnt);
  dim3 block(kTX * kTY);
  dim3 grid((p->g.nx + kTX - 1) / kTX, (p->g.ny + kTY - 1) / kTY, (p->g.nz + kZT - 1) / kZT);
  const size_t smem = bp_tma_smem(p, cnt);
  auto k = bp_tma_kernel<EPI, FDK, BU>;
  ensure_smem_attr((const void*)k, smem);
  k<<<grid, block, smem, st>>>(m, p->d_views + first, cnt, p->gc, e, p->bp_box.by, p->d_flags);
  check_launch("bp_tma_kernel");
}

template <int EPI, bool FDK>
bool try_bp_tma(cbct_plan* p, int first, int cnt, const float* proj, const BpEpi& e, cudaStream_t st) {
  if (p->bp_variant != 1 || cnt > p->bp_max_views || (reinterpret_cast<uintptr_t>(proj) % 16) != 0) return false;
  return with_bp_width(p->bp_box.bx, [&](auto W) {
    launch_bp_tma<EPI, FDK, decltype(W)::value>(p, first, cnt, proj, e, st);
  });
}

template <int EPI, bool FDK, int BU>
void prepare_bp_width(size_t smem) {
  ensure_smem_attr((const void*)bp_tma_kernel<EPI, FDK, BU>, smem);
}

template <int BU>
void prepare_bp_all(size_t smem) {
  prepare_bp_width<kStore, false, BU>(smem);
  prepare_bp_width<kStore, true, BU>(smem);
  prepare_bp_width<kRecip, false, BU>(smem);
  prepare_bp_width<kMom, false, BU>(smem);
  prepare_bp_width<kSart, false, BU>(smem);
  prepare_bp_width<kStep, false, BU>(smem);
}

template <int EPI, bool FDK>
void launch_bp(cbct_plan* p, int s, const float* proj, const BpEpi& e, cudaStream_t st) {
  const int first = p->first[s], cnt = p->count[s];
  if (cnt == 0) return;
  if (try_bp_tma<EPI, FDK>(p, first, cnt, proj, e, st)) return;
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

// Chooses the TMA-staged back-projector and its detector box: the largest
// footprint of any kTX x kTY x kZT block in any view (FP64, corner projections),
// plus margins.
void backproject_choose_variant(cbct_plan* p) {
  const cbct_geometry& g = p->g;
  p->bp_variant = 0;
  p->bp_box = SlabBox{0, 0, 0, 0};
  p->bp_max_views = 0;
  if (p->force_gather || p->bp_pref == 1 || (g.width * 4) % 16 != 0) return;
  const double vx = double(g.lx) / g.nx, vy = double(g.ly) / g.ny, vz = double(g.lz) / g.nz;
  const double ku = g.width / double(g.fov_u), kv = g.height / double(g.fov_v);
  const double bu = g.width / 2.0 - 0.5, bv = g.height / 2.0 - 0.5;
  const int bxn = (g.nx + kTX - 1) / kTX, byn = (g.ny + kTY - 1) / kTY, bzn = (g.nz + kZT - 1) / kZT;
  std::vector<std::pair<int, int>> acc(host_threads(), {0, 0});
  parallel_for(p->n_views, [&](int lo, int hi, int tid) {
    int& eu = acc[tid].first;
    int& ev = acc[tid].second;
    for (int iv = lo; iv < hi; ++iv) {
      const double th = double(p->angles[iv]) * (3.14159265358979323846 / 180.0);
      const double cs = std::cos(th), sn = std::sin(th);
      const double ox = p->offsets[2 * iv], oy = p->offsets[2 * iv + 1];
      for (int bi = 0; bi < bxn; ++bi)
        for (int bj = 0; bj < byn; ++bj) {
          const int i0 = bi * kTX, ie = std::min(i0 + kTX, g.nx) - 1;
          const int j0 = bj * kTY, je = std::min(j0 + kTY, g.ny) - 1;
          double umn = 1e30, umx = -1e30, imn = 1e30, imx = -1e30;
          for (int c = 0; c < 4; ++c) {
            const double x = (((c & 1) ? ie : i0) + 0.5) * vx - g.lx / 2.0;
            const double y = (((c & 2) ? je : j0) + 0.5) * vy - g.ly / 2.0;
            const double xr = cs * x + sn * y, yr = -sn * x + cs * y;
            const double inv = 1.0 / (yr + g.SAD);
            const double u = (g.SDD * xr * inv - ox) * ku + bu;
            umn = std::min(umn, u); umx = std::max(umx, u);
            imn = std::min(imn, inv); imx = std::max(imx, inv);
          }
          eu = std::max(eu, (int)(std::floor(umx) - std::floor(umn)) + 3 + 2);
          // rows: z spans of every z block, at the nearest and farthest magnification
          for (int bk = 0; bk < bzn; ++bk) {
            const int k0 = bk * kZT, ke = std::min(k0 + kZT, g.nz) - 1;
            const double z0 = (k0 + 0.5) * vz - g.lz / 2.0, z1 = (ke + 0.5) * vz - g.lz / 2.0;
            double vmn = 1e30, vmx = -1e30;
            for (double inv : {imn, imx})
              for (double z : {z0, z1}) {
                const double v = (g.SDD * z * inv - oy) * kv + bv;
                vmn = std::min(vmn, v); vmx = std::max(vmx, v);
              }
            ev = std::max(ev, (int)(std::floor(vmx) - std::floor(vmn)) + 3 + 2);
          }
        }
    }
  });
  int eu = 0, ev = 0;
  for (auto& a : acc) {
    eu = std::max(eu, a.first);
    ev = std::max(ev, a.second);
  }
  int w = 0;
  for (int c : kBpWidths)
    if (c >= eu + 3) { w = c; break; }
  if (w == 0 || ev > 256) return;
  p->bp_box = SlabBox{w, std::max(ev, 2), 1, 1};
  const int maxv = std::min(p->n_views, 1024);
  if (bp_tma_smem(p, maxv) > (size_t)kSmemBudget) return;
  p->bp_max_views = maxv;
  p->bp_variant = 1;
}

void backproject_prepare(cbct_plan* p) {
  if (p->bp_variant == 1) {
    const size_t sm = bp_tma_smem(p, p->bp_max_views);
    with_bp_width(p->bp_box.bx, [&](auto W) { prepare_bp_all<decltype(W)::value>(sm); });
  }
  const size_t smem = sizeof(ViewParams) * (size_t)std::min(p->n_views, kMaxViewsSmem);
  ensure_smem_attr((const void*)bp_kernel<kStore, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kStore, true>, smem);
  ensure_smem_attr((const void*)bp_kernel<kRecip, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kMom, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kSart, false>, smem);
  ensure_smem_attr((const void*)bp_kernel<kStep, false>, smem);
}

void backproject_launch(cbct_plan* p, int s, const float* proj, float* vol, int fdk_weight,
                        int accumulate, float out_scale, cudaStream_t st) {
  BpEpi e{};
  e.mask = fdk_weight ? nullptr : p->d_mask;
  e.vol = vol;
  e.scale = out_scale;
  e.accumulate = accumulate;
  if (fdk_weight) launch_bp<kStore, true>(p, s, proj, e, st);
  else launch_bp<kStore, false>(p, s, proj, e, st);
}

void backproject_recip_launch(cbct_plan* p, int s, const float* proj, float* out, cudaStream_t st) {
  BpEpi e{};
  e.mask = p->d_mask;
  e.vol = out;
  launch_bp<kRecip, false>(p, s, proj, e, st);
}

void backproject_mom_launch(cbct_plan* p, int s, const float* proj, float* z, float* xold,
                            const float* precon, float step, float mom, int nonneg, cudaStream_t st) {
  BpEpi e{};
  e.mask = p->d_mask;
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
  e.mask = p->d_mask;
  e.vol = x;
  e.aux = V;
  e.scale = step;
  e.nonneg = nonneg;
  launch_bp<kSart, false>(p, s, proj, e, st);
}

void backproject_step_launch(cbct_plan* p, int s, const float* proj, const float* z, float* out,
                             const float* precon, float step, cudaStream_t st) {
  BpEpi e{};
  e.mask = p->d_mask;
  e.vol = out;
  e.xold = const_cast<float*>(z);
  e.aux = precon;
  e.scale = step;
  launch_bp<kStep, false>(p, s, proj, e, st);
}

namespace {

// Work-list launch of one box width: records at A.dev + off.
template <int EPI, int BU>
void add_bp_group(WorkArena& A, const std::vector<BpScanRec>& recs, int total, size_t smem) {
  auto k = bp_tma_multi_kernel<EPI, false, BU>;
  ensure_smem_attr((const void*)k, smem);
  const size_t off = A.add(recs.data(), recs.size() * sizeof(BpScanRec));
  const int ci = A.n_counters++;
  const int grid = std::min(total, resident_grid((const void*)k, kTX * kTY, smem));
  const int n = (int)recs.size();
  A.ops.push_back([&A, k, off, ci, grid, n, total, smem](cudaStream_t st) {
    k<<<grid, kTX * kTY, smem, st>>>(reinterpret_cast<const BpScanRec*>(A.dev + off), n, total, A.counter(ci));
    check_launch("bp_tma_multi_kernel");
  });
}

template <int EPI>
const void* bp_multi_ptr(int c) {
  const void* k = nullptr;
  with_bp_width(kBpWidths[c], [&](auto W) { k = (const void*)bp_tma_multi_kernel<EPI, false, decltype(W)::value>; });
  return k;
}

template <int EPI>
void backproject_multi_t(WorkArena& A, const std::vector<MultiBpJob>& jobs) {
  std::vector<BpScanRec> groups[kNBpWidths];
  int totals[kNBpWidths] = {};
  size_t smem[kNBpWidths] = {};
  auto flush = [&](int c) {
    if (groups[c].empty()) return;
    with_bp_width(kBpWidths[c], [&](auto W) { add_bp_group<EPI, decltype(W)::value>(A, groups[c], totals[c], smem[c]); });
    groups[c].clear();
    totals[c] = 0;
    smem[c] = 0;
  };
  for (const MultiBpJob& j : jobs) {
    cbct_plan* p = j.p;
    BpEpi e{};
    e.mask = p->d_mask;
    e.vol = j.vol;
    e.xold = j.xold;
    e.aux = j.aux;
    e.scale = j.step;
    e.mom = j.mom;
    e.nonneg = j.nonneg;
    const int first = p->first[j.s], cnt = p->count[j.s];
    if (cnt == 0) continue;
    int w = -1;
    for (int c = 0; c < kNBpWidths; ++c)
      if (kBpWidths[c] == p->bp_box.bx) w = c;
    const bool tma = p->bp_variant == 1 && cnt <= p->bp_max_views &&
                     (reinterpret_cast<uintptr_t>(j.proj) % 16) == 0 && w >= 0;
    const int tx = (p->g.nx + kTX - 1) / kTX, ty = (p->g.ny + kTY - 1) / kTY, tz = (p->g.nz + kZT - 1) / kZT;
    bool own = !tma;
    if (tma) {
      const void* kfn = bp_multi_ptr<EPI>(w);
      const size_t sm = bp_tma_smem(p, cnt);
      ensure_smem_attr(kfn, sm);
      own = tx * ty * tz >= kMultiFillWaves * resident_grid(kfn, kTX * kTY, sm);
    }
    if (own) {
      const int s = j.s;
      const float* proj = j.proj;
      A.ops.push_back([p, s, proj, e](cudaStream_t st) { launch_bp<EPI, false>(p, s, proj, e, st); });
      continue;
    }
    BpScanRec r;
    std::memset(&r, 0, sizeof(r));
    r.map = make_bp_map(p, j.proj, cnt);
    r.views = p->d_views + first;
    r.flags = p->d_flags;
    r.gc = p->gc;
    r.e = e;
    r.n_views = cnt;
    r.BV = p->bp_box.by;
    r.tx = tx;
    r.ty = ty;
    if ((int)groups[w].size() == kMultiMaxRecs) flush(w);
    r.base = totals[w];
    totals[w] += r.tx * r.ty * tz;
    smem[w] = std::max(smem[w], bp_tma_smem(p, cnt));
    groups[w].push_back(r);
  }
  for (int c = 0; c < kNBpWidths; ++c) flush(c);
}

}  // namespace

void backproject_multi(WorkArena& A, int kind, const std::vector<MultiBpJob>& jobs) {
  if (kind == 0) backproject_multi_t<kRecip>(A, jobs);
  else backproject_multi_t<kMom>(A, jobs);
}

}  // namespace cbct
