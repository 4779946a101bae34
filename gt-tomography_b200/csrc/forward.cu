// forward.cu -- cone-beam forward projector (mult_M) for sm_100a.
//
// Semantics: conebeam_forwards_projection_kernel (xray/conebeam_projection.cu:412-528):
// one ray per detector pixel from the source to the pixel centre, clipped to
// the volume box, N = (int)(spp*nx) equidistant samples from the entry point,
// trilinear interpolation with border 0, result scaled by the sample spacing.
// Interpolation here is FP32 in software (not 9-bit texture weights).
//
// Two variants:
//  * fwd_slab_kernel (default): a CTA marches a 16x16 tile of rays of one view
//    through the volume in slabs of kTS voxels along the view's dominant axis.
//    Each slab's footprint (the box around the tile's ray pyramid) is staged
//    into shared memory by a 3-D TMA load; out-of-volume texels arrive as zeros
//    (the border rule for free).  Samples are taken in ray order, so each ray's
//    sum has the same order as the reference.
//  * fwd_gather_kernel: the same arithmetic with bounds-checked global loads.
//    Used when the plan's geometry does not fit the slab box budget or the
//    volume pitch is not TMA-aligned.
#include <climits>
#include <cmath>
#include <cstring>
#include <mutex>

#include "device_common.cuh"

namespace cbct {

namespace {

enum { kModeStore = 0, kModeResidual = 1, kModeRecip = 2 };

struct FwdOut {
  float* out;            // projections of the subset (W,H,P_s)
  const float* b;        // measured projections (residual mode; NULL reads as 0)
  const float* pw;       // per-pixel weight (residual mode; nullable)
  float scale;           // residual scale
  int mode;
  int apply_offset;      // residual mode: multiply by the sin^2 Wang weight
  int accumulate;        // store mode: out += result
  double* partials;      // residual mode: per-block sum of squares (nullable)
};

constexpr uint32_t kWaitLimit = 1u << 22;

// Sample range of a ray restricted to the box grown by half a voxel: samples
// outside it touch only border texels and add exactly 0.  Returns false when
// no sample can contribute.
__device__ __forceinline__ bool grown_range(const ViewParams& vp, const GridConst& gc, int u, int v,
                                            const Ray& r, int& k0, int& k1) {
  const float dx = fmaf(float(u), vp.Eux, vp.D0x);
  const float dy = fmaf(float(u), vp.Euy, vp.D0y);
  const float dz = fmaf(float(v), vp.Evz, vp.D0z);
  const float gx = gc.hx + 0.5005f * gc.vx, gy = gc.hy + 0.5005f * gc.vy, gz = gc.hz + 0.5005f * gc.vz;
  const float tx1 = __fdiv_rn(gx - vp.Sx, dx), tx2 = __fdiv_rn(-gx - vp.Sx, dx);
  const float ty1 = __fdiv_rn(gy - vp.Sy, dy), ty2 = __fdiv_rn(-gy - vp.Sy, dy);
  const float tz1 = __fdiv_rn(gz, dz), tz2 = __fdiv_rn(-gz, dz);
  const float tl = fmaxf(fmaxf(fminf(tx1, tx2), fminf(ty1, ty2)), fminf(tz1, tz2));
  const float th = fminf(fminf(fmaxf(tx1, tx2), fmaxf(ty1, ty2)), fmaxf(tz1, tz2));
  const float ta = fminf(r.a1, r.a2), tb = fmaxf(r.a1, r.a2);
  if (!(tl <= th) || th < ta || tl > tb) return false;
  const float f = (r.a2 - r.a1) * gc.invN;
  if (f == 0.f) { k0 = 0; k1 = gc.N - 1; return true; }
  const float q1 = (tl - r.a1) / f, q2 = (th - r.a1) / f;
  const float lo = fmaxf(fminf(q1, q2) - 1.f, 0.f);
  const float hi = fminf(fmaxf(q1, q2) + 1.f, float(gc.N - 1));
  k0 = int(floorf(lo));
  k1 = int(ceilf(hi));
  return k0 <= k1;
}

template <class V>
__device__ __forceinline__ float march_global(const V* __restrict__ vol, const GridConst& gc,
                                              const Ray& r, int k0, int k1) {
  float acc = 0.f;
  for (int k = k0; k <= k1; ++k) {
    const float kf = float(k);
    acc += fetch3_global(vol, gc.nx, gc.ny, gc.nz, fmaf(kf, r.dcx, r.c0x), fmaf(kf, r.dcy, r.c0y),
                         fmaf(kf, r.dcz, r.c0z));
  }
  return acc;
}

// Epilogue shared by both variants.  All threads of the block must call it.
__device__ __forceinline__ void fwd_epilogue(const FwdOut& o, const GridConst& gc, const ViewParams& vp,
                                             int p, int u, int v, bool active, float val,
                                             double* sh_red, int tid) {
  double sq = 0.0;
  if (active) {
    const size_t idx = ((size_t)p * gc.H + v) * gc.W + u;
    if (o.mode == kModeStore) {
      o.out[idx] = o.accumulate ? o.out[idx] + val : val;
    } else if (o.mode == kModeRecip) {
      o.out[idx] = 1.f / fmaxf(val, 1e-6f);
    } else {
      const float d = o.b ? val - o.b[idx] : val;
      sq = double(d) * double(d);
      float w = o.scale;
      if (o.pw) w *= o.pw[idx];
      if (o.apply_offset) w *= offset_weight_full(gc.fov_u, gc.W, u, vp.ox);
      o.out[idx] = d * w;
    }
  }
  if (o.partials != nullptr) {
    // Deterministic block sum; one partial per block in launch order.
    double t = warp_sum(sq);
    const int w = tid >> 5, l = tid & 31;
    if (l == 0) sh_red[w] = t;
    __syncthreads();
    if (tid < 32) {
      double q = (l < (int)(blockDim.x * blockDim.y) / 32) ? sh_red[l] : 0.0;
      q = warp_sum(q);
      if (tid == 0) {
        const size_t bid = ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        o.partials[bid] = q;
      }
    }
  }
}

// ------------------------------------------------------------------ gather
template <class V>
__global__ void __launch_bounds__(256) fwd_gather_kernel(const V* __restrict__ vol,
                                                         const ViewParams* __restrict__ views,
                                                         GridConst gc, FwdOut o) {
  __shared__ double sh_red[8];
  const int tid = threadIdx.x;
  const int u = blockIdx.x * kTU + (tid % kTU);
  const int v = blockIdx.y * kTV + (tid / kTU);
  const int p = blockIdx.z;
  const ViewParams vp = views[p];
  const bool active = (u < gc.W) && (v < gc.H);
  float val = 0.f;
  if (active) {
    const Ray r = make_ray(vp, gc, u, v);
    int k0, k1;
    if (grown_range(vp, gc, u, v, r, k0, k1)) val = march_global(vol, gc, r, k0, k1) * r.delta;
  }
  fwd_epilogue(o, gc, vp, p, u, v, active, val, sh_red, tid);
}

// ------------------------------------------------------------------ slab/TMA
template <class V, bool CHECK>
__device__ __forceinline__ float tri_box(const V* __restrict__ s, int BX, int BXY, int mx, int my,
                                         int mz, float lx, float ly, float lz, int& bad) {
  const float fx = floorf(lx), fy = floorf(ly), fz = floorf(lz);
  const float ax = lx - fx, ay = ly - fy, az = lz - fz;
  int ix = int(fx), iy = int(fy), iz = int(fz);
  if (CHECK) bad |= (ix < 0) | (ix > mx) | (iy < 0) | (iy > my) | (iz < 0) | (iz > mz);
  ix = min(max(ix, 0), mx);
  iy = min(max(iy, 0), my);
  iz = min(max(iz, 0), mz);
  const V* q = s + ix + iy * BX + iz * BXY;
  const float v000 = sm_f(q[0]), v100 = sm_f(q[1]);
  const float v010 = sm_f(q[BX]), v110 = sm_f(q[BX + 1]);
  const float v001 = sm_f(q[BXY]), v101 = sm_f(q[BXY + 1]);
  const float v011 = sm_f(q[BXY + BX]), v111 = sm_f(q[BXY + BX + 1]);
  const float c00 = fmaf(ax, v100 - v000, v000), c10 = fmaf(ax, v110 - v010, v010);
  const float c01 = fmaf(ax, v101 - v001, v001), c11 = fmaf(ax, v111 - v011, v011);
  const float c0 = fmaf(ay, c10 - c00, c00), c1 = fmaf(ay, c11 - c01, c01);
  return fmaf(az, c1 - c0, c0);
}

struct SlabShared {
  uint64_t bars[kNStage];
  int mlo, mhi, abort_flag;
  int emin[kMaxSlabs], emax[kMaxSlabs], zmin[kMaxSlabs], zmax[kMaxSlabs];
  double red[8];
};

// DOM = 1: rays mostly along y (slabs are y ranges, the in-plane cross axis is x);
// DOM = 0: rays mostly along x.
template <class V, int DOM, bool CHECK>
__device__ void slab_body(const CUtensorMap* map, const V* __restrict__ vol, const ViewParams& vp,
                         const GridConst& gc, const SlabBox& box, const FwdOut& o, int* flags,
                         unsigned char* smem_raw, SlabShared& sh) {
  const int tid = threadIdx.x;
  const int p = blockIdx.z;
  const int u0 = blockIdx.x * kTU, v0 = blockIdx.y * kTV;
  const int u = u0 + (tid % kTU), v = v0 + (tid / kTU);
  const bool active = (u < gc.W) && (v < gc.H);
  const Ray r = make_ray(vp, gc, min(u, gc.W - 1), min(v, gc.H - 1));
  const bool hit = active && (r.a2 > r.a1);
  const float c0d = DOM ? r.c0y : r.c0x, dcd = DOM ? r.dcy : r.dcx;
  const int Nd = DOM ? gc.ny : gc.nx;
  (void)Nd;

  if (tid == 0) {
    sh.mlo = INT_MAX;
    sh.mhi = INT_MIN;
    sh.abort_flag = 0;
    for (int s = 0; s < kNStage; ++s) mbar_init(&sh.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (hit) {
    const int f0 = int(floorf(c0d));
    const int f1 = int(floorf(fmaf(float(gc.N - 1), dcd, c0d)));
    const int m0 = (max(f0, kSlabBase) - kSlabBase) / kTS;
    const int m1 = (max(f1, kSlabBase) - kSlabBase) / kTS;
    atomicMin(&sh.mlo, min(m0, m1));
    atomicMax(&sh.mhi, max(m0, m1));
  }
  __syncthreads();
  const int mlo = sh.mlo, mhi = sh.mhi;
  int nslab = (mhi >= mlo) ? (mhi - mlo + 1) : 0;
  if (nslab > kMaxSlabs) {
    if (tid == 0) atomicAdd(&flags[0], 1);
    nslab = 0;
  }

  // Footprint of every slab: bounding box of the four corner rays of the tile
  // at the two bounding planes of the slab (the tile's rays form a convex
  // pyramid, so its cross-section inside the slab lies in that box).
  for (int i = tid; i < nslab; i += blockDim.x) {
    sh.emin[i] = INT_MAX; sh.emax[i] = INT_MIN;
    sh.zmin[i] = INT_MAX; sh.zmax[i] = INT_MIN;
  }
  __syncthreads();
  const int ue = min(u0 + kTU, gc.W) - 1, ve = min(v0 + kTV, gc.H) - 1;
  for (int q = tid; q < nslab * 8; q += blockDim.x) {
    const int i = q >> 3, c = q & 7;
    const int m = mlo + i;
    const float plane = float(kSlabBase + m * kTS + ((c & 4) ? kTS : 0));
    const int uc = (c & 1) ? ue : u0, vc = (c & 2) ? ve : v0;
    const float dx = fmaf(float(uc), vp.Eux, vp.D0x);
    const float dy = fmaf(float(uc), vp.Euy, vp.D0y);
    const float dz = fmaf(float(vc), vp.Evz, vp.D0z);
    float ce, cz;
    if (DOM) {
      const float wy = (plane - gc.by) / gc.ky;
      const float t = (wy - vp.Sy) / dy;
      ce = fmaf(vp.Sx + t * dx, gc.kx, gc.bx);
      cz = fmaf(t * dz, gc.kz, gc.bz);
    } else {
      const float wx = (plane - gc.bx) / gc.kx;
      const float t = (wx - vp.Sx) / dx;
      ce = fmaf(vp.Sy + t * dy, gc.ky, gc.by);
      cz = fmaf(t * dz, gc.kz, gc.bz);
    }
    // Clamp before the int conversion so that far-away planes stay finite.
    ce = fminf(fmaxf(ce, -1.0e6f), 1.0e6f);
    cz = fminf(fmaxf(cz, -1.0e6f), 1.0e6f);
    atomicMin(&sh.emin[i], int(floorf(ce)));
    atomicMax(&sh.emax[i], int(floorf(ce)));
    atomicMin(&sh.zmin[i], int(floorf(cz)));
    atomicMax(&sh.zmax[i], int(floorf(cz)));
  }
  __syncthreads();

  const int BX = box.bx, BY = box.by, BZ = box.bz, BXY = BX * BY;
  const uint32_t box_bytes = uint32_t(BX * BY * BZ * sizeof(V));
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  // Box origin of slab i, in memory order (x, y, z).
  auto origin = [&](int i, int& ox, int& oy, int& oz) {
    const int m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int sm = kSlabBase + m * kTS;
    const int ii = m - mlo;
    const int e0 = sh.emin[ii] - 1;
    oz = sh.zmin[ii] - 1;
    // x (innermost) coordinates of a TMA box start on a 16-byte boundary.
    if (DOM) { ox = e0 & ~7; oy = sm; }
    else { ox = sm & ~7; oy = e0; }
  };
  auto issue = [&](int i) {
    int ox, oy, oz;
    origin(i, ox, oy, oz);
    uint64_t* bar = &sh.bars[i % kNStage];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(smem_raw + (i % kNStage) * stage_stride, map, ox, oy, oz, bar);
  };
  if (tid == 0) {
    for (int i = 0; i < min(kNStage, nslab); ++i) issue(i);
  }

  float acc = 0.f;
  int k = 0;
  int bad = 0;
  int done = 0;  // slabs whose barrier completed
  for (int i = 0; i < nslab; ++i) {
    const int slot = i % kNStage;
    const bool ok = mbar_wait_bounded(&sh.bars[slot], (i / kNStage) & 1, kWaitLimit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); sh.abort_flag = 1; }
      break;
    }
    done = i + 1;
    int ox, oy, oz;
    origin(i, ox, oy, oz);
    const int m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int ii = m - mlo;
    if (CHECK && tid == 0) {
      // The footprint must fit the box: emax + 2 (footprint + margin) inside.
      const int eext = DOM ? (sh.emax[ii] + 2 - ox) : (sh.emax[ii] + 2 - oy);
      const int zext = sh.zmax[ii] + 2 - oz;
      if (eext >= (DOM ? BX : BY) || zext >= BZ) atomicAdd(&flags[0], 1);
    }
    if (hit) {
      const V* s = reinterpret_cast<const V*>(smem_raw + slot * stage_stride);
      const float lo = float(kSlabBase + m * kTS), hi = lo + float(kTS);
      const float fox = float(ox), foy = float(oy), foz = float(oz);
      while (k < gc.N) {
        const float kf = float(k);
        const float cd = fmaf(kf, dcd, c0d);
        const float fd = floorf(cd);
        if (vp.dsgn > 0 ? (fd >= hi) : (fd < lo)) break;
        const float cx = DOM ? fmaf(kf, r.dcx, r.c0x) : cd;
        const float cy = DOM ? cd : fmaf(kf, r.dcy, r.c0y);
        const float cz = fmaf(kf, r.dcz, r.c0z);
        acc += tri_box<V, CHECK>(s, BX, BXY, BX - 2, BY - 2, BZ - 2, cx - fox, cy - foy, cz - foz, bad);
        ++k;
      }
    }
    __syncthreads();
    if (tid == 0 && i + kNStage < nslab) {
      fence_proxy_async();
      issue(i + kNStage);
    }
  }
  if (sh.abort_flag && tid == 0) {
    // Drain loads still in flight (bounded) before the CTA exits.
    for (int i = done; i < min(done + kNStage, nslab); ++i)
      (void)mbar_wait_bounded(&sh.bars[i % kNStage], (i / kNStage) & 1, kWaitLimit);
  }
  if (CHECK) {
    if (hit && k != gc.N) bad = 1;  // every sample of a hit ray must be consumed
    if (bad) atomicAdd(&flags[0], 1);
  }

  float val = 0.f;
  if (hit) {
    val = acc * r.delta;
  } else if (active) {
    int k0, k1;
    if (grown_range(vp, gc, u, v, r, k0, k1)) val = march_global(vol, gc, r, k0, k1) * r.delta;
  }
  fwd_epilogue(o, gc, vp, p, u, v, active, val, sh.red, tid);
}

template <class V, bool CHECK>
__global__ void __launch_bounds__(256) fwd_slab_kernel(const __grid_constant__ CUtensorMap map_x,
                                                       const __grid_constant__ CUtensorMap map_y,
                                                       const V* __restrict__ vol,
                                                       const ViewParams* __restrict__ views,
                                                       GridConst gc, SlabBox box_x, SlabBox box_y,
                                                       FwdOut o, int* flags) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ SlabShared sh;
  // TMA destinations are 128-byte aligned (128 extra bytes are requested).
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  const ViewParams vp = views[blockIdx.z];
  if (vp.dom)
    slab_body<V, 1, CHECK>(&map_y, vol, vp, gc, box_y, o, flags, smem_raw, sh);
  else
    slab_body<V, 0, CHECK>(&map_x, vol, vp, gc, box_x, o, flags, smem_raw, sh);
}

// ------------------------------------------------------------------ host
size_t dtype_size(cbct_dtype dt) { return dt == CBCT_F32 ? 4 : 2; }

CUtensorMapDataType tma_dtype(cbct_dtype dt) {
  switch (dt) {
    case CBCT_F32: return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    case CBCT_F16: return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    default: return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  }
}

CUtensorMap make_map(const cbct_plan* p, cbct_dtype dt, const void* vol, const SlabBox& b) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const size_t es = dtype_size(dt);
  cuuint64_t dims[3] = {(cuuint64_t)p->g.nx, (cuuint64_t)p->g.ny, (cuuint64_t)p->g.nz};
  cuuint64_t strides[2] = {(cuuint64_t)p->g.nx * es, (cuuint64_t)p->g.nx * p->g.ny * es};
  cuuint32_t box[3] = {(cuuint32_t)b.bx, (cuuint32_t)b.by, (cuuint32_t)b.bz};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult res = tensor_map_encoder()(&m, tma_dtype(dt), 3, const_cast<void*>(vol), dims, strides, box,
                                      estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                                      CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (res != CUDA_SUCCESS)
    throw Error(CBCT_ERR_CUDA, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)res));
  return m;
}

template <class V>
void launch_typed(cbct_plan* p, int s, const void* vol_v, const FwdOut& o, cudaStream_t st,
                  cbct_dtype dt, bool use_slab) {
  const V* vol = static_cast<const V*>(vol_v);
  const int first = p->first[s], cnt = p->count[s];
  dim3 grid((p->g.width + kTU - 1) / kTU, (p->g.height + kTV - 1) / kTV, cnt);
  if (use_slab) {
    const CUtensorMap mx = make_map(p, dt, vol, p->slab[0]);
    const CUtensorMap my = make_map(p, dt, vol, p->slab[1]);
    const size_t es = sizeof(V);
    auto stage_bytes = [&](const SlabBox& b) { return ((b.bx * b.by * b.bz * es) + 127) & ~size_t(127); };
    const size_t smem = kNStage * std::max(stage_bytes(p->slab[0]), stage_bytes(p->slab[1])) + 128;
    if (p->debug_checks) {
      auto k = fwd_slab_kernel<V, true>;
      ensure_smem_attr((const void*)k, smem);
      k<<<grid, 256, smem, st>>>(mx, my, vol, p->d_views + first, p->gc, p->slab[0], p->slab[1], o,
                                 p->d_flags);
    } else {
      auto k = fwd_slab_kernel<V, false>;
      ensure_smem_attr((const void*)k, smem);
      k<<<grid, 256, smem, st>>>(mx, my, vol, p->d_views + first, p->gc, p->slab[0], p->slab[1], o,
                                 p->d_flags);
    }
    check_launch("fwd_slab_kernel");
  } else {
    fwd_gather_kernel<V><<<grid, 256, 0, st>>>(vol, p->d_views + first, p->gc, o);
    check_launch("fwd_gather_kernel");
  }
}

}  // namespace

// Chooses the slab variant and its TMA box sizes from the plan geometry: for
// every view and tile, the footprint of every slab (corner-ray bounding box,
// computed in FP64) sets the maximum box extent, plus a safety margin.
void forward_choose_variant(cbct_plan* p) {
  const cbct_geometry& g = p->g;
  p->fwd_variant = 0;
  p->slab[0] = p->slab[1] = SlabBox{0, 0, 0, 0};
  if (p->force_gather) return;
  const double kx = g.nx / (double)g.lx, ky = g.ny / (double)g.ly, kz = g.nz / (double)g.lz;
  const double bx = g.nx / 2.0 - 0.5, by = g.ny / 2.0 - 0.5, bz = g.nz / 2.0 - 0.5;
  int ext_e[2] = {0, 0}, ext_z[2] = {0, 0};
  bool ok = true;
  const int tiles_u = (g.width + kTU - 1) / kTU, tiles_v = (g.height + kTV - 1) / kTV;
  for (int iv = 0; iv < p->n_views && ok; ++iv) {
    const ViewParams& vp = p->hviews[iv];
    const int dom = vp.dom;
    const int Nd = dom ? g.ny : g.nx;
    const int nsl = (Nd + 1 - kSlabBase + kTS - 1) / kTS + 1;
    if (nsl > kMaxSlabs) { ok = false; break; }
    // Direction sign must be uniform over the view (checked at all corners).
    for (int tu = 0; tu < tiles_u; ++tu) {
      const int u0 = tu * kTU, ue = std::min(u0 + kTU, g.width) - 1;
      for (int tv = 0; tv < tiles_v; ++tv) {
        const int v0 = tv * kTV, ve = std::min(v0 + kTV, g.height) - 1;
        double cd[4][3];
        for (int c = 0; c < 4; ++c) {
          const int uc = (c & 1) ? ue : u0, vc = (c & 2) ? ve : v0;
          cd[c][0] = vp.D0x + uc * (double)vp.Eux;
          cd[c][1] = vp.D0y + uc * (double)vp.Euy;
          cd[c][2] = vp.D0z + vc * (double)vp.Evz;
          const double dd = cd[c][dom], de = cd[c][1 - dom];
          if (dd * vp.dsgn < 0.25 * std::fabs(de) || dd * vp.dsgn <= 0) ok = false;
        }
        if (!ok) break;
        for (int m = 0; m < nsl; ++m) {
          double emn = 1e30, emx = -1e30, zmn = 1e30, zmx = -1e30;
          for (int c = 0; c < 8; ++c) {
            const double plane = kSlabBase + m * kTS + ((c & 4) ? kTS : 0);
            const double* d = cd[c & 3];
            double ce, cz;
            if (dom) {
              const double t = ((plane - by) / ky - vp.Sy) / d[1];
              ce = (vp.Sx + t * d[0]) * kx + bx;
              cz = t * d[2] * kz + bz;
            } else {
              const double t = ((plane - bx) / kx - vp.Sx) / d[0];
              ce = (vp.Sy + t * d[1]) * ky + by;
              cz = t * d[2] * kz + bz;
            }
            emn = std::min(emn, ce); emx = std::max(emx, ce);
            zmn = std::min(zmn, cz); zmx = std::max(zmx, cz);
          }
          // elements from floor(min)-1 to floor(max)+1 inclusive, +2 margin
          const int ee = (int)(std::floor(emx) - std::floor(emn)) + 3 + 2;
          const int ez = (int)(std::floor(zmx) - std::floor(zmn)) + 3 + 2;
          ext_e[dom] = std::max(ext_e[dom], ee);
          ext_z[dom] = std::max(ext_z[dom], std::min(ez, g.nz + 4));
        }
      }
      if (!ok) break;
    }
  }
  if (!ok) return;
  // Box x starts are rounded down to a multiple of 8 elements (16 bytes for
  // 16-bit storage, 32 for fp32), which widens the x extent by up to 7.
  auto rup = [](int v, int a) { return (v + a - 1) / a * a; };
  SlabBox bxd{rup(kTS + 1 + 7, 8), ext_e[0], ext_z[0], 1};   // x-dominant: x is the slab axis
  SlabBox byd{rup(ext_e[1] + 7, 8), kTS + 1, ext_z[1], 1};
  for (SlabBox* b : {&bxd, &byd}) {
    if (b->by < 2) b->by = 2;
    if (b->bz < 2) b->bz = 2;
    if (b->bx > 256 || b->by > 256 || b->bz > 256) ok = false;
  }
  const size_t stage = std::max((size_t)bxd.bx * bxd.by * bxd.bz, (size_t)byd.bx * byd.by * byd.bz) * 4;
  const size_t smem = kNStage * ((stage + 127) & ~size_t(127)) + 128;
  if (!ok || smem > (size_t)kSmemBudget) return;
  p->slab[0] = bxd;
  p->slab[1] = byd;
  p->slab_smem = smem;
  p->fwd_variant = 1;
}

void forward_prepare(cbct_plan* p) {
  if (p->fwd_variant != 1) return;
  const size_t smem32 = p->slab_smem;
  ensure_smem_attr((const void*)fwd_slab_kernel<float, false>, smem32);
  ensure_smem_attr((const void*)fwd_slab_kernel<float, true>, smem32);
  ensure_smem_attr((const void*)fwd_slab_kernel<__half, false>, smem32);
  ensure_smem_attr((const void*)fwd_slab_kernel<__half, true>, smem32);
  ensure_smem_attr((const void*)fwd_slab_kernel<__nv_bfloat16, false>, smem32);
  ensure_smem_attr((const void*)fwd_slab_kernel<__nv_bfloat16, true>, smem32);
}

void forward_launch(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out, const float* b,
                    float scale, int mode, int apply_offset, int accumulate, double* norm2_out,
                    cudaStream_t st) {
  forward_launch_ex(p, s, dt, vol, out, b, nullptr, scale, mode, apply_offset, accumulate, norm2_out, st);
}

void forward_launch_ex(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out, const float* b,
                       const float* pw, float scale, int mode, int apply_offset, int accumulate,
                       double* norm2_out, cudaStream_t st) {
  FwdOut o;
  o.out = out;
  o.pw = pw;
  o.b = b;
  o.scale = scale;
  o.mode = mode;
  o.apply_offset = apply_offset;
  o.accumulate = accumulate;
  o.partials = nullptr;
  const int cnt = p->count[s];
  if (cnt == 0) return;
  const size_t nblocks = (size_t)((p->g.width + kTU - 1) / kTU) * ((p->g.height + kTV - 1) / kTV) * cnt;
  if (norm2_out) {
    if (nblocks > p->n_partials) throw Error(CBCT_ERR_INTERNAL, "partials buffer too small");
    o.partials = p->d_partials;
  }
  const size_t es = dtype_size(dt);
  bool use_slab = p->fwd_variant == 1 && ((p->g.nx * es) % 16 == 0) &&
                  (reinterpret_cast<uintptr_t>(vol) % 16 == 0);
  switch (dt) {
    case CBCT_F32: launch_typed<float>(p, s, vol, o, st, dt, use_slab); break;
    case CBCT_F16: launch_typed<__half>(p, s, vol, o, st, dt, use_slab); break;
    case CBCT_BF16: launch_typed<__nv_bfloat16>(p, s, vol, o, st, dt, use_slab); break;
    default: throw Error(CBCT_ERR_INVALID_ARGUMENT, "unknown volume dtype");
  }
  if (norm2_out) finalize_partials(p->d_partials, (int)nblocks, norm2_out, st);
}

}  // namespace cbct
