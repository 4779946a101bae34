// forward.cu -- cone-beam forward projector (mult_M) for sm_100a.
//
// Semantics: conebeam_forwards_projection_kernel (xray/conebeam_projection.cu:412-528):
// one ray per detector pixel from the source to the pixel centre, clipped to
// the volume box, N = (int)(spp*nx) equidistant samples from the entry point,
// trilinear interpolation with border 0, result scaled by the sample spacing.
// Interpolation here is FP32 in software (not 9-bit texture weights).
//
// Variants (all but the gather kernel give bitwise equal results):
//  * fwd_slab_kernel: a CTA marches a 16x16 tile of rays of one view through
//    the volume in slabs of kTS voxels along the view's dominant in-plane
//    axis.  Each slab's footprint (the box around the tile's ray pyramid) is
//    staged into shared memory by a 3-D TMA load; out-of-volume texels arrive
//    as zeros (the border rule for free).  Views whose rays run mostly along x
//    read an x/y-transposed copy of the volume, so every slab is a range of
//    memory rows and the box is never padded along its slab axis.  Samples are
//    taken in ray order, so each ray's sum has the reference's summation
//    order.  Pairs of lerps run as packed FP32 (FFMA2).
//  * fwd_pair_kernel / fwd_quad_kernel: the same slabs, but one thread marches
//    two or four vertically adjacent rays of a detector column that share
//    their in-plane sample positions, interpolating them in e and d once.  A
//    plan takes the quad kernel where adjacent rows stay under 0.66 z texel
//    apart, the pair kernel under 0.99, else the slab kernel.
//  * fwd_fan_kernel (opt-in): the in-plane sharing across a whole column,
//    through shared-memory lines.
//  * fwd_gather_kernel: the same arithmetic with bounds-checked global loads,
//    used when the geometry does not fit the slab boxes or the volume pitch is
//    not TMA-aligned.
#include <climits>
#include <cmath>
#include <cstring>
#include <type_traits>

#include "device_common.cuh"

namespace cbct {

namespace {

enum { kModeStore = 0, kModeResidual = 1, kModeRecip = 2 };

struct FwdOut {
  float* out;            // projections of the subset (W,H,P_s)
  const void* b;         // measured projections (residual mode; NULL reads as 0)
  int b_dtype;           // storage type of b (cbct_dtype)
  const float* pw;       // per-pixel weight (residual mode; nullable)
  float scale;           // residual scale
  int mode;
  int apply_offset;      // residual mode: multiply by the sin^2 Wang weight
  int accumulate;        // store mode: out += result
  double* partials;      // residual mode: per-block sum of squares (nullable)
  const float* wproj;    // projection weights of the subset (CBSubsetWeightOperator; nullable)
};


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

// Output of one ray (store, reciprocal or weighted residual); returns the
// squared residual (residual mode) for the block's partial sum.
__device__ __forceinline__ double fwd_store(const FwdOut& o, const GridConst& gc, const ViewParams& vp, int p,
                                            int u, int v, float val) {
  double sq = 0.0;
  const size_t idx = ((size_t)p * gc.H + v) * gc.W + u;
  // CBSubsetWeightOperator: mult_M multiplies the projection by w, and mult_MH
  // of the residual weights its input by w again (CBSubsetWeightOperator.h:32-49).
  const float wp = o.wproj ? o.wproj[idx] : 1.f;
  val *= wp;
  if (o.mode == kModeStore) {
    o.out[idx] = o.accumulate ? o.out[idx] + val : val;
  } else if (o.mode == kModeRecip) {
    o.out[idx] = 1.f / fmaxf(val, 1e-6f);
  } else {
    const float d = o.b ? val - ld_any(o.b, idx, o.b_dtype) : val;
    sq = double(d) * double(d);
    float w = o.scale * wp;
    if (o.pw) w *= o.pw[idx];
    if (o.apply_offset) w *= offset_weight_full(gc.fov_u, gc.W, u, vp.ox);
    o.out[idx] = d * w;
  }
  return sq;
}

// Index of a CTA of a one-scan launch in launch order (x fastest).
__device__ __forceinline__ size_t launch_block_id() {
  return ((size_t)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
}

// Tile of one CTA: detector tile (x, y) of view z of the call, and its index
// among the call's tiles in launch order (its partial-sum slot).
struct TileId {
  int x, y, z;
  size_t bid;
};

__device__ __forceinline__ TileId launch_tile() {
  return TileId{int(blockIdx.x), int(blockIdx.y), int(blockIdx.z), launch_block_id()};
}

// Deterministic block sum of sq; one partial per block in launch order.
__device__ __forceinline__ void fwd_block_partial(const FwdOut& o, double sq, double* sh_red, int tid,
                                                  size_t bid) {
  if (o.partials != nullptr) {
    double t = warp_sum(sq);
    const int w = tid >> 5, l = tid & 31;
    if (l == 0) sh_red[w] = t;
    __syncthreads();
    if (tid < 32) {
      double q = (l < (int)(blockDim.x * blockDim.y) / 32) ? sh_red[l] : 0.0;
      q = warp_sum(q);
      if (tid == 0) o.partials[bid] = q;
    }
  }
}

// Epilogue shared by the per-ray variants.  All threads of the block must call it.
__device__ __forceinline__ void fwd_epilogue(const FwdOut& o, const GridConst& gc, const ViewParams& vp,
                                             int p, int u, int v, bool active, float val,
                                             double* sh_red, int tid, size_t bid) {
  const double sq = active ? fwd_store(o, gc, vp, p, u, v, val) : 0.0;
  fwd_block_partial(o, sq, sh_red, tid, bid);
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
  fwd_epilogue(o, gc, vp, p, u, v, active, val, sh_red, tid, launch_block_id());
}

// ------------------------------------------------------------------ transpose
// volT[k][i][j] = vol[k][j][i]: the volume seen with x and y exchanged.
template <class V>
__device__ __forceinline__ void transpose_tile(const V* __restrict__ in, V* __restrict__ out, int nx, int ny, int bx,
                                               int by, int bz, V (&tile)[32][33]) {
  const size_t plane = (size_t)nx * ny;
  const V* src = in + bz * plane;
  V* dst = out + bz * plane;
  const int x0 = bx * 32, y0 = by * 32;
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int x = x0 + threadIdx.x, y = y0 + j;
    if (x < nx && y < ny) tile[j][threadIdx.x] = src[(size_t)y * nx + x];
  }
  __syncthreads();
  for (int j = threadIdx.y; j < 32; j += blockDim.y) {
    const int y = y0 + threadIdx.x, x = x0 + j;
    if (x < nx && y < ny) dst[(size_t)x * ny + y] = tile[threadIdx.x][j];
  }
}

template <class V>
__global__ void transpose_xy_kernel(const V* __restrict__ in, V* __restrict__ out, int nx, int ny) {
  __shared__ V tile[32][33];
  transpose_tile<V>(in, out, nx, ny, blockIdx.x, blockIdx.y, blockIdx.z, tile);
}

// x/y transposes of many scans' volumes in one launch: one CTA per 32x32 tile
// of one plane of one scan, scans numbered in order.
struct TransposeRec {
  const float* in;
  float* out;
  int nx, ny;
  int tx, ty;            // tiles per plane (x, y)
  int base;              // index of the scan's first CTA
};

__global__ void transpose_multi_kernel(const TransposeRec* __restrict__ recs, int n_recs) {
  __shared__ float tile[32][33];
  int lo = 0, hi = n_recs - 1;
  const int t = blockIdx.x;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (recs[mid].base <= t) lo = mid;
    else hi = mid - 1;
  }
  const TransposeRec& R = recs[lo];
  int l = t - R.base;
  const int bx = l % R.tx;
  l /= R.tx;
  transpose_tile<float>(R.in, R.out, R.nx, R.ny, bx, l % R.ty, l / R.ty, tile);
}

// ------------------------------------------------------------------ slab/TMA
struct SlabShared {
  uint64_t bars[kNStage];
  int mlo, mhi, abort_flag;
  int emin[kMaxSlabs], emax[kMaxSlabs], zmin[kMaxSlabs], zmax[kMaxSlabs];
  double red[8];
};

// Packed lerp of two pairs: a + t (b - a) as (a - t a) + t b.
__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 t) {
  const float2 nt = make_float2(-t.x, -t.y);
  return __ffma2_rn(t, b, __ffma2_rn(nt, a, a));
}

// Samples of one ray inside one slab.  (ce, cd, cz) are frame texel
// coordinates; the box origin is (oe, od, oz); BX and BY are the box
// strides.  Consumes samples while floor(cd) stays inside the slab.
template <class V, int BX, int BY = kBoxY>
struct SlabSample {
  static constexpr int BXY = BX * BY;
  // Trilinear value of one sample whose frame coordinates are (ced.x, ced.y, cz)
  // and whose floors are (fe, fd, fz).  cmo = 1.5 * 2^23 - (box origin index):
  // the element index comes out of the mantissa of an exact sum.
  static __device__ __forceinline__ float eval(const V* __restrict__ s, float2 ced, float cz, float fe, float fd,
                                               float fz, float cmo, unsigned maxidx, int& bad, bool check) {
    const float2 aed = __fadd2_rn(ced, make_float2(-fe, -fd));
    const float az = cz - fz;
    const int idx0 = int_of_biased(fmaf(fz, float(BXY), fmaf(fd, float(BX), fe)) + cmo);
    if (check) bad |= (unsigned)idx0 > maxidx;
    const unsigned idx = min((unsigned)idx0, maxidx);
    const V* q = s + idx;
    const float2 a0 = make_float2(sm_f(q[0]), sm_f(q[BX]));              // (e0,d0,z0) (e0,d1,z0)
    const float2 b0 = make_float2(sm_f(q[1]), sm_f(q[BX + 1]));          // (e1,d0,z0) (e1,d1,z0)
    const float2 a1 = make_float2(sm_f(q[BXY]), sm_f(q[BXY + BX]));      // z1
    const float2 b1 = make_float2(sm_f(q[BXY + 1]), sm_f(q[BXY + BX + 1]));
    const float2 te = make_float2(aed.x, aed.x);
    const float2 e0 = lerp2(a0, b0, te);   // z0: (d0, d1)
    const float2 e1 = lerp2(a1, b1, te);   // z1: (d0, d1)
    const float2 dz = lerp2(make_float2(e0.x, e1.x), make_float2(e0.y, e1.y), make_float2(aed.y, aed.y));
    return fmaf(az, dz.y - dz.x, dz.x);
  }
};

// Samples of one ray inside one slab.  The number of samples the slab holds
// is found first (the first k whose d coordinate leaves the slab; d is
// monotone along the ray), then they are taken in a counted loop, kFwdUnroll
// independent evaluations per iteration, added to acc in ray order.
// (ce, cd, cz) are frame texel coordinates.
constexpr int kFwdUnroll = 2;

template <class V, int BX, int SGN, bool CHECK, int BY = kBoxY>
__device__ __forceinline__ void slab_samples(const V* __restrict__ s, float& kf, float Nf, float ce0, float cd0,
                                             float cz0, float dce, float dcd, float idcd, float dcz, float lo,
                                             float hi, float cmo, unsigned maxidx, float& acc, int& bad) {
  using SS = SlabSample<V, BX, BY>;
  const float2 c0 = make_float2(ce0, cd0), dc = make_float2(dce, dcd);
  // floor(x) >= hi <=> x >= hi and floor(x) < lo <=> x < lo, lo and hi being integers.
  auto out_at = [&](float k) {
    const float x = fmaf(k, dcd, cd0);
    return SGN > 0 ? (x >= hi) : (x < lo);
  };
  // Estimate (idcd = 1 / dcd), then the exact boundary: out_at is monotone in k.
  float ke = ceilf(((SGN > 0 ? hi : lo) - cd0) * idcd);
  ke = fminf(fmaxf(ke, kf), Nf);
  while (ke > kf && out_at(ke - 1.f)) ke -= 1.f;
  while (ke < Nf && !out_at(ke)) ke += 1.f;
  float k = kf;
  for (; k + float(kFwdUnroll - 1) < ke; k += float(kFwdUnroll)) {
    float v[kFwdUnroll];
#pragma unroll
    for (int q = 0; q < kFwdUnroll; ++q) {
      const float kq = k + float(q);
      const float2 pq = __ffma2_rn(make_float2(kq, kq), dc, c0);
      const float czq = fmaf(kq, dcz, cz0);
      v[q] = SS::eval(s, pq, czq, floor_small(pq.x), floor_small(pq.y), floor_small(czq), cmo, maxidx, bad, CHECK);
    }
#pragma unroll
    for (int q = 0; q < kFwdUnroll; ++q) acc += v[q];
  }
  for (; k < ke; k += 1.f) {
    const float2 pq = __ffma2_rn(make_float2(k, k), dc, c0);
    const float czq = fmaf(k, dcz, cz0);
    acc += SS::eval(s, pq, czq, floor_small(pq.x), floor_small(pq.y), floor_small(czq), cmo, maxidx, bad, CHECK);
  }
  kf = ke;
}

// 16-bit boxes take half the shared memory, so those instantiations ask for a
// register budget that lets four CTAs share an SM.
template <class V>
constexpr int slab_min_blocks() { return sizeof(V) == 4 ? 3 : 4; }

// One CTA of the slab kernel: ray tile `tile` of the call.  Shared by the
// one-scan kernel and the work-list kernel over many scans; smem_raw is the
// 128-byte aligned dynamic shared memory (TMA destinations).
template <class V, int BX, bool CHECK, int NS>
__device__ __forceinline__ void fwd_slab_body(const CUtensorMap* map_v, const CUtensorMap* map_t,
                                              const V* __restrict__ vol, const ViewParams* __restrict__ views,
                                              const GridConst& gc, int BZ, const FwdOut& o, int* flags,
                                              const TileId& tile, unsigned char* smem_raw, SlabShared& sh) {
  constexpr int BXY = BX * kBoxY;
  const ViewParams vp = views[tile.z];
  const int dom = vp.dom;
  const CUtensorMap* map = dom ? map_v : map_t;
  const int tid = threadIdx.x;
  const int p = tile.z;
  const int u0 = tile.x * kTU, v0 = tile.y * kTV;
  const int u = u0 + (tid % kTU), v = v0 + (tid / kTU);
  const bool active = (u < gc.W) && (v < gc.H);
  const Ray r = make_ray(vp, gc, min(u, gc.W - 1), min(v, gc.H - 1));
  const bool hit = active && (r.a2 > r.a1);
  // Frame coordinates: e = cross axis, d = slab axis (y for dom = 1, x for dom = 0).
  const float ce0 = dom ? r.c0x : r.c0y, dce = dom ? r.dcx : r.dcy;
  const float cd0 = dom ? r.c0y : r.c0x, dcd = dom ? r.dcy : r.dcx;
  const float idcd = 1.f / dcd;
  const float ke = dom ? gc.kx : gc.ky, be = dom ? gc.bx : gc.by;
  const float kd = dom ? gc.ky : gc.kx, bd = dom ? gc.by : gc.bx;
  const float Se = dom ? vp.Sx : vp.Sy, Sd = dom ? vp.Sy : vp.Sx;

  if (tid == 0) {
    sh.mlo = INT_MAX;
    sh.mhi = INT_MIN;
    sh.abort_flag = 0;
    for (int s = 0; s < NS; ++s) mbar_init(&sh.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (hit) {
    const int f0 = int(floorf(cd0));
    const int f1 = int(floorf(fmaf(float(gc.N - 1), dcd, cd0)));
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
  const int ne = dom ? gc.nx : gc.ny;  // volume extent along e
  for (int q = tid; q < nslab * 8; q += blockDim.x) {
    const int i = q >> 3, c = q & 7;
    const int m = mlo + i;
    const float plane = float(kSlabBase + m * kTS + ((c & 4) ? kTS : 0));
    const int uc = (c & 1) ? ue : u0, vc = (c & 2) ? ve : v0;
    const float dx = fmaf(float(uc), vp.Eux, vp.D0x);
    const float dy = fmaf(float(uc), vp.Euy, vp.D0y);
    const float dz = fmaf(float(vc), vp.Evz, vp.D0z);
    const float de = dom ? dx : dy, dd = dom ? dy : dx;
    const float t = ((plane - bd) / kd - Sd) / dd;
    float ce = fmaf(fmaf(t, de, Se), ke, be);
    float cz = fmaf(t * dz, gc.kz, gc.bz);
    // Clamp before the int conversion so that far-away planes stay finite.
    // Samples lie inside the volume (texel floors in [-1, n-1]; outside it the
    // border reads 0), so the box only has to cover the footprint's part in it.
    const int fe = min(max(int(floorf(fminf(fmaxf(ce, -1.0e5f), 1.0e5f))), -1), ne - 1);
    const int fz = min(max(int(floorf(fminf(fmaxf(cz, -1.0e5f), 1.0e5f))), -1), gc.nz - 1);
    atomicMin(&sh.emin[i], fe);
    atomicMax(&sh.emax[i], fe);
    atomicMin(&sh.zmin[i], fz);
    atomicMax(&sh.zmax[i], fz);
  }
  __syncthreads();

  const uint32_t box_bytes = uint32_t(BX * kBoxY * BZ * sizeof(V));
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  const unsigned maxidx = unsigned(BXY * (BZ - 1) - BX - 2);
  // Box origin of slab i (visiting order), frame/memory order (e, d, z).
  auto origin = [&](int i, int& oe, int& od, int& oz, int& m) {
    m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int ii = m - mlo;
    oe = (sh.emin[ii] - 1) & ~(int(16 / sizeof(V)) - 1);   // 16-byte aligned x start
    od = kSlabBase + m * kTS;
    oz = sh.zmin[ii] - 1;
  };
  auto issue = [&](int i) {
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    uint64_t* bar = &sh.bars[i % NS];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(smem_raw + (i % NS) * stage_stride, map, oe, od, oz, bar);
  };
  if (tid == 0) {
    for (int i = 0; i < min(NS, nslab); ++i) issue(i);
  }

  float acc = 0.f;
  float kf = 0.f;
  const float Nf = float(gc.N);
  int bad = 0;
  int done = 0;
  for (int i = 0; i < nslab; ++i) {
    const int slot = i % NS;
    const bool ok = mbar_wait_bounded(&sh.bars[slot], (i / NS) & 1, gc.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); sh.abort_flag = 1; }
      break;
    }
    done = i + 1;
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    if (CHECK && tid == 0) {
      // The footprint (max + 1) plus a one-voxel margin must fit in the box.
      const int ii = m - mlo;
      if (sh.emax[ii] + 2 - oe >= BX || sh.zmax[ii] + 2 - oz >= BZ) atomicAdd(&flags[0], 1);
    }
    if (hit) {
      const V* s = reinterpret_cast<const V*>(smem_raw + slot * stage_stride);
      const float lo = float(od), hi = lo + float(kTS);
      const float cmo = kRoundC - float(oe + od * BX + oz * BXY);
      if (vp.dsgn > 0)
        slab_samples<V, BX, 1, CHECK>(s, kf, Nf, ce0, cd0, r.c0z, dce, dcd, idcd, r.dcz, lo, hi, cmo, maxidx, acc,
                                        bad);
      else
        slab_samples<V, BX, -1, CHECK>(s, kf, Nf, ce0, cd0, r.c0z, dce, dcd, idcd, r.dcz, lo, hi, cmo, maxidx, acc,
                                         bad);
    }
    __syncthreads();
    if (tid == 0 && i + NS < nslab) {
      fence_proxy_async();
      issue(i + NS);
    }
  }
  if (sh.abort_flag && tid == 0) {
    // Drain loads still in flight (bounded) before the CTA exits.
    for (int i = done; i < min(done + NS, nslab); ++i)
      if (!mbar_wait_bounded(&sh.bars[i % NS], (i / NS) & 1, kWaitLimit)) sh.abort_flag = 2;
  }
  if (CHECK) {
    if (hit && kf != Nf) bad = 1;  // every sample of a hit ray must be consumed
    if (bad) atomicAdd(&flags[0], 1);
  }

  float val = 0.f;
  if (hit) {
    val = acc * r.delta;
  } else if (active) {
    int k0, k1;
    if (grown_range(vp, gc, u, v, r, k0, k1)) val = march_global(vol, gc, r, k0, k1) * r.delta;
  }
  fwd_epilogue(o, gc, vp, p, u, v, active, val, sh.red, tid, tile.bid);
}

template <class V, int BX, bool CHECK, int NS>
__global__ void __launch_bounds__(256, slab_min_blocks<V>()) fwd_slab_kernel(const __grid_constant__ CUtensorMap map_v,
                                                       const __grid_constant__ CUtensorMap map_t,
                                                       const V* __restrict__ vol,
                                                       const ViewParams* __restrict__ views, GridConst gc,
                                                       int BZ, FwdOut o, int* flags) {
  // TMA destinations are 128-byte aligned (128 extra bytes are requested).
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  __shared__ SlabShared sh;
  fwd_slab_body<V, BX, CHECK, NS>(&map_v, &map_t, vol, views, gc, BZ, o, flags, launch_tile(), smem_raw, sh);
}

// ------------------------------------------------------------------ row pairs
// Two vertically adjacent rays of one detector column lie in the column's
// vertical plane.  When both leave the volume through its side faces their
// clip (a1, a2) is the column's, so their k-th samples share the in-plane
// position (e_k, d_k) and differ only in z; when in addition their z
// coordinates differ by less than one texel at every sample (checked at both
// ends; the difference is linear in k), the lower ray's planes fz, fz + 1 and
// the upper ray's planes are among fz, fz + 1, fz + 2.  One thread then marches
// the pair: one e/d position, three planes interpolated in e and d (12 shared
// loads instead of 16), and each ray's own z lerp.  Every value is the one the
// slab kernel computes for that ray (same texels, same operations, same
// order), so results are bitwise equal.  Other pairs (rays clipped by the top
// or bottom face, or far apart in z) run slab_samples for each ray.
// The row-pair kernel keeps one TMA stage: with 16x16 tiles its box is small
// enough for six CTAs per SM, and the other CTAs' work covers each CTA's wait
// for its next slab (two stages would halve the CTAs per SM).
#ifndef CBCT_PAIR_STAGES
#define CBCT_PAIR_STAGES 1
#endif
constexpr int kPairStages = CBCT_PAIR_STAGES;
// Rows of a row-pair box (the slab's kTS + 1 rows, padded to kBoxY by default).
#ifndef CBCT_PAIR_BOXY
#define CBCT_PAIR_BOXY 10
#endif
constexpr int kPairBoxY = CBCT_PAIR_BOXY;

struct PairShared {
  uint64_t bars[kPairStages];
  int mlo, mhi, abort_flag;
  double red[8];
};

// One sample of a paired ray: (lower ray's value, upper ray's value).
template <class V, int BX, bool CHECK, int BY = kBoxY>
__device__ __forceinline__ float2 pair_eval(const V* __restrict__ s, float k, float2 c0, float2 dc, float zl0,
                                            float dzl, float zu0, float dzu, float cmo, unsigned maxidx,
                                            unsigned maxidx3, int& bad) {
  constexpr int BXY = BX * BY;
  const float2 pq = __ffma2_rn(make_float2(k, k), dc, c0);
  const float czl = fmaf(k, dzl, zl0), czu = fmaf(k, dzu, zu0);
  const float fe = floor_small(pq.x), fd = floor_small(pq.y), fzl = floor_small(czl), fzu = floor_small(czu);
  const float2 aed = __fadd2_rn(pq, make_float2(-fe, -fd));
  const int idx0 = int_of_biased(fmaf(fzl, float(BXY), fmaf(fd, float(BX), fe)) + cmo);
  const bool up = fzu != fzl;
  if (CHECK) bad |= ((unsigned)idx0 > maxidx) | (up && (unsigned)idx0 + 2u * BXY > maxidx3) | (fzu - fzl > 1.f);
  const V* q = s + min((unsigned)idx0, maxidx);
  const V* q2 = s + min((unsigned)idx0 + 2u * BXY, maxidx3);
  const float2 te = make_float2(aed.x, aed.x);
  const float2 e0 = lerp2(make_float2(sm_f(q[0]), sm_f(q[BX])), make_float2(sm_f(q[1]), sm_f(q[BX + 1])), te);
  const float2 e1 = lerp2(make_float2(sm_f(q[BXY]), sm_f(q[BXY + BX])),
                          make_float2(sm_f(q[BXY + 1]), sm_f(q[BXY + BX + 1])), te);
  const float2 e2 = lerp2(make_float2(sm_f(q2[0]), sm_f(q2[BX])), make_float2(sm_f(q2[1]), sm_f(q2[BX + 1])), te);
  // d lerps of planes fz, fz + 1 (packed) and fz + 2: the slab kernel's formula
  const float2 d01 = lerp2(make_float2(e0.x, e1.x), make_float2(e0.y, e1.y), make_float2(aed.y, aed.y));
  const float d2 = fmaf(aed.y, e2.y, fmaf(-aed.y, e2.x, e2.x));
  const float bl = up ? d01.y : d01.x, bh = up ? d2 : d01.y;
  return make_float2(fmaf(czl - fzl, d01.y - d01.x, d01.x), fmaf(czu - fzu, bh - bl, bl));
}

#ifndef CBCT_PAIR_UNROLL
#define CBCT_PAIR_UNROLL 1
#endif
constexpr int kPairUnroll = CBCT_PAIR_UNROLL;

// The pair's samples inside one slab (counted as in slab_samples), each ray's
// values added in ray order.
template <class V, int BX, int SGN, bool CHECK, int BY = kBoxY>
__device__ __forceinline__ void pair_samples(const V* __restrict__ s, float& kf, float Nf, float ce0, float cd0,
                                             float dce, float dcd, float idcd, float zl0, float dzl, float zu0,
                                             float dzu, float lo, float hi, float cmo, unsigned maxidx,
                                             unsigned maxidx3, float& accl, float& accu, int& bad) {
  const float2 c0 = make_float2(ce0, cd0), dc = make_float2(dce, dcd);
  auto out_at = [&](float k) {
    const float x = fmaf(k, dcd, cd0);
    return SGN > 0 ? (x >= hi) : (x < lo);
  };
  float ke = ceilf(((SGN > 0 ? hi : lo) - cd0) * idcd);
  ke = fminf(fmaxf(ke, kf), Nf);
  while (ke > kf && out_at(ke - 1.f)) ke -= 1.f;
  while (ke < Nf && !out_at(ke)) ke += 1.f;
  float k = kf;
  if (kPairUnroll > 1) {
    for (; k + float(kPairUnroll - 1) < ke; k += float(kPairUnroll)) {
      float2 v[kPairUnroll];
#pragma unroll
      for (int q = 0; q < kPairUnroll; ++q)
        v[q] = pair_eval<V, BX, CHECK, BY>(s, k + float(q), c0, dc, zl0, dzl, zu0, dzu, cmo, maxidx, maxidx3, bad);
#pragma unroll
      for (int q = 0; q < kPairUnroll; ++q) {
        accl += v[q].x;
        accu += v[q].y;
      }
    }
  }
  for (; k < ke; k += 1.f) {
    const float2 v = pair_eval<V, BX, CHECK, BY>(s, k, c0, dc, zl0, dzl, zu0, dzu, cmo, maxidx, maxidx3, bad);
    accl += v.x;
    accu += v.y;
  }
  kf = ke;
}

// CTAs per SM the register budget is sized for: 80 registers (no spills) at
// six 128-thread CTAs, as many as the fp32 boxes of 16x16 tiles leave room for.
template <class V>
constexpr int pair_min_blocks() {
#ifdef CBCT_PAIR_MINB
  return CBCT_PAIR_MINB;
#else
  return kPairThreads >= 256 ? 3 : 6;
#endif
}

// One CTA of the row-pair kernel (see fwd_slab_body).
template <class V, int BX, bool CHECK>
__device__ __forceinline__ void fwd_pair_body(const CUtensorMap* map_v, const CUtensorMap* map_t,
                                              const V* __restrict__ vol, const ViewParams* __restrict__ views,
                                              const GridConst& gc, int BZ, int nsl_max, const FwdOut& o,
                                              int* flags, const TileId& tile, unsigned char* smem_raw,
                                              PairShared& sh) {
  constexpr int BXY = BX * kPairBoxY;
  const ViewParams vp = views[tile.z];
  const int dom = vp.dom;
  const CUtensorMap* map = dom ? map_v : map_t;
  const int tid = threadIdx.x;
  const int p = tile.z;
  const int u0 = tile.x * kPU, v0 = tile.y * kPV;
  const int u = u0 + (tid % kPU), va = v0 + 2 * (tid / kPU), vb = va + 1;
  const bool act_a = (u < gc.W) && (va < gc.H), act_b = (u < gc.W) && (vb < gc.H);
  const int uc = min(u, gc.W - 1);
  const Ray ra = make_ray(vp, gc, uc, min(va, gc.H - 1));
  const Ray rb = make_ray(vp, gc, uc, min(vb, gc.H - 1));
  const bool hit_a = act_a && (ra.a2 > ra.a1), hit_b = act_b && (rb.a2 > rb.a1);
  const float ke_ = dom ? gc.kx : gc.ky, be = dom ? gc.bx : gc.by;
  const float kd = dom ? gc.ky : gc.kx, bd = dom ? gc.by : gc.bx;
  const float Se = dom ? vp.Sx : vp.Sy, Sd = dom ? vp.Sy : vp.Sx;
  // Frame coordinates (e = cross axis, d = slab axis) of both rays.
  const float ce0a = dom ? ra.c0x : ra.c0y, dcea = dom ? ra.dcx : ra.dcy;
  const float cd0a = dom ? ra.c0y : ra.c0x, dcda = dom ? ra.dcy : ra.dcx;
  const float ce0b = dom ? rb.c0x : rb.c0y, dceb = dom ? rb.dcx : rb.dcy;
  const float cd0b = dom ? rb.c0y : rb.c0x, dcdb = dom ? rb.dcy : rb.dcx;
  const float idcda = 1.f / dcda, idcdb = 1.f / dcdb;
  const float Nf = float(gc.N);
  // Pairing: same clip, z difference in (0, 1) texel at both ends (the lower
  // ray first).  The margins cover the rounding of the sample coordinates.
  bool paired = false, a_low = true;
  if (hit_a && hit_b && ra.a1 == rb.a1 && ra.a2 == rb.a2) {
    const float d0 = rb.c0z - ra.c0z;
    const float d1 = fmaf(Nf - 1.f, rb.dcz, rb.c0z) - fmaf(Nf - 1.f, ra.dcz, ra.c0z);
    const bool ab = d0 >= 2e-3f && d0 <= 0.998f && d1 >= 2e-3f && d1 <= 0.998f;
    const bool ba = d0 <= -2e-3f && d0 >= -0.998f && d1 <= -2e-3f && d1 >= -0.998f;
    paired = ab || ba;
    a_low = ab;
  }
  const float zl0 = a_low ? ra.c0z : rb.c0z, dzl = a_low ? ra.dcz : rb.dcz;
  const float zu0 = a_low ? rb.c0z : ra.c0z, dzu = a_low ? rb.dcz : ra.dcz;

  if (tid == 0) {
    sh.mlo = INT_MAX;
    sh.mhi = INT_MIN;
    sh.abort_flag = 0;
    for (int s = 0; s < kPairStages; ++s) mbar_init(&sh.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  {
    int mn = INT_MAX, mx = INT_MIN;
    if (hit_a) {
      const int m0 = (max(int(floorf(cd0a)), kSlabBase) - kSlabBase) / kTS;
      const int m1 = (max(int(floorf(fmaf(Nf - 1.f, dcda, cd0a))), kSlabBase) - kSlabBase) / kTS;
      mn = min(m0, m1);
      mx = max(m0, m1);
    }
    if (hit_b) {
      const int m0 = (max(int(floorf(cd0b)), kSlabBase) - kSlabBase) / kTS;
      const int m1 = (max(int(floorf(fmaf(Nf - 1.f, dcdb, cd0b))), kSlabBase) - kSlabBase) / kTS;
      mn = min(mn, min(m0, m1));
      mx = max(mx, max(m0, m1));
    }
    if (mn <= mx) {
      atomicMin(&sh.mlo, mn);
      atomicMax(&sh.mhi, mx);
    }
  }
  __syncthreads();
  const int mlo = sh.mlo, mhi = sh.mhi;
  int nslab = (mhi >= mlo) ? (mhi - mlo + 1) : 0;
  if (nslab > nsl_max) {
    if (tid == 0) atomicAdd(&flags[0], 1);
    nslab = 0;
  }
  // Per-slab footprints (e min, e max, z min, z max) after the boxes.
  const uint32_t box_bytes = uint32_t(BX * kPairBoxY * BZ * sizeof(V));
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  int* const emin = reinterpret_cast<int*>(smem_raw + kPairStages * stage_stride);
  int* const emax = emin + nsl_max;
  int* const zmin = emax + nsl_max;
  int* const zmax = zmin + nsl_max;
  for (int i = tid; i < nslab; i += blockDim.x) {
    emin[i] = INT_MAX; emax[i] = INT_MIN;
    zmin[i] = INT_MAX; zmax[i] = INT_MIN;
  }
  __syncthreads();
  // Footprint of every slab: the tile's four corner rays at the slab's two
  // bounding planes, clamped to the volume's texel range.
  const int ue = min(u0 + kPU, gc.W) - 1, ve = min(v0 + kPV, gc.H) - 1;
  const int ne = dom ? gc.nx : gc.ny;
  for (int q = tid; q < nslab * 8; q += blockDim.x) {
    const int i = q >> 3, c = q & 7;
    const int m = mlo + i;
    const float plane = float(kSlabBase + m * kTS + ((c & 4) ? kTS : 0));
    const int ucc = (c & 1) ? ue : u0, vcc = (c & 2) ? ve : v0;
    const float dx = fmaf(float(ucc), vp.Eux, vp.D0x);
    const float dy = fmaf(float(ucc), vp.Euy, vp.D0y);
    const float dz = fmaf(float(vcc), vp.Evz, vp.D0z);
    const float de = dom ? dx : dy, dd = dom ? dy : dx;
    const float t = ((plane - bd) / kd - Sd) / dd;
    const float ce = fmaf(fmaf(t, de, Se), ke_, be);
    const float cz = fmaf(t * dz, gc.kz, gc.bz);
    const int fe = min(max(int(floorf(fminf(fmaxf(ce, -1.0e5f), 1.0e5f))), -1), ne - 1);
    const int fz = min(max(int(floorf(fminf(fmaxf(cz, -1.0e5f), 1.0e5f))), -1), gc.nz - 1);
    atomicMin(&emin[i], fe);
    atomicMax(&emax[i], fe);
    atomicMin(&zmin[i], fz);
    atomicMax(&zmax[i], fz);
  }
  __syncthreads();

  const unsigned maxidx = unsigned(BXY * (BZ - 1) - BX - 2);   // two-plane loads stay in the box
  const unsigned maxidx3 = unsigned(BXY * BZ - BX - 2);        // the third plane's loads
  auto origin = [&](int i, int& oe, int& od, int& oz, int& m) {
    m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int ii = m - mlo;
    oe = (emin[ii] - 1) & ~(int(16 / sizeof(V)) - 1);   // 16-byte aligned x start
    od = kSlabBase + m * kTS;
    oz = zmin[ii] - 1;
  };
  auto issue = [&](int i) {
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    uint64_t* bar = &sh.bars[i % kPairStages];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(smem_raw + (i % kPairStages) * stage_stride, map, oe, od, oz, bar);
  };
  if (tid == 0) {
    for (int i = 0; i < min(kPairStages, nslab); ++i) issue(i);
  }

  float acca = 0.f, accb = 0.f;   // paired: lower / upper ray
  float kfa = 0.f, kfb = 0.f;     // paired: kfa is the pair's next sample
  int bad = 0;
  int done = 0;
  for (int i = 0; i < nslab; ++i) {
    const int slot = i % kPairStages;
    const bool ok = mbar_wait_bounded(&sh.bars[slot], (i / kPairStages) & 1, gc.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); sh.abort_flag = 1; }
      break;
    }
    done = i + 1;
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    if (CHECK && tid == 0) {
      const int ii = m - mlo;
      if (emax[ii] + 2 - oe >= BX || zmax[ii] + 2 - oz >= BZ) atomicAdd(&flags[0], 1);
    }
    const V* s = reinterpret_cast<const V*>(smem_raw + slot * stage_stride);
    const float lo = float(od), hi = lo + float(kTS);
    const float cmo = kRoundC - float(oe + od * BX + oz * BXY);
    constexpr int PY = kPairBoxY;
    if (paired) {
      if (vp.dsgn > 0)
        pair_samples<V, BX, 1, CHECK, PY>(s, kfa, Nf, ce0a, cd0a, dcea, dcda, idcda, zl0, dzl, zu0, dzu, lo, hi,
                                          cmo, maxidx, maxidx3, acca, accb, bad);
      else
        pair_samples<V, BX, -1, CHECK, PY>(s, kfa, Nf, ce0a, cd0a, dcea, dcda, idcda, zl0, dzl, zu0, dzu, lo, hi,
                                           cmo, maxidx, maxidx3, acca, accb, bad);
    } else {
      if (hit_a) {
        if (vp.dsgn > 0)
          slab_samples<V, BX, 1, CHECK, PY>(s, kfa, Nf, ce0a, cd0a, ra.c0z, dcea, dcda, idcda, ra.dcz, lo, hi, cmo,
                                            maxidx, acca, bad);
        else
          slab_samples<V, BX, -1, CHECK, PY>(s, kfa, Nf, ce0a, cd0a, ra.c0z, dcea, dcda, idcda, ra.dcz, lo, hi, cmo,
                                             maxidx, acca, bad);
      }
      if (hit_b) {
        if (vp.dsgn > 0)
          slab_samples<V, BX, 1, CHECK, PY>(s, kfb, Nf, ce0b, cd0b, rb.c0z, dceb, dcdb, idcdb, rb.dcz, lo, hi, cmo,
                                            maxidx, accb, bad);
        else
          slab_samples<V, BX, -1, CHECK, PY>(s, kfb, Nf, ce0b, cd0b, rb.c0z, dceb, dcdb, idcdb, rb.dcz, lo, hi, cmo,
                                             maxidx, accb, bad);
      }
    }
    __syncthreads();
    if (tid == 0 && i + kPairStages < nslab) {
      fence_proxy_async();
      issue(i + kPairStages);
    }
  }
  if (sh.abort_flag && tid == 0) {
    for (int i = done; i < min(done + kPairStages, nslab); ++i)
      if (!mbar_wait_bounded(&sh.bars[i % kPairStages], (i / kPairStages) & 1, kWaitLimit)) sh.abort_flag = 2;
  }
  if (CHECK) {
    // every sample of a hit ray must be consumed
    if (paired ? kfa != Nf : ((hit_a && kfa != Nf) || (hit_b && kfb != Nf))) bad = 1;
    if (bad) atomicAdd(&flags[0], 1);
  }
  float vala = 0.f, valb = 0.f;
  if (paired) {
    vala = (a_low ? acca : accb) * ra.delta;
    valb = (a_low ? accb : acca) * rb.delta;
  } else {
    int k0, k1;
    if (hit_a) vala = acca * ra.delta;
    else if (act_a && grown_range(vp, gc, u, va, ra, k0, k1)) vala = march_global(vol, gc, ra, k0, k1) * ra.delta;
    if (hit_b) valb = accb * rb.delta;
    else if (act_b && grown_range(vp, gc, u, vb, rb, k0, k1)) valb = march_global(vol, gc, rb, k0, k1) * rb.delta;
  }
  double sq = 0.0;
  if (act_a) sq += fwd_store(o, gc, vp, p, u, va, vala);
  if (act_b) sq += fwd_store(o, gc, vp, p, u, vb, valb);
  fwd_block_partial(o, sq, sh.red, tid, tile.bid);
}

template <class V, int BX, bool CHECK>
__global__ void __launch_bounds__(kPairThreads, pair_min_blocks<V>())
    fwd_pair_kernel(const __grid_constant__ CUtensorMap map_v, const __grid_constant__ CUtensorMap map_t,
                    const V* __restrict__ vol, const ViewParams* __restrict__ views, GridConst gc, int BZ,
                    int nsl_max, FwdOut o, int* flags) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  __shared__ PairShared sh;
  fwd_pair_body<V, BX, CHECK>(&map_v, &map_t, vol, views, gc, BZ, nsl_max, o, flags, launch_tile(), smem_raw, sh);
}

// ------------------------------------------------------------------ row quads
// The row-pair argument for four adjacent rows of a column: when all four rays
// leave through the side faces (one clip) and, sorted by z, each lies less
// than two texels above the lowest at both ends of the ray (the second-lowest
// less than one), their planes are among the lowest ray's fz .. fz + 3.  One thread marches the quad: one e/d
// position, four planes interpolated in e and d (16 shared loads for four
// samples), each ray's own z lerp on its two planes.  Values are the slab
// kernel's for every ray, so results are bitwise equal.  Quads that do not
// qualify run as two pairs (or single rays) exactly as the row-pair kernel.

// Rows of a quad box: the slab's kTS + 1 rows and no padding.  The two quads
// of a warp read planes two or three apart; with a plane stride of BX * 9
// words (8 mod 32 banks for BX = 8 mod 16) those fall 16 or 24 banks apart,
// where the padded stride (16 mod 32) puts planes two apart on the same banks.
#ifndef CBCT_QUAD_BOXY
#define CBCT_QUAD_BOXY 9
#endif
constexpr int kQuadBoxY = CBCT_QUAD_BOXY;
static_assert(kQuadBoxY >= kTS + 1, "a quad box holds the slab's rows and the next one");

// One sample of a quad (rays sorted by z; z0/dz hold their z start and step).
template <class V, int BX, bool CHECK>
__device__ __forceinline__ float4 quad_eval(const V* __restrict__ s, float k, float2 c0, float2 dc, float4 z0,
                                            float4 dz, float cmo, unsigned maxidx, int& bad) {
  constexpr int BXY = BX * kQuadBoxY;
  const float2 pq = __ffma2_rn(make_float2(k, k), dc, c0);
  const float fe = floor_small(pq.x), fd = floor_small(pq.y);
  const float2 aed = __fadd2_rn(pq, make_float2(-fe, -fd));
  const float c0z = fmaf(k, dz.x, z0.x), c1z = fmaf(k, dz.y, z0.y);
  const float c2z = fmaf(k, dz.z, z0.z), c3z = fmaf(k, dz.w, z0.w);
  const float f0 = floor_small(c0z), f1 = floor_small(c1z), f2 = floor_small(c2z), f3 = floor_small(c3z);
  const float s1 = f1 - f0, s2 = f2 - f0, s3 = f3 - f0;   // 0, 1 or 2
  const int idx0 = int_of_biased(fmaf(f0, float(BXY), fmaf(fd, float(BX), fe)) + cmo);
  if (CHECK) {
    const float smax = fmaxf(s1, fmaxf(s2, s3)), smin = fminf(s1, fminf(s2, s3));
    bad |= ((unsigned)idx0 > maxidx) | (smax >= 1.f && (unsigned)idx0 + 2u * BXY > maxidx) | (smax > 2.f) |
           (smin < 0.f) | (s1 > 1.f);
  }
  // planes fz, fz + 1 from q; fz + 2, fz + 3 from q2 (in the box whenever a ray
  // needs them; clamped otherwise)
  const V* q = s + min((unsigned)idx0, maxidx);
  const V* q2 = s + min((unsigned)idx0 + 2u * BXY, maxidx);
  const float2 te = make_float2(aed.x, aed.x);
  const float2 e0 = lerp2(make_float2(sm_f(q[0]), sm_f(q[BX])), make_float2(sm_f(q[1]), sm_f(q[BX + 1])), te);
  const float2 e1 = lerp2(make_float2(sm_f(q[BXY]), sm_f(q[BXY + BX])),
                          make_float2(sm_f(q[BXY + 1]), sm_f(q[BXY + BX + 1])), te);
  const float2 e2 = lerp2(make_float2(sm_f(q2[0]), sm_f(q2[BX])), make_float2(sm_f(q2[1]), sm_f(q2[BX + 1])), te);
  const float2 e3 = lerp2(make_float2(sm_f(q2[BXY]), sm_f(q2[BXY + BX])),
                          make_float2(sm_f(q2[BXY + 1]), sm_f(q2[BXY + BX + 1])), te);
  const float2 td = make_float2(aed.y, aed.y);
  const float2 d01 = lerp2(make_float2(e0.x, e1.x), make_float2(e0.y, e1.y), td);   // planes fz, fz + 1
  const float2 d23 = lerp2(make_float2(e2.x, e3.x), make_float2(e2.y, e3.y), td);   // planes fz + 2, fz + 3
  // Each ray lerps between two consecutive planes of the four: base value and
  // difference picked by its plane offset (the same subtraction hi - lo for
  // every ray that uses the pair, so the result is unchanged).
  const float g0 = d01.y - d01.x, g1 = d23.x - d01.y, g2 = d23.y - d23.x;
  auto ray = [&](float sk, float cz, float fz) {
    const float lo = sk < 0.5f ? d01.x : (sk < 1.5f ? d01.y : d23.x);
    const float gd = sk < 0.5f ? g0 : (sk < 1.5f ? g1 : g2);
    return fmaf(cz - fz, gd, lo);
  };
  // the second-lowest ray is under one texel above the lowest: planes fz, fz + 1 or fz + 1, fz + 2
  const float lo1 = s1 < 0.5f ? d01.x : d01.y, g1s = s1 < 0.5f ? g0 : g1;
  return make_float4(fmaf(c0z - f0, g0, d01.x), fmaf(c1z - f1, g1s, lo1), ray(s2, c2z, f2), ray(s3, c3z, f3));
}

// The quad's samples inside one slab, each ray's values added in ray order.
#ifndef CBCT_QUAD_UNROLL
#define CBCT_QUAD_UNROLL 1
#endif

template <class V, int BX, int SGN, bool CHECK>
__device__ __forceinline__ void quad_samples(const V* __restrict__ s, float& kf, float Nf, float ce0, float cd0,
                                             float dce, float dcd, float idcd, float4 z0, float4 dz, float lo,
                                             float hi, float cmo, unsigned maxidx, float4& acc, int& bad) {
  const float2 c0 = make_float2(ce0, cd0), dc = make_float2(dce, dcd);
  auto out_at = [&](float k) {
    const float x = fmaf(k, dcd, cd0);
    return SGN > 0 ? (x >= hi) : (x < lo);
  };
  float ke = ceilf(((SGN > 0 ? hi : lo) - cd0) * idcd);
  ke = fminf(fmaxf(ke, kf), Nf);
  while (ke > kf && out_at(ke - 1.f)) ke -= 1.f;
  while (ke < Nf && !out_at(ke)) ke += 1.f;
  float k = kf;
#if CBCT_QUAD_UNROLL > 1
  // Two quad-samples evaluated before they are added (in ray order).
  for (; k + 1.f < ke; k += 2.f) {
    const float4 v0 = quad_eval<V, BX, CHECK>(s, k, c0, dc, z0, dz, cmo, maxidx, bad);
    const float4 v1 = quad_eval<V, BX, CHECK>(s, k + 1.f, c0, dc, z0, dz, cmo, maxidx, bad);
    acc.x += v0.x;
    acc.y += v0.y;
    acc.z += v0.z;
    acc.w += v0.w;
    acc.x += v1.x;
    acc.y += v1.y;
    acc.z += v1.z;
    acc.w += v1.w;
  }
#endif
  for (; k < ke; k += 1.f) {
    const float4 v = quad_eval<V, BX, CHECK>(s, k, c0, dc, z0, dz, cmo, maxidx, bad);
    acc.x += v.x;
    acc.y += v.y;
    acc.z += v.z;
    acc.w += v.w;
  }
  kf = ke;
}

// Two rays of one column (rows a, b) outside a quad: a pair when they qualify,
// else each on its own.  Frame coordinates: (ce0, cd0, dce, dcd, idcd) per ray.
struct RayFrame {
  float ce0, cd0, dce, dcd, idcd, c0z, dcz;
};

__device__ __forceinline__ RayFrame ray_frame(const Ray& r, int dom) {
  RayFrame f;
  f.ce0 = dom ? r.c0x : r.c0y;
  f.dce = dom ? r.dcx : r.dcy;
  f.cd0 = dom ? r.c0y : r.c0x;
  f.dcd = dom ? r.dcy : r.dcx;
  f.idcd = 1.f / f.dcd;
  f.c0z = r.c0z;
  f.dcz = r.dcz;
  return f;
}

// Pair test of the row-pair kernel: 1 = pair with a lower, -1 = pair with b
// lower, 0 = no pair.
__device__ __forceinline__ int pair_kind(const Ray& ra, const Ray& rb, bool hit_a, bool hit_b, float Nf) {
  if (!(hit_a && hit_b && ra.a1 == rb.a1 && ra.a2 == rb.a2)) return 0;
  const float d0 = rb.c0z - ra.c0z;
  const float d1 = fmaf(Nf - 1.f, rb.dcz, rb.c0z) - fmaf(Nf - 1.f, ra.dcz, ra.c0z);
  if (d0 >= 2e-3f && d0 <= 0.998f && d1 >= 2e-3f && d1 <= 0.998f) return 1;
  if (d0 <= -2e-3f && d0 >= -0.998f && d1 <= -2e-3f && d1 >= -0.998f) return -1;
  return 0;
}

template <class V, int BX, int SGN, bool CHECK>
__device__ __forceinline__ void half_samples(const V* __restrict__ s, int kind, bool hit_a, bool hit_b,
                                             const RayFrame& fa, const RayFrame& fb, float& kfa, float& kfb,
                                             float Nf, float lo, float hi, float cmo, unsigned maxidx,
                                             unsigned maxidx3, float& acca, float& accb, int& bad) {
  if (kind != 0) {
    const bool al = kind > 0;
    float accl = al ? acca : accb, accu = al ? accb : acca;
    constexpr int QY = kQuadBoxY;
    pair_samples<V, BX, SGN, CHECK, QY>(s, kfa, Nf, fa.ce0, fa.cd0, fa.dce, fa.dcd, fa.idcd, al ? fa.c0z : fb.c0z,
                                        al ? fa.dcz : fb.dcz, al ? fb.c0z : fa.c0z, al ? fb.dcz : fa.dcz, lo, hi,
                                        cmo, maxidx, maxidx3, accl, accu, bad);
    acca = al ? accl : accu;
    accb = al ? accu : accl;
    return;
  }
  constexpr int QY = kQuadBoxY;
  if (hit_a)
    slab_samples<V, BX, SGN, CHECK, QY>(s, kfa, Nf, fa.ce0, fa.cd0, fa.c0z, fa.dce, fa.dcd, fa.idcd, fa.dcz, lo, hi,
                                        cmo, maxidx, acca, bad);
  if (hit_b)
    slab_samples<V, BX, SGN, CHECK, QY>(s, kfb, Nf, fb.ce0, fb.cd0, fb.c0z, fb.dce, fb.dcd, fb.idcd, fb.dcz, lo, hi,
                                        cmo, maxidx, accb, bad);
}

// CTAs per SM the register budget is sized for: four 128-thread CTAs (124
// registers, no spills), as many as the fp32 boxes of 16x32 tiles leave room
// for; the half-size 16-bit boxes leave room for five (96 registers).
#ifndef CBCT_QUAD_MINB16
#define CBCT_QUAD_MINB16 5
#endif
template <class V>
constexpr int quad_min_blocks() {
#ifdef CBCT_QUAD_MINB
  return CBCT_QUAD_MINB;
#else
  return kQuadThreads >= 256 ? 2 : kQuadThreads >= 128 ? (sizeof(V) == 4 ? 4 : CBCT_QUAD_MINB16) : 6;
#endif
}

// One CTA of the row-quad kernel (see fwd_slab_body).
template <class V, int BX, bool CHECK>
__device__ __forceinline__ void fwd_quad_body(const CUtensorMap* map_v, const CUtensorMap* map_t,
                                              const V* __restrict__ vol, const ViewParams* __restrict__ views,
                                              const GridConst& gc, int BZ, int nsl_max, const FwdOut& o,
                                              int* flags, const TileId& tile, unsigned char* smem_raw,
                                              PairShared& sh) {
  constexpr int BXY = BX * kQuadBoxY;
  const ViewParams vp = views[tile.z];
  const int dom = vp.dom;
  const CUtensorMap* map = dom ? map_v : map_t;
  const int tid = threadIdx.x;
  const int p = tile.z;
  const int u0 = tile.x * kQU, v0 = tile.y * kQV;
  const int u = u0 + (tid % kQU), vq = v0 + 4 * (tid / kQU);
  const int uc = min(u, gc.W - 1);
  const float Nf = float(gc.N);
  Ray r[4];
  bool act[4], hit[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    act[i] = (u < gc.W) && (vq + i < gc.H);
    r[i] = make_ray(vp, gc, uc, min(vq + i, gc.H - 1));
    hit[i] = act[i] && (r[i].a2 > r[i].a1);
  }
  RayFrame f[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) f[i] = ray_frame(r[i], dom);
  // Quad test: one clip; sorted by z (rows run one way), every ray within
  // [0.002, 1.998] texels above the lowest at both ends, the second-lowest
  // within [0.002, 0.998].
  bool quad = hit[0] && hit[1] && hit[2] && hit[3];
#pragma unroll
  for (int i = 1; i < 4; ++i) quad = quad && r[i].a1 == r[0].a1 && r[i].a2 == r[0].a2;
  const bool up = r[1].c0z > r[0].c0z;   // z grows with the row
  if (quad) {
    const int lo_i = up ? 0 : 3;
    const float zs = r[lo_i].c0z, ze = fmaf(Nf - 1.f, r[lo_i].dcz, r[lo_i].c0z);
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (i == lo_i) continue;
      const float d0 = r[i].c0z - zs, d1 = fmaf(Nf - 1.f, r[i].dcz, r[i].c0z) - ze;
      const float dmax = (up ? i == 1 : i == 2) ? 0.998f : 1.998f;
      quad = quad && d0 >= 2e-3f && d0 <= dmax && d1 >= 2e-3f && d1 <= dmax;
    }
  }
  // Sorted z parameters of the quad (lowest first).
  const float4 qz0 = up ? make_float4(f[0].c0z, f[1].c0z, f[2].c0z, f[3].c0z)
                        : make_float4(f[3].c0z, f[2].c0z, f[1].c0z, f[0].c0z);
  const float4 qdz = up ? make_float4(f[0].dcz, f[1].dcz, f[2].dcz, f[3].dcz)
                        : make_float4(f[3].dcz, f[2].dcz, f[1].dcz, f[0].dcz);
  const int kind01 = quad ? 0 : pair_kind(r[0], r[1], hit[0], hit[1], Nf);
  const int kind23 = quad ? 0 : pair_kind(r[2], r[3], hit[2], hit[3], Nf);
  const float ke_ = dom ? gc.kx : gc.ky, be = dom ? gc.bx : gc.by;
  const float kd = dom ? gc.ky : gc.kx, bd = dom ? gc.by : gc.bx;
  const float Se = dom ? vp.Sx : vp.Sy, Sd = dom ? vp.Sy : vp.Sx;

  if (tid == 0) {
    sh.mlo = INT_MAX;
    sh.mhi = INT_MIN;
    sh.abort_flag = 0;
    for (int st = 0; st < kPairStages; ++st) mbar_init(&sh.bars[st], 1);
    fence_mbar_init();
  }
  __syncthreads();
  {
    int mn = INT_MAX, mx = INT_MIN;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      if (!hit[i]) continue;
      const int m0 = (max(int(floorf(f[i].cd0)), kSlabBase) - kSlabBase) / kTS;
      const int m1 = (max(int(floorf(fmaf(Nf - 1.f, f[i].dcd, f[i].cd0))), kSlabBase) - kSlabBase) / kTS;
      mn = min(mn, min(m0, m1));
      mx = max(mx, max(m0, m1));
    }
    if (mn <= mx) {
      atomicMin(&sh.mlo, mn);
      atomicMax(&sh.mhi, mx);
    }
  }
  __syncthreads();
  const int mlo = sh.mlo, mhi = sh.mhi;
  int nslab = (mhi >= mlo) ? (mhi - mlo + 1) : 0;
  if (nslab > nsl_max) {
    if (tid == 0) atomicAdd(&flags[0], 1);
    nslab = 0;
  }
  const uint32_t box_bytes = uint32_t(BX * kQuadBoxY * BZ * sizeof(V));
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  int* const emin = reinterpret_cast<int*>(smem_raw + kPairStages * stage_stride);
  int* const emax = emin + nsl_max;
  int* const zmin = emax + nsl_max;
  int* const zmax = zmin + nsl_max;
  for (int i = tid; i < nslab; i += blockDim.x) {
    emin[i] = INT_MAX; emax[i] = INT_MIN;
    zmin[i] = INT_MAX; zmax[i] = INT_MIN;
  }
  __syncthreads();
  const int ue = min(u0 + kQU, gc.W) - 1, ve = min(v0 + kQV, gc.H) - 1;
  const int ne = dom ? gc.nx : gc.ny;
  for (int qq = tid; qq < nslab * 8; qq += blockDim.x) {
    const int i = qq >> 3, c = qq & 7;
    const int m = mlo + i;
    const float plane = float(kSlabBase + m * kTS + ((c & 4) ? kTS : 0));
    const int ucc = (c & 1) ? ue : u0, vcc = (c & 2) ? ve : v0;
    const float dx = fmaf(float(ucc), vp.Eux, vp.D0x);
    const float dy = fmaf(float(ucc), vp.Euy, vp.D0y);
    const float dzz = fmaf(float(vcc), vp.Evz, vp.D0z);
    const float de = dom ? dx : dy, dd = dom ? dy : dx;
    const float t = ((plane - bd) / kd - Sd) / dd;
    const float ce = fmaf(fmaf(t, de, Se), ke_, be);
    const float cz = fmaf(t * dzz, gc.kz, gc.bz);
    const int fe = min(max(int(floorf(fminf(fmaxf(ce, -1.0e5f), 1.0e5f))), -1), ne - 1);
    const int fz = min(max(int(floorf(fminf(fmaxf(cz, -1.0e5f), 1.0e5f))), -1), gc.nz - 1);
    atomicMin(&emin[i], fe);
    atomicMax(&emax[i], fe);
    atomicMin(&zmin[i], fz);
    atomicMax(&zmax[i], fz);
  }
  __syncthreads();

  const unsigned maxidx = unsigned(BXY * (BZ - 1) - BX - 2);   // two-plane loads stay in the box
  const unsigned maxidx3 = unsigned(BXY * BZ - BX - 2);        // the pair's third plane
  auto origin = [&](int i, int& oe, int& od, int& oz, int& m) {
    m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int ii = m - mlo;
    oe = (emin[ii] - 1) & ~(int(16 / sizeof(V)) - 1);   // 16-byte aligned x start
    od = kSlabBase + m * kTS;
    oz = zmin[ii] - 1;
  };
  auto issue = [&](int i) {
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    uint64_t* bar = &sh.bars[i % kPairStages];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(smem_raw + (i % kPairStages) * stage_stride, map, oe, od, oz, bar);
  };
  if (tid == 0) {
    for (int i = 0; i < min(kPairStages, nslab); ++i) issue(i);
  }

  float4 acc = make_float4(0.f, 0.f, 0.f, 0.f);   // quad: sorted by z; else per row
  float kf[4] = {0.f, 0.f, 0.f, 0.f};            // quad / pairs: kf[0], kf[2] lead
  int bad = 0;
  int done = 0;
  for (int i = 0; i < nslab; ++i) {
    const int slot = i % kPairStages;
    const bool ok = mbar_wait_bounded(&sh.bars[slot], (i / kPairStages) & 1, gc.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); sh.abort_flag = 1; }
      break;
    }
    done = i + 1;
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    if (CHECK && tid == 0) {
      const int ii = m - mlo;
      if (emax[ii] + 2 - oe >= BX || zmax[ii] + 2 - oz >= BZ) atomicAdd(&flags[0], 1);
    }
    const V* sm = reinterpret_cast<const V*>(smem_raw + slot * stage_stride);
    const float lo = float(od), hi = lo + float(kTS);
    const float cmo = kRoundC - float(oe + od * BX + oz * BXY);
    if (quad) {
      if (vp.dsgn > 0)
        quad_samples<V, BX, 1, CHECK>(sm, kf[0], Nf, f[0].ce0, f[0].cd0, f[0].dce, f[0].dcd, f[0].idcd, qz0, qdz, lo,
                                      hi, cmo, maxidx, acc, bad);
      else
        quad_samples<V, BX, -1, CHECK>(sm, kf[0], Nf, f[0].ce0, f[0].cd0, f[0].dce, f[0].dcd, f[0].idcd, qz0, qdz,
                                       lo, hi, cmo, maxidx, acc, bad);
    } else if (vp.dsgn > 0) {
      half_samples<V, BX, 1, CHECK>(sm, kind01, hit[0], hit[1], f[0], f[1], kf[0], kf[1], Nf, lo, hi, cmo, maxidx,
                                    maxidx3, acc.x, acc.y, bad);
      half_samples<V, BX, 1, CHECK>(sm, kind23, hit[2], hit[3], f[2], f[3], kf[2], kf[3], Nf, lo, hi, cmo, maxidx,
                                    maxidx3, acc.z, acc.w, bad);
    } else {
      half_samples<V, BX, -1, CHECK>(sm, kind01, hit[0], hit[1], f[0], f[1], kf[0], kf[1], Nf, lo, hi, cmo, maxidx,
                                     maxidx3, acc.x, acc.y, bad);
      half_samples<V, BX, -1, CHECK>(sm, kind23, hit[2], hit[3], f[2], f[3], kf[2], kf[3], Nf, lo, hi, cmo, maxidx,
                                     maxidx3, acc.z, acc.w, bad);
    }
    __syncthreads();
    if (tid == 0 && i + kPairStages < nslab) {
      fence_proxy_async();
      issue(i + kPairStages);
    }
  }
  if (sh.abort_flag && tid == 0) {
    for (int i = done; i < min(done + kPairStages, nslab); ++i)
      if (!mbar_wait_bounded(&sh.bars[i % kPairStages], (i / kPairStages) & 1, kWaitLimit)) sh.abort_flag = 2;
  }
  if (CHECK) {
    // every sample of a hit ray must be consumed
    if (quad) {
      if (kf[0] != Nf) bad = 1;
    } else {
      if (kind01 != 0 ? kf[0] != Nf : ((hit[0] && kf[0] != Nf) || (hit[1] && kf[1] != Nf))) bad = 1;
      if (kind23 != 0 ? kf[2] != Nf : ((hit[2] && kf[2] != Nf) || (hit[3] && kf[3] != Nf))) bad = 1;
    }
    if (bad) atomicAdd(&flags[0], 1);
  }
  // Per-row sums (the quad's are sorted by z).
  float sum[4];
  if (quad && !up) {
    sum[0] = acc.w; sum[1] = acc.z; sum[2] = acc.y; sum[3] = acc.x;
  } else {
    sum[0] = acc.x; sum[1] = acc.y; sum[2] = acc.z; sum[3] = acc.w;
  }
  double sq = 0.0;
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    float val = 0.f;
    int k0, k1;
    if (hit[i])
      val = sum[i] * r[i].delta;
    else if (act[i] && grown_range(vp, gc, u, vq + i, r[i], k0, k1))
      val = march_global(vol, gc, r[i], k0, k1) * r[i].delta;
    if (act[i]) sq += fwd_store(o, gc, vp, p, u, vq + i, val);
  }
  fwd_block_partial(o, sq, sh.red, tid, tile.bid);
}

template <class V, int BX, bool CHECK>
__global__ void __launch_bounds__(kQuadThreads, quad_min_blocks<V>())
    fwd_quad_kernel(const __grid_constant__ CUtensorMap map_v, const __grid_constant__ CUtensorMap map_t,
                    const V* __restrict__ vol, const ViewParams* __restrict__ views, GridConst gc, int BZ,
                    int nsl_max, FwdOut o, int* flags) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  __shared__ PairShared sh;
  fwd_quad_body<V, BX, CHECK>(&map_v, &map_t, vol, views, gc, BZ, nsl_max, o, flags, launch_tile(), smem_raw, sh);
}

// ------------------------------------------------------------------ fan
// The rays of one detector column lie in one vertical plane (the detector's
// v axis is the world z axis).  A ray that enters and leaves the volume
// through its side faces has the clip (a1, a2) of the column's in-plane path,
// so its k-th sample sits at the column's k-th in-plane position (e_k, d_k);
// only z differs between the rows.  The fan kernel gives each warp one column
// of a kFU x kFV tile (lane = detector row).  Per slab, the warp first
// interpolates the column's samples in e and d on every z plane its rays
// reach ("lines", one value per sample and plane), then every ray takes its
// samples as linear interpolations in z between two line entries.  This is
// the slab kernel's trilinear tree (e, then d, then z) with the e/d part
// shared by the column's rays, so results are bitwise those of the per-ray
// kernels.  Rays clipped by the top or bottom face (their own a1/a2) take the
// per-ray trilinear path on the same box.
struct FanShared {
  uint64_t bars[kNStage];
  int mlo, mhi, abort_flag;
  double red[8];
  float tile[kFV][kFU + 1];  // results, transposed for a coalesced epilogue
};

// The column's samples inside one slab, in chunks of kFKC (warp-level; every
// lane of the warp calls it).  kcol: the column's next sample (warp-uniform).
template <class V, int BX, int SGN, bool CHECK>
__device__ __forceinline__ void fan_slab(const V* __restrict__ s, float* __restrict__ lines, int LZ, int BZ,
                                         int lane, int N, int& kcol, float2 c0, float2 dc, bool shared, float c0z,
                                         float dcz, float lo, float hi, int oz, float orgf, float& acc, int& bad) {
  constexpr int BXY = BX * kBoxY;
  constexpr unsigned FULL = 0xffffffffu;
  const unsigned maxidx = unsigned(BXY * BZ - BX - 2);
  auto outside = [&](float fd) { return SGN > 0 ? (fd >= hi) : (fd < lo); };
  for (;;) {
    if (kcol >= N) return;
    // Samples of the chunk still inside the slab (a prefix, floor(d) being
    // monotone along the ray).
    bool in = false;
    if (lane < kFKC && kcol + lane < N) {
      const float kj = float(kcol + lane);
      in = !outside(floorf(fmaf(kj, dc.y, c0.y)));
    }
    const int nk = __ffs(~__ballot_sync(FULL, in)) - 1;
    if (nk <= 0) return;
    // z planes the shared rays reach over the chunk.
    int zl = INT_MAX, zh = INT_MIN;
    if (shared) {
      const int fa = int(floorf(fmaf(float(kcol), dcz, c0z)));
      const int fb = int(floorf(fmaf(float(kcol + nk - 1), dcz, c0z)));
      zl = min(fa, fb);
      zh = max(fa, fb);
    }
    zl = __reduce_min_sync(FULL, zl);
    zh = __reduce_max_sync(FULL, zh);
    int nz = zh - zl + 2;
    if (CHECK && (nz > LZ || zl < oz || zh + 1 >= oz + BZ)) bad = 1;
    nz = min(nz, LZ);
    // Lines: lane (j, g) interpolates sample j on planes g, g + G, ...
    const int G = 32 / nk;
    const int j = lane % nk, g = lane / nk;
    if (g < G) {
      const float kfj = float(kcol + j);
      const float2 pa = __ffma2_rn(make_float2(kfj, kfj), dc, c0);
      const float fe = floor_small(pa.x), fd = floor_small(pa.y);
      const float2 aed = __fadd2_rn(pa, make_float2(-fe, -fd));
      const float2 te = make_float2(aed.x, aed.x);
      const float td = aed.y;
      int idx = int(fmaf(float(zl + g), float(BXY), fmaf(fd, float(BX), fe)) - orgf);
      float* L = lines + j * LZ;
      for (int z = g; z < nz; z += G, idx += G * BXY) {
        if (CHECK) bad |= (unsigned)idx > maxidx;
        const V* q = s + min((unsigned)idx, maxidx);
        const float2 a0 = make_float2(sm_f(q[0]), sm_f(q[BX]));
        const float2 b0 = make_float2(sm_f(q[1]), sm_f(q[BX + 1]));
        const float2 e = lerp2(a0, b0, te);  // (d0, d1) rows on plane z
        L[z] = fmaf(td, e.y, fmaf(-td, e.x, e.x));
      }
    }
    __syncwarp();
    if (shared) {
      const float* L = lines;
      for (int jj = 0; jj < nk; ++jj, L += LZ) {
        const float cz = fmaf(float(kcol + jj), dcz, c0z);
        const float fz = floor_small(cz);
        const float az = cz - fz;
        int iz = int(fz) - zl;
        if (CHECK) bad |= (unsigned)iz > (unsigned)(nz - 2);
        iz = min(max(iz, 0), nz - 2);
        acc += fmaf(az, L[iz + 1] - L[iz], L[iz]);
      }
    }
    kcol += nk;
    __syncwarp();
    if (nk < kFKC) return;
  }
}

template <class V, int BX, bool CHECK>
__global__ void __launch_bounds__(256, 3) fwd_fan_kernel(const __grid_constant__ CUtensorMap map_v,
                                                      const __grid_constant__ CUtensorMap map_t,
                                                      const V* __restrict__ vol,
                                                      const ViewParams* __restrict__ views, GridConst gc,
                                                      int BZ, int LZ, int nsl_max, FwdOut o, int* flags) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  __shared__ FanShared sh;
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  constexpr int BXY = BX * kBoxY;
  const ViewParams vp = views[blockIdx.z];
  const int dom = vp.dom;
  const CUtensorMap* map = dom ? &map_v : &map_t;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int p = blockIdx.z;
  const int u0 = blockIdx.x * kFU, v0 = blockIdx.y * kFV;
  const int u = u0 + warp, v = v0 + lane;
  const bool active = (u < gc.W) && (v < gc.H);
  const int uc = min(u, gc.W - 1);
  const Ray r = make_ray(vp, gc, uc, min(v, gc.H - 1));
  const bool hit = active && (r.a2 > r.a1);
  // The column's in-plane clip: make_ray's without the z faces.
  const float dx = fmaf(float(uc), vp.Eux, vp.D0x);
  const float dy = fmaf(float(uc), vp.Euy, vp.D0y);
  const float tx1 = __fdiv_rn(gc.hx - vp.Sx, dx), tx2 = __fdiv_rn(-gc.hx - vp.Sx, dx);
  const float ty1 = __fdiv_rn(gc.hy - vp.Sy, dy), ty2 = __fdiv_rn(-gc.hy - vp.Sy, dy);
  const float a1c = fmaxf(fmaxf(fminf(tx1, tx2), fminf(ty1, ty2)), 0.f);
  const float a2c = fminf(fminf(fmaxf(tx1, tx2), fmaxf(ty1, ty2)), 1.f);
  const bool shared = hit && r.a1 == a1c && r.a2 == a2c;
  const bool own = hit && !shared;
  const bool any_shared = __any_sync(0xffffffffu, shared);
  // Frame coordinates (e = cross axis, d = slab axis) of this lane's ray; for
  // shared rays they are the column's.
  const float ce0 = dom ? r.c0x : r.c0y, dce = dom ? r.dcx : r.dcy;
  const float cd0 = dom ? r.c0y : r.c0x, dcd = dom ? r.dcy : r.dcx;
  const float idcd = 1.f / dcd;
  // The column's frame coordinates, from the first shared lane.
  const int src = any_shared ? __ffs(__ballot_sync(0xffffffffu, shared)) - 1 : 0;
  const float2 cc0 = make_float2(__shfl_sync(0xffffffffu, ce0, src), __shfl_sync(0xffffffffu, cd0, src));
  const float2 cdc = make_float2(__shfl_sync(0xffffffffu, dce, src), __shfl_sync(0xffffffffu, dcd, src));

  if (tid == 0) {
    sh.mlo = INT_MAX;
    sh.mhi = INT_MIN;
    sh.abort_flag = 0;
    for (int s = 0; s < kNStage; ++s) mbar_init(&sh.bars[s], 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (hit) {
    const int f0 = int(floorf(cd0));
    const int f1 = int(floorf(fmaf(float(gc.N - 1), dcd, cd0)));
    const int m0 = (max(f0, kSlabBase) - kSlabBase) / kTS;
    const int m1 = (max(f1, kSlabBase) - kSlabBase) / kTS;
    atomicMin(&sh.mlo, min(m0, m1));
    atomicMax(&sh.mhi, max(m0, m1));
  }
  __syncthreads();
  const int mlo = sh.mlo, mhi = sh.mhi;
  int nslab = (mhi >= mlo) ? (mhi - mlo + 1) : 0;
  if (nslab > nsl_max) {
    if (tid == 0) atomicAdd(&flags[0], 1);
    nslab = 0;
  }
  // Per-slab footprints (e min, e max, z min, z max) live after the lines.
  const uint32_t box_bytes = uint32_t(BX * kBoxY * BZ * sizeof(V));
  const uint32_t stage_stride = (box_bytes + 127u) & ~127u;
  int* foot = reinterpret_cast<int*>(smem_raw + kNStage * stage_stride + (size_t)kFU * kFKC * LZ * sizeof(float));
  const float ke = dom ? gc.kx : gc.ky, be = dom ? gc.bx : gc.by;
  const float kd = dom ? gc.ky : gc.kx, bd = dom ? gc.by : gc.bx;
  const float Se = dom ? vp.Sx : vp.Sy, Sd = dom ? vp.Sy : vp.Sx;
  for (int i = tid; i < nslab; i += blockDim.x) {
    foot[i] = INT_MAX; foot[nsl_max + i] = INT_MIN;
    foot[2 * nsl_max + i] = INT_MAX; foot[3 * nsl_max + i] = INT_MIN;
  }
  __syncthreads();
  // Footprint of every slab: the four corner rays of the tile at the slab's
  // two bounding planes.
  const int ue = min(u0 + kFU, gc.W) - 1, ve = min(v0 + kFV, gc.H) - 1;
  const int ne = dom ? gc.nx : gc.ny;  // volume extent along e
  for (int q = tid; q < nslab * 8; q += blockDim.x) {
    const int i = q >> 3, c = q & 7;
    const int m = mlo + i;
    const float plane = float(kSlabBase + m * kTS + ((c & 4) ? kTS : 0));
    const int ucc = (c & 1) ? ue : u0, vcc = (c & 2) ? ve : v0;
    const float ddx = fmaf(float(ucc), vp.Eux, vp.D0x);
    const float ddy = fmaf(float(ucc), vp.Euy, vp.D0y);
    const float ddz = fmaf(float(vcc), vp.Evz, vp.D0z);
    const float de = dom ? ddx : ddy, dd = dom ? ddy : ddx;
    const float t = ((plane - bd) / kd - Sd) / dd;
    float ce = fmaf(fmaf(t, de, Se), ke, be);
    float cz = fmaf(t * ddz, gc.kz, gc.bz);
    // Samples lie inside the volume (texel floors in [-1, n-1]; outside it the
    // border reads 0), so the box only has to cover the footprint's part in it.
    const int fe = min(max(int(floorf(fminf(fmaxf(ce, -1.0e5f), 1.0e5f))), -1), ne - 1);
    const int fz = min(max(int(floorf(fminf(fmaxf(cz, -1.0e5f), 1.0e5f))), -1), gc.nz - 1);
    atomicMin(&foot[i], fe);
    atomicMax(&foot[nsl_max + i], fe);
    atomicMin(&foot[2 * nsl_max + i], fz);
    atomicMax(&foot[3 * nsl_max + i], fz);
  }
  __syncthreads();

  const unsigned maxidx = unsigned(BXY * (BZ - 1) - BX - 2);
  float* lines = reinterpret_cast<float*>(smem_raw + kNStage * stage_stride) + warp * (kFKC * LZ);
  auto origin = [&](int i, int& oe, int& od, int& oz, int& m) {
    m = (vp.dsgn > 0) ? mlo + i : mhi - i;
    const int ii = m - mlo;
    oe = (foot[ii] - 1) & ~(int(16 / sizeof(V)) - 1);
    od = kSlabBase + m * kTS;
    oz = foot[2 * nsl_max + ii] - 1;
  };
  auto issue = [&](int i) {
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    uint64_t* bar = &sh.bars[i % kNStage];
    mbar_arrive_expect_tx(bar, box_bytes);
    tma_load_3d(smem_raw + (i % kNStage) * stage_stride, map, oe, od, oz, bar);
  };
  if (tid == 0) {
    for (int i = 0; i < min(kNStage, nslab); ++i) issue(i);
  }

  float acc = 0.f;
  float kf = 0.f;   // own rays: next sample
  int kcol = 0;     // the column's next sample
  const float Nf = float(gc.N);
  int bad = 0;
  int done = 0;
  for (int i = 0; i < nslab; ++i) {
    const int slot = i % kNStage;
    const bool ok = mbar_wait_bounded(&sh.bars[slot], (i / kNStage) & 1, gc.wait_limit);
    if (__syncthreads_or(!ok)) {
      if (tid == 0) { atomicAdd(&flags[1], 1); sh.abort_flag = 1; }
      break;
    }
    done = i + 1;
    int oe, od, oz, m;
    origin(i, oe, od, oz, m);
    if (CHECK && tid == 0) {
      const int ii = m - mlo;
      if (foot[nsl_max + ii] + 2 - oe >= BX || foot[3 * nsl_max + ii] + 2 - oz >= BZ) atomicAdd(&flags[0], 1);
    }
    const V* s = reinterpret_cast<const V*>(smem_raw + slot * stage_stride);
    const float lo = float(od), hi = lo + float(kTS);
    const float orgf = float(oe + od * BX + oz * BXY);
    if (any_shared) {
      if (vp.dsgn > 0)
        fan_slab<V, BX, 1, CHECK>(s, lines, LZ, BZ, lane, gc.N, kcol, cc0, cdc, shared, r.c0z, r.dcz, lo, hi, oz,
                                  orgf, acc, bad);
      else
        fan_slab<V, BX, -1, CHECK>(s, lines, LZ, BZ, lane, gc.N, kcol, cc0, cdc, shared, r.c0z, r.dcz, lo, hi, oz,
                                   orgf, acc, bad);
    }
    if (own) {
      const float cmo = kRoundC - orgf;
      if (vp.dsgn > 0)
        slab_samples<V, BX, 1, CHECK>(s, kf, Nf, ce0, cd0, r.c0z, dce, dcd, idcd, r.dcz, lo, hi, cmo, maxidx, acc,
                                        bad);
      else
        slab_samples<V, BX, -1, CHECK>(s, kf, Nf, ce0, cd0, r.c0z, dce, dcd, idcd, r.dcz, lo, hi, cmo, maxidx, acc,
                                         bad);
    }
    __syncthreads();
    if (tid == 0 && i + kNStage < nslab) {
      fence_proxy_async();
      issue(i + kNStage);
    }
  }
  if (sh.abort_flag && tid == 0) {
    for (int i = done; i < min(done + kNStage, nslab); ++i)
      (void)mbar_wait_bounded(&sh.bars[i % kNStage], (i / kNStage) & 1, kWaitLimit);
  }
  if (CHECK && !sh.abort_flag) {
    if ((shared && kcol != gc.N) || (own && kf != Nf)) bad = 1;  // every sample of a hit ray is consumed
    if (bad) atomicAdd(&flags[0], 1);
  }

  float val = 0.f;
  if (hit) {
    val = acc * r.delta;
  } else if (active) {
    int k0, k1;
    if (grown_range(vp, gc, u, v, r, k0, k1)) val = march_global(vol, gc, r, k0, k1) * r.delta;
  }
  // Transpose through shared memory so that the epilogue's accesses run along u.
  sh.tile[lane][warp] = val;
  __syncthreads();
  const int tu = tid % kFU, tv = tid / kFU;
  const int eu = u0 + tu, ev = v0 + tv;
  fwd_epilogue(o, gc, vp, p, eu, ev, eu < gc.W && ev < gc.H, sh.tile[tv][tu], sh.red, tid, launch_block_id());
}

// ------------------------------------------------------------------ host
CUtensorMapDataType tma_dtype(cbct_dtype dt) {
  switch (dt) {
    case CBCT_F32: return CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    case CBCT_F16: return CU_TENSOR_MAP_DATA_TYPE_FLOAT16;
    default: return CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
  }
}

// ------------------------------------------------------------------ work list
// Work-list (persistent) forward projector over many scans: resident CTAs
// take items -- one ray tile of one view of one scan -- from an atomic counter
// until the list is empty and run the one-scan kernel's body on them, so every
// ray gets the arithmetic of its own launch.  A scan's items are numbered in
// its one-scan launch order (x fastest), which is also its partial-sum slot.
enum { kVarSlab1 = 0, kVarSlab2 = 1, kVarPair = 2, kVarQuad = 3 };

struct alignas(128) FwdScanRec {
  CUtensorMap map_v, map_t;    // volume and x/y-transposed volume, the plan's box
  const void* vol;
  const ViewParams* views;     // the subset's views
  int* flags;
  GridConst gc;
  FwdOut o;
  int BZ, nsl_max;
  int tx, ty;                  // ray tiles per view (x, y)
  int base;                    // work-list index of the scan's first tile
};

template <int VAR>
constexpr int var_threads() { return VAR == kVarPair ? kPairThreads : VAR == kVarQuad ? kQuadThreads : 256; }
template <int VAR, class V>
constexpr int var_min_blocks() {
#ifdef CBCT_MULTI_PAIR_MINB
  if (VAR == kVarPair) return CBCT_MULTI_PAIR_MINB;
#endif
  return VAR == kVarPair ? pair_min_blocks<V>() : VAR == kVarQuad ? quad_min_blocks<V>() : slab_min_blocks<V>();
}

template <int VAR, class V, int BX>
__global__ void __launch_bounds__(var_threads<VAR>(), var_min_blocks<VAR, V>())
    fwd_multi_kernel(const FwdScanRec* __restrict__ recs, int n_recs, int total, int* __restrict__ counter) {
  extern __shared__ __align__(128) unsigned char smem_dyn[];
  unsigned char* smem_raw =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_dyn) + 127) & ~uintptr_t(127));
  using Shared = typename std::conditional<VAR <= kVarSlab2, SlabShared, PairShared>::type;
  __shared__ Shared sh;
  __shared__ int item;
  __shared__ int base[kMultiMaxRecs];
  constexpr int kBars = VAR == kVarSlab1 ? 1 : VAR == kVarSlab2 ? 2 : kPairStages;
  for (int i = threadIdx.x; i < n_recs; i += blockDim.x) base[i] = recs[i].base;
  int last = -1;
  for (;;) {
    if (threadIdx.x == 0) item = atomicAdd(counter, 1);
    __syncthreads();
    const int t = item;
    if (t >= total) break;
    // Broadcast: the compiler may then keep the record's fields uniform.
    const int lo = __shfl_sync(0xffffffffu, find_rec(base, n_recs, t), 0);
    const FwdScanRec& R = recs[lo];
    int l = t - base[lo];
    TileId tile;
    tile.bid = (size_t)l;
    tile.x = l % R.tx;
    l /= R.tx;
    tile.y = l % R.ty;
    tile.z = l / R.ty;
    if (threadIdx.x == 0 && lo != last) {   // the thread that issues the TMA loads
      tensormap_acquire(&R.map_v);
      tensormap_acquire(&R.map_t);
      last = lo;
    }
    const V* vol = static_cast<const V*>(R.vol);
    if constexpr (VAR == kVarSlab1)
      fwd_slab_body<V, BX, false, 1>(&R.map_v, &R.map_t, vol, R.views, R.gc, R.BZ, R.o, R.flags, tile, smem_raw, sh);
    else if constexpr (VAR == kVarSlab2)
      fwd_slab_body<V, BX, false, 2>(&R.map_v, &R.map_t, vol, R.views, R.gc, R.BZ, R.o, R.flags, tile, smem_raw, sh);
    else if constexpr (VAR == kVarPair)
      fwd_pair_body<V, BX, false>(&R.map_v, &R.map_t, vol, R.views, R.gc, R.BZ, R.nsl_max, R.o, R.flags, tile,
                                  smem_raw, sh);
    else
      fwd_quad_body<V, BX, false>(&R.map_v, &R.map_t, vol, R.views, R.gc, R.BZ, R.nsl_max, R.o, R.flags, tile,
                                  smem_raw, sh);
    __syncthreads();
    // A wait that gave up is counted in the scan's flag word and its loads
    // drained; only a CTA whose drain also gave up (a copy may still land in
    // its shared memory) stops taking items.
    const bool ok = sh.abort_flag != 2;
    if (threadIdx.x == 0) {
      for (int i = 0; i < kBars; ++i) mbar_inval(&sh.bars[i]);
    }
    if (!ok) break;
  }
}

CUtensorMap make_map(cbct_dtype dt, const void* vol, int n0, int n1, int n2, const SlabBox& b) {
  CUtensorMap m;
  std::memset(&m, 0, sizeof(m));
  const size_t es = dtype_size(dt);
  cuuint64_t dims[3] = {(cuuint64_t)n0, (cuuint64_t)n1, (cuuint64_t)n2};
  cuuint64_t strides[2] = {(cuuint64_t)n0 * es, (cuuint64_t)n0 * n1 * es};
  cuuint32_t box[3] = {(cuuint32_t)b.bx, (cuuint32_t)b.by, (cuuint32_t)b.bz};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult res = tensor_map_encoder()(&m, tma_dtype(dt), 3, const_cast<void*>(vol), dims, strides, box, estr,
                                      CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                      CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (res != CUDA_SUCCESS)
    throw Error(CBCT_ERR_CUDA, "cuTensorMapEncodeTiled failed with code " + std::to_string((int)res));
  return m;
}

// Dynamic shared memory of a slab or fan launch: kNStage TMA stages of the
// box (128-byte aligned) + the fan kernel's lines + alignment slack.
static size_t forward_smem(const SlabBox& b, size_t es, int lz, int nsl = 0) {
  return kNStage * ((b.bx * b.by * b.bz * es + 127) & ~size_t(127)) + (size_t)kFU * kFKC * lz * sizeof(float) +
         4 * sizeof(int) * (size_t)nsl + 128;
}

// Slabs a ray can cross in the larger in-plane direction.
static int slabs_max(const cbct_geometry& g) {
  return (std::max(g.nx, g.ny) + 1 - kSlabBase + kTS - 1) / kTS + 1;
}

// Dynamic shared memory of a row-pair launch: kPairStages boxes (128-byte
// aligned), the per-slab footprints, alignment slack.
static size_t pair_smem(const SlabBox& b, size_t es, int nsl) {
  return kPairStages * ((b.bx * b.by * b.bz * es + 127) & ~size_t(127)) + 4 * sizeof(int) * (size_t)nsl + 128;
}

template <class V>
const SlabBox& box_for(const cbct_plan* p) { return sizeof(V) == 4 ? p->slab : p->slab16; }

// Two stages while they leave the register-bound number of CTAs per SM;
// boxes so large that they would not (small volumes under detectors of about
// one pixel per voxel) stage one slab at a time, and the other CTAs' samples
// cover each CTA's wait.  Returns the stages and sets the dynamic shared memory.
template <class V>
int slab_stages(const SlabBox& b, size_t& smem) {
  const size_t stage = (b.bx * b.by * b.bz * sizeof(V) + 127) & ~size_t(127);
  const size_t per_cta = sizeof(SlabShared) + 1024 + 128;
  const bool two = (2 * stage + per_cta) * slab_min_blocks<V>() <= size_t(228) * 1024;
  smem = (two ? 2 : 1) * stage + 128;
  return two ? 2 : 1;
}

template <class V, int BX>
void launch_slab(cbct_plan* p, const V* vol, const V* volT, const FwdOut& o, dim3 grid, int first,
                 cudaStream_t st, cbct_dtype dt) {
  const SlabBox& b = box_for<V>(p);
  const CUtensorMap mv = make_map(dt, vol, p->g.nx, p->g.ny, p->g.nz, b);
  const CUtensorMap mt = make_map(dt, volT ? (const void*)volT : (const void*)vol, volT ? p->g.ny : p->g.nx,
                                  volT ? p->g.nx : p->g.ny, p->g.nz, b);
  size_t smem = 0;
  const bool two = slab_stages<V>(b, smem) == 2;
  auto pick = [&](auto k2, auto k1) { return two ? k2 : k1; };
  auto k = p->debug_checks ? pick(fwd_slab_kernel<V, BX, true, 2>, fwd_slab_kernel<V, BX, true, 1>)
                           : pick(fwd_slab_kernel<V, BX, false, 2>, fwd_slab_kernel<V, BX, false, 1>);
  ensure_smem_attr((const void*)k, smem);
  k<<<grid, 256, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, o, p->d_flags);
  check_launch("fwd_slab_kernel");
}

template <class V>
const SlabBox& pair_box_for(const cbct_plan* p) { return sizeof(V) == 4 ? p->pair : p->pair16; }

template <class V, int BX>
void launch_pair(cbct_plan* p, const V* vol, const V* volT, const FwdOut& o, int first, int cnt, cudaStream_t st,
                 cbct_dtype dt) {
  const SlabBox& b = pair_box_for<V>(p);
  const CUtensorMap mv = make_map(dt, vol, p->g.nx, p->g.ny, p->g.nz, b);
  const CUtensorMap mt = make_map(dt, volT ? (const void*)volT : (const void*)vol, volT ? p->g.ny : p->g.nx,
                                  volT ? p->g.nx : p->g.ny, p->g.nz, b);
  const int nsl = slabs_max(p->g);
  const size_t smem = pair_smem(b, sizeof(V), nsl);
  const dim3 grid((p->g.width + kPU - 1) / kPU, (p->g.height + kPV - 1) / kPV, cnt);
  if (p->debug_checks) {
    auto k = fwd_pair_kernel<V, BX, true>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kPairThreads, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, nsl, o, p->d_flags);
  } else {
    auto k = fwd_pair_kernel<V, BX, false>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kPairThreads, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, nsl, o, p->d_flags);
  }
  check_launch("fwd_pair_kernel");
}

template <class V>
const SlabBox& quad_box_for(const cbct_plan* p) { return sizeof(V) == 4 ? p->quad : p->quad16; }

template <class V, int BX>
void launch_quad(cbct_plan* p, const V* vol, const V* volT, const FwdOut& o, int first, int cnt, cudaStream_t st,
                 cbct_dtype dt) {
  const SlabBox& b = quad_box_for<V>(p);
  const CUtensorMap mv = make_map(dt, vol, p->g.nx, p->g.ny, p->g.nz, b);
  const CUtensorMap mt = make_map(dt, volT ? (const void*)volT : (const void*)vol, volT ? p->g.ny : p->g.nx,
                                  volT ? p->g.nx : p->g.ny, p->g.nz, b);
  const int nsl = slabs_max(p->g);
  const size_t smem = pair_smem(b, sizeof(V), nsl);
  const dim3 grid((p->g.width + kQU - 1) / kQU, (p->g.height + kQV - 1) / kQV, cnt);
  if (p->debug_checks) {
    auto k = fwd_quad_kernel<V, BX, true>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kQuadThreads, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, nsl, o, p->d_flags);
  } else {
    auto k = fwd_quad_kernel<V, BX, false>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kQuadThreads, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, nsl, o, p->d_flags);
  }
  check_launch("fwd_quad_kernel");
}

template <class V>
const SlabBox& fan_box_for(const cbct_plan* p) { return sizeof(V) == 4 ? p->fan : p->fan16; }

template <class V, int BX>
void launch_fan(cbct_plan* p, const V* vol, const V* volT, const FwdOut& o, int first, int cnt, cudaStream_t st,
                cbct_dtype dt) {
  const SlabBox& b = fan_box_for<V>(p);
  const CUtensorMap mv = make_map(dt, vol, p->g.nx, p->g.ny, p->g.nz, b);
  const CUtensorMap mt = make_map(dt, volT ? (const void*)volT : (const void*)vol, volT ? p->g.ny : p->g.nx,
                                  volT ? p->g.nx : p->g.ny, p->g.nz, b);
  const int nsl = slabs_max(p->g);
  const size_t smem = forward_smem(b, sizeof(V), p->fan_lz, nsl);
  const dim3 grid((p->g.width + kFU - 1) / kFU, (p->g.height + kFV - 1) / kFV, cnt);
  if (p->debug_checks) {
    auto k = fwd_fan_kernel<V, BX, true>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kFU * 32, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, p->fan_lz, nsl, o, p->d_flags);
  } else {
    auto k = fwd_fan_kernel<V, BX, false>;
    ensure_smem_attr((const void*)k, smem);
    k<<<grid, kFU * 32, smem, st>>>(mv, mt, vol, p->d_views + first, p->gc, b.bz, p->fan_lz, nsl, o, p->d_flags);
  }
  check_launch("fwd_fan_kernel");
}

template <class V>
void launch_typed(cbct_plan* p, int s, const void* vol_v, const FwdOut& o, cudaStream_t st, cbct_dtype dt,
                  bool use_slab) {
  const V* vol = static_cast<const V*>(vol_v);
  const int first = p->first[s], cnt = p->count[s];
  dim3 grid((p->g.width + kTU - 1) / kTU, (p->g.height + kTV - 1) / kTV, cnt);
  if (!use_slab) {
    fwd_gather_kernel<V><<<grid, 256, 0, st>>>(vol, p->d_views + first, p->gc, o);
    check_launch("fwd_gather_kernel");
    return;
  }
  const V* volT = nullptr;
  if (p->subset_has_xdom[s]) {
    V* t = static_cast<V*>(p->d_volT);
    dim3 tg((p->g.nx + 31) / 32, (p->g.ny + 31) / 32, p->g.nz);
    transpose_xy_kernel<V><<<tg, dim3(32, 8), 0, st>>>(vol, t, p->g.nx, p->g.ny);
    check_launch("transpose_xy_kernel");
    volT = t;
  }
  if (p->fwd_variant == 4) {
    switch (quad_box_for<V>(p).bx) {
      case 40: launch_quad<V, 40>(p, vol, volT, o, first, cnt, st, dt); break;
      case 56: launch_quad<V, 56>(p, vol, volT, o, first, cnt, st, dt); break;
      case 72: launch_quad<V, 72>(p, vol, volT, o, first, cnt, st, dt); break;
      case 104: launch_quad<V, 104>(p, vol, volT, o, first, cnt, st, dt); break;
      case 136: launch_quad<V, 136>(p, vol, volT, o, first, cnt, st, dt); break;
      default: throw Error(CBCT_ERR_INTERNAL, "unsupported quad box width");
    }
    return;
  }
  if (p->fwd_variant == 3) {
    switch (pair_box_for<V>(p).bx) {
      case 40: launch_pair<V, 40>(p, vol, volT, o, first, cnt, st, dt); break;
      case 56: launch_pair<V, 56>(p, vol, volT, o, first, cnt, st, dt); break;
      case 72: launch_pair<V, 72>(p, vol, volT, o, first, cnt, st, dt); break;
      case 104: launch_pair<V, 104>(p, vol, volT, o, first, cnt, st, dt); break;
      case 136: launch_pair<V, 136>(p, vol, volT, o, first, cnt, st, dt); break;
      default: throw Error(CBCT_ERR_INTERNAL, "unsupported pair box width");
    }
    return;
  }
  if (p->fwd_variant == 2) {
    switch (fan_box_for<V>(p).bx) {
      case 24: launch_fan<V, 24>(p, vol, volT, o, first, cnt, st, dt); break;
      case 40: launch_fan<V, 40>(p, vol, volT, o, first, cnt, st, dt); break;
      case 56: launch_fan<V, 56>(p, vol, volT, o, first, cnt, st, dt); break;
      case 72: launch_fan<V, 72>(p, vol, volT, o, first, cnt, st, dt); break;
      default: throw Error(CBCT_ERR_INTERNAL, "unsupported fan box width");
    }
    return;
  }
  switch (box_for<V>(p).bx) {
    case 40: launch_slab<V, 40>(p, vol, volT, o, grid, first, st, dt); break;
    case 56: launch_slab<V, 56>(p, vol, volT, o, grid, first, st, dt); break;
    case 72: launch_slab<V, 72>(p, vol, volT, o, grid, first, st, dt); break;
    case 104: launch_slab<V, 104>(p, vol, volT, o, grid, first, st, dt); break;
    case 136: launch_slab<V, 136>(p, vol, volT, o, grid, first, st, dt); break;
    default: throw Error(CBCT_ERR_INTERNAL, "unsupported slab box width");
  }
}

template <class V, int BX>
void prepare_width(size_t smem) {
  ensure_smem_attr((const void*)fwd_slab_kernel<V, BX, false, 2>, smem);
  ensure_smem_attr((const void*)fwd_slab_kernel<V, BX, true, 2>, smem);
  ensure_smem_attr((const void*)fwd_slab_kernel<V, BX, false, 1>, smem);
  ensure_smem_attr((const void*)fwd_slab_kernel<V, BX, true, 1>, smem);
}

template <class V, int BX>
void prepare_quad_width(size_t smem) {
  ensure_smem_attr((const void*)fwd_quad_kernel<V, BX, false>, smem);
  ensure_smem_attr((const void*)fwd_quad_kernel<V, BX, true>, smem);
}

template <class V, int BX>
void prepare_pair_width(size_t smem) {
  ensure_smem_attr((const void*)fwd_pair_kernel<V, BX, false>, smem);
  ensure_smem_attr((const void*)fwd_pair_kernel<V, BX, true>, smem);
}

template <class V, int BX>
void prepare_fan_width(size_t smem) {
  ensure_smem_attr((const void*)fwd_fan_kernel<V, BX, false>, smem);
  ensure_smem_attr((const void*)fwd_fan_kernel<V, BX, true>, smem);
}

template <class V>
void prepare_typed(const cbct_plan* p) {
  if (p->fwd_variant == 4) {
    const SlabBox& b = quad_box_for<V>(p);
    const size_t qs = pair_smem(b, sizeof(V), slabs_max(p->g));
    switch (b.bx) {
      case 40: prepare_quad_width<V, 40>(qs); break;
      case 56: prepare_quad_width<V, 56>(qs); break;
      case 72: prepare_quad_width<V, 72>(qs); break;
      case 104: prepare_quad_width<V, 104>(qs); break;
      case 136: prepare_quad_width<V, 136>(qs); break;
      default: break;
    }
  }
  if (p->fwd_variant == 3) {
    const SlabBox& b = pair_box_for<V>(p);
    const size_t ps = pair_smem(b, sizeof(V), slabs_max(p->g));
    switch (b.bx) {
      case 40: prepare_pair_width<V, 40>(ps); break;
      case 56: prepare_pair_width<V, 56>(ps); break;
      case 72: prepare_pair_width<V, 72>(ps); break;
      case 104: prepare_pair_width<V, 104>(ps); break;
      case 136: prepare_pair_width<V, 136>(ps); break;
      default: break;
    }
  }
  if (p->fwd_variant == 2) {
    const SlabBox& f = fan_box_for<V>(p);
    const size_t fs = forward_smem(f, sizeof(V), p->fan_lz, slabs_max(p->g));
    switch (f.bx) {
      case 24: prepare_fan_width<V, 24>(fs); break;
      case 40: prepare_fan_width<V, 40>(fs); break;
      case 56: prepare_fan_width<V, 56>(fs); break;
      case 72: prepare_fan_width<V, 72>(fs); break;
      default: break;
    }
  }
  const SlabBox& b = box_for<V>(p);
  const size_t smem = forward_smem(b, sizeof(V), 0);
  switch (b.bx) {
    case 40: prepare_width<V, 40>(smem); break;
    case 56: prepare_width<V, 56>(smem); break;
    case 72: prepare_width<V, 72>(smem); break;
    case 104: prepare_width<V, 104>(smem); break;
    case 136: prepare_width<V, 136>(smem); break;
    default: break;
  }
}

}  // namespace

// Largest footprint of one slab over every view and tile of a TU x TV tiling
// (corner-ray bounding box in the view's frame, computed in FP64): e extent
// and z extent in elements, including margins.  False when some view cannot
// use slabs (a ray not dominated by its view's slab axis, or too many slabs).
static bool slab_extents(const cbct_plan* p, int TU, int TV, int& ext_e, int& ext_z) {
  const cbct_geometry& g = p->g;
  const double kx = g.nx / (double)g.lx, ky = g.ny / (double)g.ly, kz = g.nz / (double)g.lz;
  const double bx = g.nx / 2.0 - 0.5, by = g.ny / 2.0 - 0.5, bz = g.nz / 2.0 - 0.5;
  const int tiles_u = (g.width + TU - 1) / TU, tiles_v = (g.height + TV - 1) / TV;
  struct Acc { int e = 0, z = 0, ok = 1; };
  std::vector<Acc> acc(host_threads());
  // The in-plane coordinate of a ray does not depend on the detector row, so the
  // e extent is a function of (view, tile column, slab); the z extent comes from
  // the products t * dz at the extreme path parameters and rows of each tile.
  parallel_for(p->n_views, [&](int lo, int hi, int tid) {
    Acc& a = acc[tid];
    std::vector<double> dz0(tiles_v), dz1(tiles_v);
    for (int iv = lo; iv < hi && a.ok; ++iv) {
      const ViewParams& vp = p->hviews[iv];
      const int dom = vp.dom;
      const int Nd = dom ? g.ny : g.nx;
      const double ke = dom ? kx : ky, be = dom ? bx : by, kd = dom ? ky : kx, bd = dom ? by : bx;
      const double Se = dom ? vp.Sx : vp.Sy, Sd = dom ? vp.Sy : vp.Sx;
      const int nsl = (Nd + 1 - kSlabBase + kTS - 1) / kTS + 1;
      if (nsl > kMaxSlabs) { a.ok = 0; break; }
      for (int tv = 0; tv < tiles_v; ++tv) {
        const int v0 = tv * TV, ve = std::min(v0 + TV, g.height) - 1;
        dz0[tv] = vp.D0z + v0 * (double)vp.Evz;
        dz1[tv] = vp.D0z + ve * (double)vp.Evz;
      }
      for (int tu = 0; tu < tiles_u && a.ok; ++tu) {
        const int uc[2] = {tu * TU, std::min(tu * TU + TU, g.width) - 1};
        double de[2], dd[2];
        for (int c = 0; c < 2; ++c) {
          const double dx = vp.D0x + uc[c] * (double)vp.Eux, dy = vp.D0y + uc[c] * (double)vp.Euy;
          de[c] = dom ? dx : dy;
          dd[c] = dom ? dy : dx;
          // The slab axis must dominate every ray of the view with a uniform sign.
          if (dd[c] * vp.dsgn <= 0 || dd[c] * vp.dsgn < 0.25 * std::fabs(de[c])) a.ok = 0;
        }
        if (!a.ok) break;
        for (int m = 0; m < nsl; ++m) {
          double emn = 1e30, emx = -1e30, tmn = 1e30, tmx = -1e30;
          for (int c = 0; c < 4; ++c) {
            const double plane = kSlabBase + m * kTS + ((c & 2) ? kTS : 0);
            const double t = ((plane - bd) / kd - Sd) / dd[c & 1];
            const double ce = (Se + t * de[c & 1]) * ke + be;
            emn = std::min(emn, ce); emx = std::max(emx, ce);
            tmn = std::min(tmn, t); tmx = std::max(tmx, t);
          }
          // elements from floor(min)-1 to floor(max)+1 inclusive, +2 margin; the
          // kernels clamp footprints to the volume, whose extent bounds the box
          const int Ne = dom ? g.nx : g.ny;
          a.e = std::max(a.e, std::min((int)(std::floor(emx) - std::floor(emn)) + 3 + 2, Ne + 4));
          for (int tv = 0; tv < tiles_v; ++tv) {
            const double z00 = tmn * dz0[tv], z01 = tmn * dz1[tv], z10 = tmx * dz0[tv], z11 = tmx * dz1[tv];
            const double zmn = std::min(std::min(z00, z01), std::min(z10, z11)) * kz + bz;
            const double zmx = std::max(std::max(z00, z01), std::max(z10, z11)) * kz + bz;
            const int ez = (int)(std::floor(zmx) - std::floor(zmn)) + 3 + 2;
            a.z = std::max(a.z, std::min(ez, g.nz + 4));
          }
        }
      }
    }
  });
  ext_e = ext_z = 0;
  bool ok = true;
  for (const Acc& a : acc) {
    ext_e = std::max(ext_e, a.e);
    ext_z = std::max(ext_z, a.z);
    ok = ok && a.ok;
  }
  return ok;
}

// Largest z distance (texels) between the rays of adjacent detector rows at a
// point of the volume.  A point P lies at ray parameter t = (P - S).n / SDD,
// n the unit vector from the source towards the detector centre, so over the
// volume t <= (SAD + hx |sin| + hy |cos|) / SDD; rows are dv apart at t = 1.
static double row_dz_max(const cbct_plan* p) {
  const cbct_geometry& g = p->g;
  const double kz = g.nz / (double)g.lz, dv = double(g.fov_v) / g.height;
  double m = 0;
  for (int iv = 0; iv < p->n_views; ++iv) {
    const double th = double(p->angles[iv]) * (3.14159265358979323846 / 180.0);
    const double tmax = (g.SAD + 0.5 * g.lx * std::fabs(std::sin(th)) + 0.5 * g.ly * std::fabs(std::cos(th))) / g.SDD;
    m = std::max(m, tmax * dv * kz);
  }
  return m;
}

// Chooses the forward variant and its TMA boxes from the plan geometry: the
// row-pair kernel where adjacent detector rows are less than one z texel
// apart over the whole volume (so pairs share their planes) and its boxes fit,
// else the per-ray slab kernel where its boxes fit, else the gather kernel.
// CBCT_OPT_FORWARD_KERNEL forces slab (1), gather (2), fan (3) or pairs (4).
void forward_choose_variant(cbct_plan* p) {
  p->fwd_variant = 0;
  p->slab = SlabBox{0, 0, 0, 0};
  p->fan = SlabBox{0, 0, 0, 0};
  p->pair = p->pair16 = SlabBox{0, 0, 0, 0};
  p->quad = p->quad16 = SlabBox{0, 0, 0, 0};
  // Per view range (subsets, the all-views entry and bin segments).
  p->subset_has_xdom.assign(p->first.size(), 0);
  for (size_t s = 0; s < p->first.size(); ++s)
    for (int i = p->first[s]; i < p->first[s] + p->count[s]; ++i)
      if (p->hviews[i].dom == 0) p->subset_has_xdom[s] = 1;
  if (p->force_gather || p->fwd_pref == 2) return;
  // The x start of a box is rounded down to a 16-byte boundary (4 fp32 or 8
  // 16-bit elements), which widens the box by up to 3 or 7 elements.
  auto width = [](const auto& list, int ext, int slack) {
    for (int w : list)
      if (w >= ext + slack) return w;
    return 0;
  };
  int e, z;
  if (slab_extents(p, kTU, kTV, e, z)) {
    const int w32 = width(kBoxWidths, e, 3), w16 = width(kBoxWidths, e, 7);
    const int boxz = std::max(z, 2);
    const SlabBox b32{w32, kBoxY, boxz, 1}, b16{w16, kBoxY, boxz, 1};
    if (w32 && w16 && boxz <= 256 && forward_smem(b32, 4, 0) <= (size_t)kSmemBudget &&
        forward_smem(b16, 2, 0) <= (size_t)kSmemBudget) {
      p->slab = b32;
      p->slab16 = b16;
      p->slab_smem = forward_smem(b32, 4, 0);
      p->fwd_variant = 1;
    }
  }
  const double row_dz = row_dz_max(p);
  if ((p->fwd_pref == 4 || (p->fwd_pref == 0 && p->fwd_variant == 1 && row_dz < 0.99)) &&
      slab_extents(p, kPU, kPV, e, z)) {
    const int w32 = width(kBoxWidths, e, 3), w16 = width(kBoxWidths, e, 7);
    const int boxz = std::max(z, 3);
    const SlabBox b32{w32, kPairBoxY, boxz, 1}, b16{w16, kPairBoxY, boxz, 1};
    const int nsl = slabs_max(p->g);
    if (w32 && w16 && boxz <= 256 && pair_smem(b32, 4, nsl) <= (size_t)kSmemBudget &&
        pair_smem(b16, 2, nsl) <= (size_t)kSmemBudget) {
      p->pair = b32;
      p->pair16 = b16;
      p->fwd_variant = 3;
    }
  }
  // Row quads where four adjacent rows stay within two z texels (3 row steps
  // under 0.66 texel each, margin included).
  if ((p->fwd_pref == 5 || (p->fwd_pref == 0 && p->fwd_variant == 3 && row_dz < 0.66)) &&
      slab_extents(p, kQU, kQV, e, z)) {
    const int w32 = width(kBoxWidths, e, 3), w16 = width(kBoxWidths, e, 7);
    const int boxz = std::max(z, 4);
    const SlabBox b32{w32, kQuadBoxY, boxz, 1}, b16{w16, kQuadBoxY, boxz, 1};
    const int nsl = slabs_max(p->g);
    if (w32 && w16 && boxz <= 256 && pair_smem(b32, 4, nsl) <= (size_t)kSmemBudget &&
        pair_smem(b16, 2, nsl) <= (size_t)kSmemBudget) {
      p->quad = b32;
      p->quad16 = b16;
      p->fwd_variant = 4;
    }
  }
  if (p->fwd_pref == 3 && slab_extents(p, kFU, kFV, e, z)) {
    const int w32 = width(kFanWidths, e, 3), w16 = width(kFanWidths, e, 7);
    const int boxz = std::max(z, 2);
    const int lz = (boxz + 1) | 1;  // odd: consecutive lines start in different banks
    const SlabBox b32{w32, kBoxY, boxz, 1}, b16{w16, kBoxY, boxz, 1};
    const int nsl = slabs_max(p->g);
    if (w32 && w16 && boxz <= 256 && forward_smem(b32, 4, lz, nsl) <= (size_t)kSmemBudget &&
        forward_smem(b16, 2, lz, nsl) <= (size_t)kSmemBudget) {
      p->fan = b32;
      p->fan16 = b16;
      p->fan_lz = lz;
      p->fwd_variant = 2;
    }
  }
}

void forward_prepare(cbct_plan* p) {
  if (p->fwd_variant < 1) return;
  prepare_typed<float>(p);
  prepare_typed<__half>(p);
  prepare_typed<__nv_bfloat16>(p);
  bool any_x = false;
  for (size_t s = 0; s < p->subset_has_xdom.size(); ++s) any_x = any_x || p->subset_has_xdom[s];
  if (any_x && !p->d_volT)
    p->d_volT = plan_alloc_n<float>(p, (size_t)p->g.nx * p->g.ny * p->g.nz);
}

void forward_launch(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out, const float* b,
                    float scale, int mode, int apply_offset, int accumulate, double* norm2_out,
                    cudaStream_t st) {
  forward_launch_ex(p, s, dt, vol, out, b, nullptr, scale, mode, apply_offset, accumulate, norm2_out, st);
}

void forward_launch_ex(cbct_plan* p, int s, cbct_dtype dt, const void* vol, float* out, const void* b,
                       const float* pw, float scale, int mode, int apply_offset, int accumulate,
                       double* norm2_out, cudaStream_t st, cbct_dtype b_dtype) {
  FwdOut o;
  o.out = out;
  o.pw = pw;
  o.b = b;
  o.b_dtype = b_dtype;
  o.scale = scale;
  o.mode = mode;
  o.apply_offset = apply_offset;
  o.accumulate = accumulate;
  o.partials = nullptr;
  const int cnt = p->count[s];
  if (cnt == 0) return;
  o.wproj = p->d_pweights ? p->d_pweights + (size_t)p->g.width * p->g.height * p->first[s] : nullptr;
  const size_t es = dtype_size(dt);
  const bool use_slab = p->fwd_variant >= 1 && ((size_t)p->g.nx * es) % 16 == 0 &&
                        ((size_t)p->g.ny * es) % 16 == 0 && (reinterpret_cast<uintptr_t>(vol) % 16 == 0) &&
                        (!p->subset_has_xdom[s] || p->d_volT != nullptr);
  // One partial sum per block of the kernel that will run.
  const bool fan = use_slab && p->fwd_variant == 2, pair = use_slab && p->fwd_variant == 3;
  const bool quad = use_slab && p->fwd_variant == 4;
  const int TU = fan ? kFU : pair ? kPU : quad ? kQU : kTU, TV = fan ? kFV : pair ? kPV : quad ? kQV : kTV;
  const size_t nblocks = (size_t)((p->g.width + TU - 1) / TU) * ((p->g.height + TV - 1) / TV) * cnt;
  if (norm2_out) {
    if (nblocks > p->n_partials) throw Error(CBCT_ERR_INTERNAL, "partials buffer too small");
    o.partials = p->d_partials;
  }
  switch (dt) {
    case CBCT_F32: launch_typed<float>(p, s, vol, o, st, dt, use_slab); break;
    case CBCT_F16: launch_typed<__half>(p, s, vol, o, st, dt, use_slab); break;
    case CBCT_BF16: launch_typed<__nv_bfloat16>(p, s, vol, o, st, dt, use_slab); break;
    default: throw Error(CBCT_ERR_INVALID_ARGUMENT, "unknown volume dtype");
  }
  if (norm2_out) finalize_partials(p->d_partials, (int)nblocks, norm2_out, st);
}

namespace {

template <int VAR, int BX>
void add_fwd_group(WorkArena& A, const std::vector<FwdScanRec>& recs, int total, size_t smem) {
  auto k = fwd_multi_kernel<VAR, float, BX>;
  ensure_smem_attr((const void*)k, smem);
  const size_t off = A.add(recs.data(), recs.size() * sizeof(FwdScanRec));
  const int ci = A.n_counters++;
  const int threads = var_threads<VAR>();
  const int grid = std::min(total, resident_grid((const void*)k, threads, smem));
  const int n = (int)recs.size();
  A.ops.push_back([&A, k, off, ci, grid, threads, n, total, smem](cudaStream_t st) {
    k<<<grid, threads, smem, st>>>(reinterpret_cast<const FwdScanRec*>(A.dev + off), n, total, A.counter(ci));
    check_launch("fwd_multi_kernel");
  });
}

template <int VAR>
const void* fwd_multi_ptr_v(int c) {
  switch (kBoxWidths[c]) {
    case 40: return (const void*)fwd_multi_kernel<VAR, float, 40>;
    case 56: return (const void*)fwd_multi_kernel<VAR, float, 56>;
    case 72: return (const void*)fwd_multi_kernel<VAR, float, 72>;
    case 104: return (const void*)fwd_multi_kernel<VAR, float, 104>;
    case 136: return (const void*)fwd_multi_kernel<VAR, float, 136>;
    default: throw Error(CBCT_ERR_INTERNAL, "unsupported forward box width");
  }
}

const void* fwd_multi_ptr(int var, int c) {
  return var == kVarSlab1 ? fwd_multi_ptr_v<kVarSlab1>(c) : var == kVarSlab2 ? fwd_multi_ptr_v<kVarSlab2>(c)
         : var == kVarPair ? fwd_multi_ptr_v<kVarPair>(c) : fwd_multi_ptr_v<kVarQuad>(c);
}

int var_threads_of(int var) {
  return var == kVarPair ? var_threads<kVarPair>() : var == kVarQuad ? var_threads<kVarQuad>() : 256;
}

template <int VAR>
void add_fwd_group_w(WorkArena& A, int c, const std::vector<FwdScanRec>& g, int total, size_t smem) {
  switch (kBoxWidths[c]) {
    case 40: add_fwd_group<VAR, 40>(A, g, total, smem); break;
    case 56: add_fwd_group<VAR, 56>(A, g, total, smem); break;
    case 72: add_fwd_group<VAR, 72>(A, g, total, smem); break;
    case 104: add_fwd_group<VAR, 104>(A, g, total, smem); break;
    case 136: add_fwd_group<VAR, 136>(A, g, total, smem); break;
    default: throw Error(CBCT_ERR_INTERNAL, "unsupported forward box width");
  }
}

}  // namespace

void forward_multi(WorkArena& A, const std::vector<MultiFwdJob>& jobs) {
  std::vector<FwdScanRec> groups[4][5];
  int totals[4][5] = {};
  size_t smem[4][5] = {};
  // Transposes of the volumes the next launches read, one launch for all.
  std::vector<TransposeRec> tr;
  int tr_total = 0;
  auto flush_transposes = [&]() {
    if (tr.empty()) return;
    const size_t off = A.add(tr.data(), tr.size() * sizeof(TransposeRec));
    const int n = (int)tr.size(), total = tr_total;
    A.ops.push_back([&A, off, n, total](cudaStream_t st) {
      transpose_multi_kernel<<<total, dim3(32, 8), 0, st>>>(reinterpret_cast<const TransposeRec*>(A.dev + off), n);
      check_launch("transpose_multi_kernel");
    });
    tr.clear();
    tr_total = 0;
  };
  auto flush = [&](int v, int c) {
    if (groups[v][c].empty()) return;
    flush_transposes();
    if (v == kVarSlab1) add_fwd_group_w<kVarSlab1>(A, c, groups[v][c], totals[v][c], smem[v][c]);
    else if (v == kVarSlab2) add_fwd_group_w<kVarSlab2>(A, c, groups[v][c], totals[v][c], smem[v][c]);
    else if (v == kVarPair) add_fwd_group_w<kVarPair>(A, c, groups[v][c], totals[v][c], smem[v][c]);
    else add_fwd_group_w<kVarQuad>(A, c, groups[v][c], totals[v][c], smem[v][c]);
    groups[v][c].clear();
    totals[v][c] = 0;
    smem[v][c] = 0;
  };
  std::vector<std::function<void(cudaStream_t)>> after;
  for (const MultiFwdJob& j : jobs) {
    cbct_plan* p = j.p;
    const int s = j.s, first = p->first[s], cnt = p->count[s];
    if (cnt == 0) continue;
    const bool tma = p->fwd_variant >= 1 && ((size_t)p->g.nx * 4) % 16 == 0 && ((size_t)p->g.ny * 4) % 16 == 0 &&
                     (reinterpret_cast<uintptr_t>(j.vol) % 16 == 0) && (!p->subset_has_xdom[s] || p->d_volT);
    const int fv = p->fwd_variant;
    auto one_scan = [&A](const MultiFwdJob& jj) {
      A.ops.push_back([jj](cudaStream_t st) {
        forward_launch_ex(jj.p, jj.s, CBCT_F32, jj.vol, jj.out, jj.b, nullptr, 1.f, kModeResidual, jj.apply_offset,
                          0, jj.norm2_out, st, jj.b_dtype);
      });
    };
    if (!tma || fv == 2 || p->debug_checks) {
      one_scan(j);
      continue;
    }
    const int nsl = slabs_max(p->g);
    int var, TU, TV;
    SlabBox b;
    size_t sm = 0;
    if (fv == 4) {
      b = p->quad; var = kVarQuad; TU = kQU; TV = kQV; sm = pair_smem(b, 4, nsl);
    } else if (fv == 3) {
      b = p->pair; var = kVarPair; TU = kPU; TV = kPV; sm = pair_smem(b, 4, nsl);
    } else {
      b = p->slab; TU = kTU; TV = kTV;
      var = slab_stages<float>(b, sm) == 2 ? kVarSlab2 : kVarSlab1;
    }
    int w = -1;
    for (int c = 0; c < 5; ++c)
      if (kBoxWidths[c] == b.bx) w = c;
    if (w < 0) throw Error(CBCT_ERR_INTERNAL, "unsupported forward box width");
    const int tx = (p->g.width + TU - 1) / TU, ty = (p->g.height + TV - 1) / TV;
    const int nblocks = tx * ty * cnt;
    {
      const void* kfn = fwd_multi_ptr(var, w);
      ensure_smem_attr(kfn, sm);
      if (nblocks >= kMultiFillWaves * resident_grid(kfn, var_threads_of(var), sm)) {
        one_scan(j);
        continue;
      }
    }
    const float* volT = nullptr;
    if (p->subset_has_xdom[s]) {
      float* t = static_cast<float*>(p->d_volT);
      if ((int)tr.size() == kMultiMaxRecs) flush_transposes();
      TransposeRec q{j.vol, t, p->g.nx, p->g.ny, (p->g.nx + 31) / 32, (p->g.ny + 31) / 32, tr_total};
      tr_total += q.tx * q.ty * p->g.nz;
      tr.push_back(q);
      volT = t;
    }
    FwdOut o{};
    o.out = j.out;
    o.b = j.b;
    o.b_dtype = j.b_dtype;
    o.pw = nullptr;
    o.scale = 1.f;
    o.mode = kModeResidual;
    o.apply_offset = j.apply_offset;
    o.accumulate = 0;
    o.partials = nullptr;
    o.wproj = p->d_pweights ? p->d_pweights + (size_t)p->g.width * p->g.height * first : nullptr;
    FwdScanRec r;
    std::memset(&r, 0, sizeof(r));
    r.map_v = make_map(CBCT_F32, j.vol, p->g.nx, p->g.ny, p->g.nz, b);
    r.map_t = make_map(CBCT_F32, volT ? (const void*)volT : (const void*)j.vol, volT ? p->g.ny : p->g.nx,
                       volT ? p->g.nx : p->g.ny, p->g.nz, b);
    r.vol = j.vol;
    r.views = p->d_views + first;
    r.flags = p->d_flags;
    r.gc = p->gc;
    r.BZ = b.bz;
    r.nsl_max = nsl;
    r.tx = tx;
    r.ty = ty;
    if (j.norm2_out) {
      if ((size_t)nblocks > p->n_partials) throw Error(CBCT_ERR_INTERNAL, "partials buffer too small");
      o.partials = p->d_partials;
      double* part = p->d_partials;
      double* out = j.norm2_out;
      after.push_back([part, nblocks, out](cudaStream_t st) { finalize_partials(part, nblocks, out, st); });
    }
    r.o = o;
    if ((int)groups[var][w].size() == kMultiMaxRecs) flush(var, w);
    r.base = totals[var][w];
    totals[var][w] += nblocks;
    smem[var][w] = std::max(smem[var][w], sm);
    groups[var][w].push_back(r);
  }
  for (int v = 0; v < 4; ++v)
    for (int c = 0; c < 5; ++c) flush(v, c);
  flush_transposes();
  for (auto& f : after) A.ops.push_back(std::move(f));
}

}  // namespace cbct
