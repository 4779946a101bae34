// phantom.cu -- seeded ellipsoid phantoms on the device.
//
// Synthetic inputs for the benchmarks and tests: a sum of ellipsoids,
// voxelised with supersampling, and its exact line integrals along the rays
// of a plan (source to detector-pixel centre, clipped to the volume box as
// conebeam_projection.cu:478-484 clips), so that measured data are not made
// by the projector under test.
//
// Ellipsoid record (10 floats): cx cy cz ax ay az phi theta psi density.
// R = Rz(phi) Ry(theta) Rx(psi); a point q is inside when
// |diag(1/a) R^T (q - c)| <= 1.
#include "device_common.cuh"

namespace cbct {

namespace {

struct Ell {
  double c[3];
  double inva[3];
  double R[9];
  double rho;
  double rmax2;  // squared bounding radius
};

__device__ void ell_load(const float* e, Ell& E) {
  const double cp = cos((double)e[6]), sp = sin((double)e[6]);
  const double ct = cos((double)e[7]), st = sin((double)e[7]);
  const double cs = cos((double)e[8]), ss = sin((double)e[8]);
  E.R[0] = cp * ct; E.R[1] = cp * st * ss - sp * cs; E.R[2] = cp * st * cs + sp * ss;
  E.R[3] = sp * ct; E.R[4] = sp * st * ss + cp * cs; E.R[5] = sp * st * cs - cp * ss;
  E.R[6] = -st;     E.R[7] = ct * ss;                E.R[8] = ct * cs;
  for (int i = 0; i < 3; ++i) {
    E.c[i] = e[i];
    E.inva[i] = 1.0 / (double)e[3 + i];
  }
  E.rho = e[9];
  const double am = fmax(fmax((double)e[3], (double)e[4]), (double)e[5]);
  E.rmax2 = am * am;
}

constexpr int kMaxEllSmem = 256;

__global__ void voxelize_kernel(const float* __restrict__ ell, int K, GridConst gc, int ss,
                                float* __restrict__ vol) {
  __shared__ Ell se[kMaxEllSmem];
  const size_t n = (size_t)gc.nx * gc.ny * gc.nz;
  const double hv = 0.5 * sqrt((double)gc.vx * gc.vx + (double)gc.vy * gc.vy + (double)gc.vz * gc.vz);
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x, base = blockIdx.x * (size_t)blockDim.x;
       base < n; idx += (size_t)gridDim.x * blockDim.x, base += (size_t)gridDim.x * blockDim.x) {
    const bool valid = idx < n;
    const int i = valid ? int(idx % gc.nx) : 0;
    const int j = valid ? int((idx / gc.nx) % gc.ny) : 0;
    const int k = valid ? int(idx / ((size_t)gc.nx * gc.ny)) : 0;
    const double px = (i + 0.5) * gc.vx - gc.hx, py = (j + 0.5) * gc.vy - gc.hy, pz = (k + 0.5) * gc.vz - gc.hz;
    double acc = 0.0;
    for (int e0 = 0; e0 < K; e0 += kMaxEllSmem) {
      const int ne = min(kMaxEllSmem, K - e0);
      __syncthreads();
      for (int q = threadIdx.x; q < ne; q += blockDim.x) ell_load(ell + 10 * (e0 + q), se[q]);
      __syncthreads();
      if (!valid) continue;
      for (int q = 0; q < ne; ++q) {
        const Ell& E = se[q];
        const double dx = px - E.c[0], dy = py - E.c[1], dz = pz - E.c[2];
        const double rb = sqrt(E.rmax2) + hv;
        if (dx * dx + dy * dy + dz * dz > rb * rb) continue;
        int hits = 0;
        for (int sz = 0; sz < ss; ++sz)
          for (int sy = 0; sy < ss; ++sy)
            for (int sx = 0; sx < ss; ++sx) {
              const double qx = dx + ((sx + 0.5) / ss - 0.5) * gc.vx;
              const double qy = dy + ((sy + 0.5) / ss - 0.5) * gc.vy;
              const double qz = dz + ((sz + 0.5) / ss - 0.5) * gc.vz;
              const double l0 = (E.R[0] * qx + E.R[3] * qy + E.R[6] * qz) * E.inva[0];
              const double l1 = (E.R[1] * qx + E.R[4] * qy + E.R[7] * qz) * E.inva[1];
              const double l2 = (E.R[2] * qx + E.R[5] * qy + E.R[8] * qz) * E.inva[2];
              hits += (l0 * l0 + l1 * l1 + l2 * l2 <= 1.0);
            }
        acc += E.rho * hits;
      }
    }
    if (valid) vol[idx] = float(acc / double(ss * ss * ss));
  }
}

__global__ void project_kernel(const float* __restrict__ ell, int K, const ViewParams* __restrict__ views,
                               int n_views, GridConst gc, float* __restrict__ proj) {
  __shared__ Ell se[kMaxEllSmem];
  const size_t n = (size_t)gc.W * gc.H * n_views;
  for (size_t base = blockIdx.x * (size_t)blockDim.x; base < n; base += (size_t)gridDim.x * blockDim.x) {
    const size_t idx = base + threadIdx.x;
    const bool valid = idx < n;
    const int u = valid ? int(idx % gc.W) : 0;
    const int v = valid ? int((idx / gc.W) % gc.H) : 0;
    const int p = valid ? int(idx / ((size_t)gc.W * gc.H)) : 0;
    const ViewParams vp = views[p];
    const double d[3] = {vp.D0x + u * (double)vp.Eux, vp.D0y + u * (double)vp.Euy, vp.D0z + v * (double)vp.Evz};
    const double S[3] = {vp.Sx, vp.Sy, 0.0};
    const double h[3] = {gc.hx, gc.hy, gc.hz};
    double a1 = 0.0, a2 = 1.0;
    for (int a = 0; a < 3; ++a) {
      const double t1 = (h[a] - S[a]) / d[a], t2 = (-h[a] - S[a]) / d[a];
      a1 = fmax(a1, fmin(t1, t2));
      a2 = fmin(a2, fmax(t1, t2));
    }
    const double dl = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double acc = 0.0;
    for (int e0 = 0; e0 < K; e0 += kMaxEllSmem) {
      const int ne = min(kMaxEllSmem, K - e0);
      __syncthreads();
      for (int q = threadIdx.x; q < ne; q += blockDim.x) ell_load(ell + 10 * (e0 + q), se[q]);
      __syncthreads();
      if (!valid || !(a2 > a1)) continue;
      for (int q = 0; q < ne; ++q) {
        const Ell& E = se[q];
        const double qx = S[0] - E.c[0], qy = S[1] - E.c[1], qz = S[2] - E.c[2];
        const double s0 = (E.R[0] * qx + E.R[3] * qy + E.R[6] * qz) * E.inva[0];
        const double s1 = (E.R[1] * qx + E.R[4] * qy + E.R[7] * qz) * E.inva[1];
        const double s2 = (E.R[2] * qx + E.R[5] * qy + E.R[8] * qz) * E.inva[2];
        const double d0 = (E.R[0] * d[0] + E.R[3] * d[1] + E.R[6] * d[2]) * E.inva[0];
        const double d1 = (E.R[1] * d[0] + E.R[4] * d[1] + E.R[7] * d[2]) * E.inva[1];
        const double d2 = (E.R[2] * d[0] + E.R[5] * d[1] + E.R[8] * d[2]) * E.inva[2];
        const double A = d0 * d0 + d1 * d1 + d2 * d2;
        const double B = s0 * d0 + s1 * d1 + s2 * d2;
        const double C = s0 * s0 + s1 * s1 + s2 * s2 - 1.0;
        const double disc = B * B - A * C;
        if (disc <= 0.0) continue;
        const double sq = sqrt(disc);
        const double t0 = fmax((-B - sq) / A, a1), t1 = fmin((-B + sq) / A, a2);
        if (t1 > t0) acc += E.rho * (t1 - t0) * dl;
      }
    }
    if (valid) proj[idx] = float(acc);
  }
}

}  // namespace

void phantom_voxelize_launch(const GridConst& gc, const float* ell, int K, int ss, float* vol, cudaStream_t st) {
  const size_t n = (size_t)gc.nx * gc.ny * gc.nz;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 32);
  voxelize_kernel<<<blocks, 256, 0, st>>>(ell, K, gc, ss, vol);
  check_launch("voxelize_kernel");
}

void phantom_project_launch(cbct_plan* p, int s, const float* ell, int K, float* proj, cudaStream_t st) {
  const size_t n = (size_t)p->g.width * p->g.height * p->count[s];
  if (n == 0) return;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 32);
  project_kernel<<<blocks, 256, 0, st>>>(ell, K, p->d_views + p->first[s], p->count[s], p->gc, proj);
  check_launch("project_kernel");
}

}  // namespace cbct
