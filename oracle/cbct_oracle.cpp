// cbct_oracle.cpp -- CPU restatement of gt-tomography's cone-beam hot path.
//
// TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA library
// (gt-tomography_b200/csrc): tests, the smoke entry and the CPU-baseline leg of
// bench.py call it.  The product path never links or calls it.
//
// Parity status: UNPINNED against the reference's own outputs.  The reference
// (xray/conebeam_projection.cu) cannot be built here: it needs the Gadgetron
// toolbox, Boost and HDF5 (none installed) and uses legacy texture references
// that CUDA 12 removed.  The reference ships no tests, golden vectors or
// fixtures for this path.  The restatement below is therefore pinned only by
// closed-form known answers (analytic ellipsoid line integrals, uniform
// volumes, single-voxel cases) and by self-consistency fixtures.
//
// Every routine is templated on the arithmetic type T: T=double is the FP64
// oracle, T=float is the OpenMP CPU baseline of the same algorithm.
// Interpolation modes: 0 = exact trilinear/bilinear (CUDA texture semantics:
// normalised coordinates, texel coordinate x*N-0.5, border texels = 0);
// 1 = texture-emulating (fractional weights rounded to 8 fractional bits, as
// CUDA's 9-bit fixed-point linear filtering does).
//
// Build: see oracle/build.py (g++ -O3 -fopenmp -shared -fPIC).

#include <algorithm>
#include <array>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>
#include <omp.h>

namespace {

constexpr double kPi = 3.14159265358979323846;

// Plain geometry block shared with the Python wrapper (oracle/oracle.py).
struct Geom {
  int nx, ny, nz;          // volume size in voxels (x fastest)
  double lx, ly, lz;       // volume size in mm (is_dims_in_mm)
  int W, H;                // detector size in pixels (u fastest)
  double fov_u, fov_v;     // detector size in mm (CBCT_geometry::FOV)
  double SAD, SDD;         // source-axis and source-detector distance in mm
};

template <class T>
inline T quantise_weight(T a, int mode) {
  if (mode == 1) return std::nearbyint(a * T(256)) / T(256);
  return a;
}

// Trilinear fetch at texel coordinates (cx,cy,cz) with border value 0.
// Follows the tex3D(image_tex, ...) fetch of conebeam_projection.cu:518
// (linear filter, cudaAddressModeBorder, conebeam_projection.cu:35-36).
template <class T, class V>
inline T fetch3(const V* vol, int nx, int ny, int nz, T cx, T cy, T cz, int mode) {
  T fx = std::floor(cx), fy = std::floor(cy), fz = std::floor(cz);
  long ix = (long)fx, iy = (long)fy, iz = (long)fz;
  T ax = quantise_weight<T>(cx - fx, mode);
  T ay = quantise_weight<T>(cy - fy, mode);
  T az = quantise_weight<T>(cz - fz, mode);
  T acc = 0;
  for (int dz = 0; dz < 2; ++dz) {
    long z = iz + dz;
    if (z < 0 || z >= nz) continue;
    T wz = dz ? az : T(1) - az;
    for (int dy = 0; dy < 2; ++dy) {
      long y = iy + dy;
      if (y < 0 || y >= ny) continue;
      T wy = dy ? ay : T(1) - ay;
      const V* row = vol + ((size_t)z * ny + y) * nx;
      for (int dx = 0; dx < 2; ++dx) {
        long x = ix + dx;
        if (x < 0 || x >= nx) continue;
        T wx = dx ? ax : T(1) - ax;
        acc += wz * wy * wx * T(row[x]);
      }
    }
  }
  return acc;
}

// Bilinear fetch on one detector layer, border 0 (tex2DLayered at
// conebeam_projection.cu:1029, texture declared at :38-39).
template <class T, class V>
inline T fetch2(const V* img, int W, int H, T cu, T cv, int mode) {
  T fu = std::floor(cu), fv = std::floor(cv);
  long iu = (long)fu, iv = (long)fv;
  T au = quantise_weight<T>(cu - fu, mode);
  T av = quantise_weight<T>(cv - fv, mode);
  T acc = 0;
  for (int dv = 0; dv < 2; ++dv) {
    long v = iv + dv;
    if (v < 0 || v >= H) continue;
    T wv = dv ? av : T(1) - av;
    for (int du = 0; du < 2; ++du) {
      long u = iu + du;
      if (u < 0 || u >= W) continue;
      T wu = du ? au : T(1) - au;
      acc += wv * wu * T(img[(size_t)v * W + u]);
    }
  }
  return acc;
}

// Ray of detector pixel (u,v) in view p: source S and direction d = E - S.
// Restates conebeam_projection.cu:441-473 (rotation from float3x3.h:54-63).
template <class T>
inline void ray_of(const Geom& g, T th, T ox, T oy, int u, int v, T S[3], T d[3]) {
  T c = std::cos(th), s = std::sin(th);
  S[0] = T(g.SAD) * s;
  S[1] = -T(g.SAD) * c;
  S[2] = 0;
  T q = ((T(u) + T(0.5)) / T(g.W) - T(0.5)) * T(g.fov_u) + ox;
  T r = ((T(v) + T(0.5)) / T(g.H) - T(0.5)) * T(g.fov_v) + oy;
  T add = T(g.SDD) - T(g.SAD);
  T E[3] = {c * q - s * add, s * q + c * add, r};
  for (int i = 0; i < 3; ++i) d[i] = E[i] - S[i];
}

// Clip parameters a1 (entry, >=0) and a2 (exit, <=1) of the ray against the
// volume box (conebeam_projection.cu:478-484).
template <class T>
inline void clip_box(const Geom& g, const T S[3], const T d[3], T& a1, T& a2) {
  T L[3] = {T(g.lx), T(g.ly), T(g.lz)};
  T mx = -INFINITY, mn = INFINITY;
  for (int i = 0; i < 3; ++i) {
    T thi = (L[i] / 2 - S[i]) / d[i];
    T tlo = (-L[i] / 2 - S[i]) / d[i];
    mx = std::max(mx, std::min(thi, tlo));
    mn = std::min(mn, std::max(thi, tlo));
  }
  a1 = std::max(mx, T(0));
  a2 = std::min(mn, T(1));
}

inline int samples_per_ray(const Geom& g, double spp) {
  // conebeam_projection.cu:625 passes samples_per_pixel*float(matrix_size_x)
  // into an int parameter: truncation toward zero.
  return (int)(float(spp) * float(g.nx));
}

// Forward projection (mult_M): conebeam_forwards_projection_kernel,
// conebeam_projection.cu:412-528.
template <class T, class V>
void forward(const Geom& g, const float* angles, const float* offs, int P, double spp,
             int mode, const V* vol, V* proj, int accumulate) {
  const int N = samples_per_ray(g, spp);
  const T L[3] = {T(g.lx), T(g.ly), T(g.lz)};
  const T NN[3] = {T(g.nx), T(g.ny), T(g.nz)};
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int p = 0; p < P; ++p) {
    for (int v = 0; v < g.H; ++v) {
      const T th = T(angles[p]) * T(kPi / 180.0);
      for (int u = 0; u < g.W; ++u) {
        T S[3], d[3];
        ray_of<T>(g, th, T(offs[2 * p]), T(offs[2 * p + 1]), u, v, S, d);
        T a1, a2;
        clip_box<T>(g, S, d, a1, a2);
        T len2 = 0;
        for (int i = 0; i < 3; ++i) len2 += ((a2 - a1) * d[i]) * ((a2 - a1) * d[i]);
        const T delta = std::sqrt(len2) / T(N);
        T c0[3], dc[3];
        for (int i = 0; i < 3; ++i) {
          T p0 = (S[i] + a1 * d[i]) / L[i] + T(0.5);          // normalised start
          T st = d[i] / L[i] * ((a2 - a1) / T(N));             // normalised step
          c0[i] = p0;
          dc[i] = st;
        }
        T acc = 0;
        for (int k = 0; k < N; ++k) {
          T cx = (c0[0] + dc[0] * T(k)) * NN[0] - T(0.5);
          T cy = (c0[1] + dc[1] * T(k)) * NN[1] - T(0.5);
          T cz = (c0[2] + dc[2] * T(k)) * NN[2] - T(0.5);
          acc += fetch3<T, V>(vol, g.nx, g.ny, g.nz, cx, cy, cz, mode);
        }
        size_t idx = ((size_t)p * g.H + v) * g.W + u;
        T out = acc * delta;
        if (accumulate) proj[idx] = V(T(proj[idx]) + out);
        else proj[idx] = V(out);
      }
    }
  }
}

// Back-projection (mult_MH): conebeam_backwards_projection_kernel<FBP>,
// conebeam_projection.cu:922-1037.  fbp selects the FDK distance weight of
// :1009-1024 (U = (SAD + r sin(beta - phi))/SAD, weight 1/U^2).
template <class T, class V>
void backproject(const Geom& g, const float* angles, const float* offs, int P, int fbp,
                 int mode, const V* proj, V* vol, int accumulate) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < g.nz; ++k) {
    for (int j = 0; j < g.ny; ++j) {
      for (int i = 0; i < g.nx; ++i) {
        const T x = ((T(i) + T(0.5)) / T(g.nx) - T(0.5)) * T(g.lx);
        const T y = ((T(j) + T(0.5)) / T(g.ny) - T(0.5)) * T(g.ly);
        const T z = ((T(k) + T(0.5)) / T(g.nz) - T(0.5)) * T(g.lz);
        T acc = 0;
        for (int p = 0; p < P; ++p) {
          const T th = T(angles[p]) * T(kPi / 180.0);
          const T c = std::cos(th), s = std::sin(th);
          const T xr = c * x + s * y;             // Rz(-theta) * pos
          const T yr = -s * x + c * y;
          const T dy = yr + T(g.SAD);
          const T ex = T(g.SDD) * (xr / dy) - T(offs[2 * p]);
          const T ez = T(g.SDD) * (z / dy) - T(offs[2 * p + 1]);
          const T cu = (ex / T(g.fov_u) + T(0.5)) * T(g.W) - T(0.5);
          const T cv = (ez / T(g.fov_v) + T(0.5)) * T(g.H) - T(0.5);
          T w = 1;
          if (fbp) {
            const T r = std::hypot(x, y);
            const T phi = std::atan2(y, x);
            const T ym = r * std::sin(th - phi);
            const T U = (T(g.SAD) + ym) / T(g.SAD);
            w = T(1) / (U * U);
          }
          acc += w * fetch2<T, V>(proj + (size_t)p * g.W * g.H, g.W, g.H, cu, cv, mode);
        }
        size_t idx = ((size_t)k * g.ny + j) * g.nx + i;
        vol[idx] = V((accumulate ? T(vol[idx]) : T(0)) + acc);
      }
    }
  }
}

// Wang offset weights.  variant 0 = offset_correct_kernel (sin^2, zeroing,
// conebeam_projection.cu:233-262); variant 1 = offset_correct_kernel_sqrt
// (sin, no zeroing, :303-331).
template <class T>
void offset_weight(const Geom& g, const float* offs, int P, int variant, T* proj) {
#pragma omp parallel for collapse(2)
  for (int p = 0; p < P; ++p) {
    for (int v = 0; v < g.H; ++v) {
      const T o = T(offs[2 * p]);
      const T sg = o / std::fabs(o);          // NaN when o == 0: no weight applied
      const T omega = T(g.fov_u) / 2 - std::fabs(o);
      for (int u = 0; u < g.W; ++u) {
        size_t idx = ((size_t)p * g.H + v) * g.W + u;
        if (variant == 0) {
          const T t = (T(g.fov_u) * (T(u) / T(g.W) - T(0.5)) + o) * sg;
          if (std::fabs(t) <= omega) {
            T sw = std::sin(T(kPi) * (t + omega) / (4 * omega));
            proj[idx] *= sw * sw;
          }
          if (t < -omega) proj[idx] *= 0;
        } else {
          const T t = (T(g.fov_u) * ((T(u) + T(0.5)) / T(g.W) - T(0.5)) + o) * sg;
          if (std::fabs(t) <= std::fabs(omega)) proj[idx] *= std::sin(T(kPi) * (t + omega) / (4 * omega));
        }
      }
    }
  }
}

// Parker short-scan weights, redundancy_correct_kernel and S/B/b helpers,
// conebeam_projection.cu:151-194 (q = 0.1, epsilon = 0.001).
template <class T>
inline T parker_S(T beta) {
  if (beta <= T(-0.5)) return 0;
  if (beta < T(0.5)) return T(0.5) * (T(1) + std::sin(T(kPi) * beta));
  return 1;
}
template <class T>
void parker_weight(const Geom& g, const float* angles, int P, T* proj) {
  const T eps = T(0.001), q = T(0.1);
  const T delta = std::atan(T(g.fov_u) / (T(2) * T(g.SDD)));
  const T tan_delta = std::tan(delta);
#pragma omp parallel for collapse(2)
  for (int p = 0; p < P; ++p) {
    for (int v = 0; v < g.H; ++v) {
      const T beta = T(angles[p]) * T(kPi / 180.0);
      for (int u = 0; u < g.W; ++u) {
        const T alpha = -std::atan((T(u) / T(g.W) - T(0.5)) * T(2) * tan_delta);
        const T bp = q * (T(2) * (delta - alpha) + eps);
        const T bm = q * (T(2) * (delta + alpha) + eps);
        const T omega = T(0.5) * (parker_S<T>(beta / bp - T(0.5)) +
                                  parker_S<T>((beta + T(2) * (alpha - delta) - eps) / bp + T(0.5)) -
                                  parker_S<T>((beta - T(kPi) + T(2) * alpha) / bm - T(0.5)) -
                                  parker_S<T>((beta - T(kPi) - T(2) * delta - eps) / bm + T(0.5)));
        proj[((size_t)p * g.H + v) * g.W + u] *= omega;
      }
    }
  }
}

// ---------------------------------------------------------------- FFT (FP64)
using cd = std::complex<double>;

void fft_pow2(std::vector<cd>& a, bool inverse) {
  const size_t n = a.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) std::swap(a[i], a[j]);
  }
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = 2 * kPi / double(len) * (inverse ? 1 : -1);
    for (size_t i = 0; i < n; i += len) {
      for (size_t k = 0; k < len / 2; ++k) {
        cd w(std::cos(ang * k), std::sin(ang * k));
        cd u = a[i + k], v = a[i + k + len / 2] * w;
        a[i + k] = u + v;
        a[i + k + len / 2] = u - v;
      }
    }
  }
}

// Unnormalised DFT of any length (Bluestein for non powers of two).
void dft_any(std::vector<cd>& a, bool inverse) {
  const size_t n = a.size();
  if ((n & (n - 1)) == 0) { fft_pow2(a, inverse); return; }
  size_t m = 1;
  while (m < 2 * n - 1) m <<= 1;
  const double sgn = inverse ? 1.0 : -1.0;
  std::vector<cd> w(n);
  for (size_t k = 0; k < n; ++k) {
    double ang = kPi * double((k * k) % (2 * n)) / double(n);
    w[k] = cd(std::cos(ang), sgn * std::sin(ang));
  }
  std::vector<cd> A(m, 0.0), B(m, 0.0);
  for (size_t k = 0; k < n; ++k) A[k] = a[k] * w[k];
  B[0] = std::conj(w[0]);
  for (size_t k = 1; k < n; ++k) B[k] = B[m - k] = std::conj(w[k]);
  fft_pow2(A, false);
  fft_pow2(B, false);
  for (size_t i = 0; i < m; ++i) A[i] *= B[i];
  fft_pow2(A, true);
  for (size_t k = 0; k < n; ++k) a[k] = A[k] / double(m) * w[k];
}

// FDK row filter of conebeam_projection.cu:1504-1511 in FP64: centre-pad
// each row of width W to 2W (data at [W/2, W/2+W), Gadgetron pad<>), real
// FFT, multiply bins 0..W by the real filter (length W+1), inverse FFT,
// divide by 2W (cb_ifft, :138), crop [W/2, W/2+W).
void fdk_filter_rows(int W, long rows, const double* filt, double* data) {
  const int L = 2 * W, off = W / 2;
#pragma omp parallel
  {
    std::vector<cd> a(L);
#pragma omp for schedule(static)
    for (long r = 0; r < rows; ++r) {
      double* row = data + (size_t)r * W;
      std::fill(a.begin(), a.end(), cd(0, 0));
      for (int i = 0; i < W; ++i) a[off + i] = row[i];
      dft_any(a, false);
      // Hermitian spectrum of a real signal: bins k and L-k share filt[k].
      for (int k = 0; k <= W; ++k) a[k] *= filt[k];
      for (int k = W + 1; k < L; ++k) a[k] *= filt[L - k];
      dft_any(a, true);
      for (int i = 0; i < W; ++i) row[i] = a[off + i].real() / double(L);
    }
  }
}

// hoCuConebeamProjectionOperator::compute_cosine_weights,
// hoCuConebeamProjectionOperator.cpp:64-102.
void cosine_weights(const Geom& g, double* w) {
  for (int y = 0; y < g.H; ++y)
    for (int x = 0; x < g.W; ++x) {
      double xx = (double(x) / double(g.W) - 0.5) * g.fov_u;
      double yy = (double(y) / double(g.H) - 0.5) * g.fov_v;
      double s = g.SAD * xx / g.SDD, v = g.SAD * yy / g.SDD;
      w[(size_t)y * g.W + x] = double(float(g.SAD / std::sqrt(g.SAD * g.SAD + s * s + v * v)));
    }
}

// Default frequency filter (Guo et al.), hoCuConebeamProjectionOperator.cpp:26-62.
// Length W+1; evaluated in float as the reference does, then normalised so
// that its absolute sum equals W+1.
void default_filter(int W, double* out) {
  const int K = W + 1;
  const float A2 = float(0.2 * double(K) * double(K));
  double sum = 0;
  std::vector<float> h(K);
  for (int i = 0; i < K; ++i) {
    float k = float(i);
    if (k * k < A2) h[i] = k * A2 / (A2 - k * k) * std::exp(-A2 / (A2 - k * k));
    else h[i] = 0.f;
    sum += std::fabs(double(h[i]));
  }
  for (int i = 0; i < K; ++i) out[i] = double(h[i]) * (double(K) / sum);
}

}  // namespace

extern "C" {

// ------------------------------------------------------------ projectors
int oracle_forward_f64(const Geom* g, const float* angles, const float* offs, int P, double spp,
                       int mode, const double* vol, double* proj, int accumulate) {
  forward<double, double>(*g, angles, offs, P, spp, mode, vol, proj, accumulate);
  return 0;
}
int oracle_forward_f32(const Geom* g, const float* angles, const float* offs, int P, double spp,
                       int mode, const float* vol, float* proj, int accumulate) {
  forward<float, float>(*g, angles, offs, P, spp, mode, vol, proj, accumulate);
  return 0;
}
int oracle_backproject_f64(const Geom* g, const float* angles, const float* offs, int P, int fbp,
                           int mode, const double* proj, double* vol, int accumulate) {
  backproject<double, double>(*g, angles, offs, P, fbp, mode, proj, vol, accumulate);
  return 0;
}
int oracle_backproject_f32(const Geom* g, const float* angles, const float* offs, int P, int fbp,
                           int mode, const float* proj, float* vol, int accumulate) {
  backproject<float, float>(*g, angles, offs, P, fbp, mode, proj, vol, accumulate);
  return 0;
}
int oracle_samples_per_ray(const Geom* g, double spp) { return samples_per_ray(*g, spp); }

// ------------------------------------------------------------ weights
void oracle_offset_weight(const Geom* g, const float* offs, int P, int variant, double* proj) {
  offset_weight<double>(*g, offs, P, variant, proj);
}
void oracle_parker_weight(const Geom* g, const float* angles, int P, double* proj) {
  parker_weight<double>(*g, angles, P, proj);
}
void oracle_cosine_weights(const Geom* g, double* w) { cosine_weights(*g, w); }
void oracle_default_filter(int W, double* out) { default_filter(W, out); }
void oracle_fdk_filter_rows(int W, long rows, const double* filt, double* data) {
  fdk_filter_rows(W, rows, filt, data);
}

// Short-scan test of hoCuConebeamProjectionOperator.h:57-65: the span (after
// the angles were shifted to start at 0) is compared to pi + 3*delta.
int oracle_is_short_scan(const Geom* g, const float* angles, int P) {
  float span = *std::max_element(angles, angles + P);
  float delta = std::atan(float(g->fov_u) / (2.0f * float(g->SDD)));
  return (span * float(kPi) / 180.0f > float(kPi) + 3.0f * delta) ? 0 : 1;
}

// Whole FDK of hoCuConebeamProjectionOperator::mult_MH with FBP
// (hoCuConebeamProjectionOperator.cpp:235-254, conebeam_projection.cu:1483-1521,
// :1614-1618): cosine weight, [Parker], ramp filter, [offset sin^2 weight],
// back-projection with the 1/U^2 weight, then x *= 2/P.
int oracle_fdk(const Geom* g, const float* angles, const float* offs, int P, int short_scan,
               int offset_corr, const double* filt, const double* proj_in, double* vol) {
  const size_t npx = (size_t)g->W * g->H;
  std::vector<double> p(proj_in, proj_in + npx * P);
  std::vector<double> cw(npx);
  cosine_weights(*g, cw.data());
  for (int v = 0; v < P; ++v)
    for (size_t i = 0; i < npx; ++i) p[v * npx + i] *= cw[i];
  if (short_scan) parker_weight<double>(*g, angles, P, p.data());
  fdk_filter_rows(g->W, (long)g->H * P, filt, p.data());
  if (offset_corr) offset_weight<double>(*g, offs, P, 0, p.data());
  backproject<double, double>(*g, angles, offs, P, 1, 0, p.data(), vol, 0);
  const double s = 2.0 / double(P);
  for (size_t i = 0; i < (size_t)g->nx * g->ny * g->nz; ++i) vol[i] *= s;
  return 0;
}

// ------------------------------------------------------------ subsets
// CBSubsetOperator<ARRAY>::setup, CBSubsetOperator.cpp:52-115: views that
// belong to a bin are dealt round-robin to n_subsets subsets in index order
// (:76-82), each subset is re-sorted by bin with std::sort (:86-87), and the
// permutation is the concatenation of the subsets (:100-104).
// view_bin[i] < 0 marks a view outside every bin.  Returns the number of
// views placed in order_out.
int oracle_subset_partition(int n_views, const int* view_bin, int n_subsets, int* order_out,
                            int* subset_sizes_out) {
  std::map<unsigned, unsigned> bins;
  for (int i = 0; i < n_views; ++i)
    if (view_bin[i] >= 0) bins[(unsigned)i] = (unsigned)view_bin[i];
  std::vector<std::vector<unsigned>> sub(n_subsets);
  int k = 0;
  for (int i = 0; i < n_views; ++i)
    if (bins.find((unsigned)i) != bins.end()) { sub[k % n_subsets].push_back(i); ++k; }
  for (auto& s : sub)
    std::sort(s.begin(), s.end(), [&](unsigned a, unsigned b) { return bins[a] < bins[b]; });
  int n = 0;
  for (int s = 0; s < n_subsets; ++s) {
    subset_sizes_out[s] = (int)sub[s].size();
    for (unsigned v : sub[s]) order_out[n++] = (int)v;
  }
  return n;
}

// ------------------------------------------------------------ solvers
// Operator pair of cuConebeamProjectionOperator for one subset:
// mult_M = plain forward (cuConebeamProjectionOperator.cpp:38-80, the offset
// weight there is commented out); mult_MH = back-projection of a copy of the
// input multiplied by the sin^2 offset weight when offset correction is on
// (.cpp:82-116 and conebeam_projection.cu:1242-1244).
struct SubsetOp {
  const Geom* g;
  const float* angles;
  const float* offs;
  const int* sizes;
  const int* offcorr;
  int S;
  double spp;
  int mode;
  const unsigned char* mask = nullptr;  // apply_mask after mult_MH (cuConebeamProjectionOperator.cpp:113-114)
  const double* weights = nullptr;      // CBSubsetWeightOperator projection weights (all views, subset order)
  const int* view_bin = nullptr;        // bin of every view (subset order); NULL: one bin
  int n_bins = 1;
  size_t npx() const { return (size_t)g->W * g->H; }
  size_t nvox() const { return (size_t)g->nx * g->ny * g->nz; }
  int first(int s) const { int f = 0; for (int i = 0; i < s; ++i) f += sizes[i]; return f; }
  // Runs of views of one bin inside subset s (a subset is sorted by bin,
  // CBSubsetOperator.cpp:86-87): (bin, first view, count).
  std::vector<std::array<int, 3>> runs(int s) const {
    std::vector<std::array<int, 3>> r;
    const int f = first(s);
    for (int i = 0; i < sizes[s];) {
      const int b = view_bin ? view_bin[f + i] : 0;
      int n = 1;
      while (i + n < sizes[s] && (view_bin ? view_bin[f + i + n] : 0) == b) ++n;
      r.push_back({b, f + i, n});
      i += n;
    }
    return r;
  }
  // CBSubsetWeightOperator::mult_M (CBSubsetWeightOperator.h:32-43): out = w * (A x).
  // With bins, each bin's views project that bin's volume
  // (cuConebeamProjectionOperator.cpp:49-78).
  void M(int s, const double* x, double* out) const {
    const int f = first(s);
    for (const auto& run : runs(s))
      forward<double, double>(*g, angles + run[1], offs + 2 * run[1], run[2], spp, mode, x + nvox() * run[0],
                              out + npx() * (run[1] - f), 0);
    if (weights)
      for (size_t i = 0; i < npx() * sizes[s]; ++i) out[i] *= weights[npx() * f + i];
  }
  // CBSubsetWeightOperator::mult_MH (.h:44-49): the input times w goes into mult_MH.
  // With bins, every bin's volume receives its own views (none: 0 or unchanged).
  void MH(int s, const double* in_raw, double* x, int acc) const {
    const int f = first(s);
    std::vector<double> wtmp;
    const double* in = in_raw;
    if (weights) {
      wtmp.assign(in_raw, in_raw + npx() * sizes[s]);
      for (size_t i = 0; i < wtmp.size(); ++i) wtmp[i] *= weights[npx() * f + i];
      in = wtmp.data();
    }
    std::vector<double> tmp;
    if (offcorr[s]) {
      tmp.assign(in, in + npx() * sizes[s]);
      offset_weight<double>(*g, offs + 2 * f, sizes[s], 0, tmp.data());
      in = tmp.data();
    }
    std::vector<int> seen(n_bins, 0);
    for (const auto& run : runs(s)) {
      double* xb = x + nvox() * run[0];
      backproject<double, double>(*g, angles + run[1], offs + 2 * run[1], run[2], 0, mode,
                                  in + npx() * (run[1] - f), xb, acc || seen[run[0]]);
      seen[run[0]] = 1;
    }
    for (int b = 0; b < n_bins; ++b)
      if (!seen[b] && !acc) std::fill(x + nvox() * b, x + nvox() * (b + 1), 0.0);
    if (mask) {
      for (size_t i = 0; i < nvox(); ++i) x[i] *= double(mask[i]);
    }
  }
};

// osMOMSolverD<ARRAY>::solve without regularisers, solvers/osMOMSolverD.h:82-196.
// b holds the projections in subset-contiguous order.  resid_norm2 (optional,
// iters*S entries) receives ||A_s x - b_s||^2 for each subset step (the
// VERBOSE print of :147-149).  Returns z, the momentum point (:195).
static const unsigned char* g_solver_mask = nullptr;
static const double* g_solver_weights = nullptr;
static const int* g_solver_view_bin = nullptr;
static int g_solver_bins = 1;

// Mask and projection weights used by the next oracle_osmom / oracle_ossart call (NULL = none).
void oracle_set_solver_mask(const unsigned char* mask) { g_solver_mask = mask; }
void oracle_set_solver_weights(const double* w) { g_solver_weights = w; }
// Total-variation regularisation of the next oracle_osmom call (weight 0: none):
// osMOMSolverD with one cuTVPrimalDualOperator(alpha) of this weight, the
// solver's tau and reg_steps.
static double g_tv_weight = 0.0, g_tv_alpha = 0.0, g_tv_tau = 1e-3;
static int g_tv_steps = 1;
void oracle_set_solver_tv(double weight, double alpha, double tau, int reg_steps) {
  g_tv_weight = weight;
  g_tv_alpha = alpha;
  g_tv_tau = tau;
  g_tv_steps = reg_steps;
}

// denoise of osMOMSolverD.h:205-231 with one TV operator, whose weight the
// solver normalises to 1 (avg_lambda = the weight, :124-126): primal-dual steps
// from x toward s.  The TV primal step (operators/cuTVPrimalDualOperator.cu:9-37)
// takes periodic forward differences, scales them by sigma / (1 + sigma alpha)
// and projects each gradient vector onto the unit ball; the dual step (:40-62)
// adds the negative divergence; updateG (osMOMSolverD.h:233-247, the generic
// version that osMOMSolverD<cuNDArray<float>> runs) resolves the
// preconditioned data term.  Every bin is a separate 3-D image.
static void tv_denoise(const Geom* g, int n_bins, std::vector<double>& x, const std::vector<double>& s,
                       const std::vector<double>& D, double lambda, double alpha, double tau0, int steps, double gam) {
  const int nx = g->nx, ny = g->ny, nz = g->nz;
  const size_t nv = (size_t)nx * ny * nz;
  double tau = tau0, sigma = 1.0 / (tau * 4.0 * 4.0);
  std::vector<double> P(3 * nv);
  auto at = [&](int i, int j, int k) { return ((size_t)k * ny + j) * nx + i; };
  for (int it = 0; it < steps; ++it) {
    const double scale = sigma / (1.0 + sigma * alpha);
    for (int b = 0; b < n_bins; ++b) {
      double* xb = x.data() + nv * b;
      const double* sb = s.data() + nv * b;
      const double* Db = D.data() + nv * b;
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const size_t c = at(i, j, k);
            const double v = xb[c];
            double d[3] = {(xb[at((i + 1) % nx, j, k)] - v) * scale, (xb[at(i, (j + 1) % ny, k)] - v) * scale,
                           (xb[at(i, j, (k + 1) % nz)] - v) * scale};
            const double m = std::max(1.0, std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]));
            for (int a = 0; a < 3; ++a) P[a * nv + c] = d[a] / m;
          }
      for (int k = 0; k < nz; ++k)
        for (int j = 0; j < ny; ++j)
          for (int i = 0; i < nx; ++i) {
            const size_t c = at(i, j, k);
            const double gv = (P[at((i + nx - 1) % nx, j, k)] - P[c]) +
                              (P[nv + at(i, (j + ny - 1) % ny, k)] - P[nv + c]) +
                              (P[2 * nv + at(i, j, (k + nz - 1) % nz)] - P[2 * nv + c]);
            xb[c] = ((xb[c] - tau * gv) + tau / lambda * (sb[c] / Db[c])) / ((1.0 / Db[c]) * (tau / lambda) + 1.0);
          }
    }
    const double theta = 1.0 / std::sqrt(1.0 + 2.0 * gam * tau);
    tau *= theta;
    sigma /= theta;
  }
}

// Per-iteration copies of z from the next oracle_osmom call (iters * images
// doubles; NULL: none).
static double* g_solver_snapshots = nullptr;
void oracle_set_solver_snapshots(double* buf) { g_solver_snapshots = buf; }

// Bins (CBCT_binning) of the next oracle_osmom call: view_bin per view in
// subset order (NULL: one bin); images then hold n_bins volumes.
void oracle_set_solver_bins(int n_bins, const int* view_bin) {
  g_solver_bins = view_bin ? n_bins : 1;
  g_solver_view_bin = view_bin;
}

int oracle_osmom(const Geom* g, const float* angles, const float* offs, const int* sizes,
                 const int* offcorr, int S, double spp, int iters, double beta, double gamma,
                 int nonneg, const double* x0, const double* b, double* z_out,
                 double* resid_norm2) {
  SubsetOp A{g, angles, offs, sizes, offcorr, S, spp, 0};
  A.mask = g_solver_mask;
  A.weights = g_solver_weights;
  A.view_bin = g_solver_view_bin;
  A.n_bins = g_solver_bins;
  const size_t nv = (size_t)g->nx * g->ny * g->nz * A.n_bins;
  int P = 0;
  for (int s = 0; s < S; ++s) P += sizes[s];
  std::vector<double> z(nv, 0.0), x, xold, D(nv, 1.0), tmp_img(nv);
  if (x0) std::copy(x0, x0 + nv, z.begin());
  x = z;
  xold = z;
  std::vector<double> proj((size_t)P * A.npx());
  // Preconditioner D = 1/max(A^T A 1, 1e-6) over all subsets (:115-120).
  for (int s = 0; s < S; ++s) A.M(s, D.data(), proj.data() + A.npx() * A.first(s));
  std::vector<double> pre(nv, 0.0);
  for (int s = 0; s < S; ++s) A.MH(s, proj.data() + A.npx() * A.first(s), pre.data(), 1);
  for (size_t i = 0; i < nv; ++i) D[i] = 1.0 / std::max(pre[i], 1e-6);
  double asum_D = 0;
  for (size_t i = 0; i < nv; ++i) asum_D += std::fabs(D[i]);
  const double gam = g_tv_weight > 0 ? 0.35 / g_tv_weight / (double(nv) / asum_D) : 0.0;
  double t = 1, told = 1;
  int step = 0;
  for (int it = 0; it < iters; ++it) {
    for (int s = 0; s < S; ++s, ++step) {
      t = 0.5 * (1 + std::sqrt(1 + 4 * t * t));
      double* r = proj.data() + A.npx() * A.first(s);
      const double* bs = b + A.npx() * A.first(s);
      A.M(s, x.data(), r);
      double n2 = 0;
      for (size_t i = 0; i < A.npx() * sizes[s]; ++i) { r[i] -= bs[i]; n2 += r[i] * r[i]; }
      if (resid_norm2) resid_norm2[step] = n2;
      A.MH(s, r, tmp_img.data(), 0);
      const double a = -beta / (1 + gamma * it) * S;
      for (size_t i = 0; i < nv; ++i) z[i] += a * (tmp_img[i] * D[i]);
      if (g_tv_weight > 0)                              // denoise with the TV prior
        tv_denoise(g, A.n_bins, x, z, D, g_tv_weight, g_tv_alpha, g_tv_tau, g_tv_steps, gam);
      else
        x = z;                                          // denoise: x = z (:211-213)
      if (nonneg) for (auto& e : x) e = std::max(e, 0.0);
      const double m = (told - 1) / t;
      for (size_t i = 0; i < nv; ++i) z[i] = x[i] * (1 + m) - m * xold[i];
      std::swap(x, xold);
      x = z;
      told = t;
    }
    if (g_solver_snapshots) std::copy(z.begin(), z.end(), g_solver_snapshots + (size_t)it * nv);
  }
  std::copy(z.begin(), z.end(), z_out);
  return 0;
}

// osSARTSolver<ARRAY>::solve, solvers/osSARTSolver.h:33-126.  cost_out
// (optional, iters entries) receives the per-iteration ||A x - b||^2 printed
// at :110-116.
int oracle_ossart(const Geom* g, const float* angles, const float* offs, const int* sizes,
                  const int* offcorr, int S, double spp, int iters, double beta, double gamma,
                  int nonneg, const double* x0, const double* b, double* x_out, double* cost_out) {
  SubsetOp A{g, angles, offs, sizes, offcorr, S, spp, 0};
  A.mask = g_solver_mask;
  A.weights = g_solver_weights;
  const size_t nv = (size_t)g->nx * g->ny * g->nz;
  int P = 0;
  for (int s = 0; s < S; ++s) P += sizes[s];
  const size_t np = (size_t)P * A.npx();
  std::vector<double> x(nv, 0.0);
  if (x0) std::copy(x0, x0 + nv, x.begin());
  std::vector<double> ones_img(nv, 1.0), Wp(np), tmp(np), tmp_img(nv);
  for (int s = 0; s < S; ++s) A.M(s, ones_img.data(), Wp.data() + A.npx() * A.first(s));
  for (auto& e : Wp) e = 1.0 / std::max(e, 1e-6);
  std::vector<double> ones_proj(np, 1.0);
  std::vector<std::vector<double>> V(S, std::vector<double>(nv));
  for (int s = 0; s < S; ++s) {
    A.MH(s, ones_proj.data() + A.npx() * A.first(s), V[s].data(), 0);
    for (auto& e : V[s]) e = 1.0 / std::max(e, 1e-6);
  }
  std::vector<int> order(S);
  for (int s = 0; s < S; ++s) order[s] = s;
  for (int it = 0; it < iters; ++it) {
    for (int is = 0; is < S; ++is) {
      const int s = order[is];
      const size_t o = A.npx() * A.first(s), n = A.npx() * sizes[s];
      A.M(s, x.data(), tmp.data() + o);
      for (size_t i = 0; i < n; ++i) tmp[o + i] = -(tmp[o + i] - b[o + i]) * Wp[o + i];
      A.MH(s, tmp.data() + o, tmp_img.data(), 0);
      const double a = beta / (1 + gamma * it);
      for (size_t i = 0; i < nv; ++i) {
        x[i] += a * (tmp_img[i] * V[s][i]);
        if (nonneg) x[i] = std::max(x[i], 0.0);
      }
    }
    std::reverse(order.begin(), order.end());
    if (cost_out) {
      double c = 0;
      for (int s = 0; s < S; ++s) {
        const size_t o = A.npx() * A.first(s), n = A.npx() * sizes[s];
        A.M(s, x.data(), tmp.data() + o);
        for (size_t i = 0; i < n; ++i) { double r = tmp[o + i] - b[o + i]; c += r * r; }
      }
      cost_out[it] = c;
    }
  }
  std::copy(x.begin(), x.end(), x_out);
  return 0;
}

// ------------------------------------------------------------ phantoms
// Ellipsoid record: cx, cy, cz, ax, ay, az (semi-axes, mm), phi, theta, psi
// (rotation R = Rz(phi) Ry(theta) Rx(psi), radians), density (1/mm).
static void ell_rot(const double* e, double R[9]) {
  double cp = std::cos(e[6]), sp = std::sin(e[6]);
  double ct = std::cos(e[7]), st = std::sin(e[7]);
  double cs = std::cos(e[8]), ss = std::sin(e[8]);
  // Rz(phi) * Ry(theta) * Rx(psi)
  R[0] = cp * ct; R[1] = cp * st * ss - sp * cs; R[2] = cp * st * cs + sp * ss;
  R[3] = sp * ct; R[4] = sp * st * ss + cp * cs; R[5] = sp * st * cs - cp * ss;
  R[6] = -st;     R[7] = ct * ss;                R[8] = ct * cs;
}

// Supersampled voxelisation (ss^3 points per voxel) of a sum of ellipsoids.
void oracle_phantom_voxelize(const double* ell, int K, const Geom* g, int ss, double* vol) {
  std::vector<double> R(9 * (size_t)K);
  for (int e = 0; e < K; ++e) ell_rot(ell + 10 * e, R.data() + 9 * e);
  const double vx = g->lx / g->nx, vy = g->ly / g->ny, vz = g->lz / g->nz;
#pragma omp parallel for collapse(2) schedule(dynamic, 1)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        double acc = 0;
        for (int sz = 0; sz < ss; ++sz)
          for (int sy = 0; sy < ss; ++sy)
            for (int sx = 0; sx < ss; ++sx) {
              double p[3] = {-g->lx / 2 + (i + (sx + 0.5) / ss) * vx,
                             -g->ly / 2 + (j + (sy + 0.5) / ss) * vy,
                             -g->lz / 2 + (k + (sz + 0.5) / ss) * vz};
              for (int e = 0; e < K; ++e) {
                const double* E = ell + 10 * e;
                const double* r = R.data() + 9 * e;
                double q[3] = {p[0] - E[0], p[1] - E[1], p[2] - E[2]};
                // local = R^T q
                double l0 = (r[0] * q[0] + r[3] * q[1] + r[6] * q[2]) / E[3];
                double l1 = (r[1] * q[0] + r[4] * q[1] + r[7] * q[2]) / E[4];
                double l2 = (r[2] * q[0] + r[5] * q[1] + r[8] * q[2]) / E[5];
                if (l0 * l0 + l1 * l1 + l2 * l2 <= 1.0) acc += E[9];
              }
            }
        vol[((size_t)k * g->ny + j) * g->nx + i] = acc / double(ss * ss * ss);
      }
}

// Exact line integrals of the box-truncated ellipsoid phantom along the rays
// of the forward projector (source to detector-pixel centre, clipped to the
// volume box as conebeam_projection.cu:478-484 does).
void oracle_phantom_project(const double* ell, int K, const Geom* g, const float* angles,
                            const float* offs, int P, double* proj) {
  std::vector<double> R(9 * (size_t)K);
  for (int e = 0; e < K; ++e) ell_rot(ell + 10 * e, R.data() + 9 * e);
#pragma omp parallel for collapse(2) schedule(dynamic, 4)
  for (int p = 0; p < P; ++p)
    for (int v = 0; v < g->H; ++v) {
      const double th = double(angles[p]) * (kPi / 180.0);
      for (int u = 0; u < g->W; ++u) {
        double S[3], d[3];
        ray_of<double>(*g, th, double(offs[2 * p]), double(offs[2 * p + 1]), u, v, S, d);
        double a1, a2;
        clip_box<double>(*g, S, d, a1, a2);
        const double dl = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        double acc = 0;
        if (a2 > a1) {
          for (int e = 0; e < K; ++e) {
            const double* E = ell + 10 * e;
            const double* r = R.data() + 9 * e;
            double q[3] = {S[0] - E[0], S[1] - E[1], S[2] - E[2]};
            double s0 = (r[0] * q[0] + r[3] * q[1] + r[6] * q[2]) / E[3];
            double s1 = (r[1] * q[0] + r[4] * q[1] + r[7] * q[2]) / E[4];
            double s2 = (r[2] * q[0] + r[5] * q[1] + r[8] * q[2]) / E[5];
            double d0 = (r[0] * d[0] + r[3] * d[1] + r[6] * d[2]) / E[3];
            double d1 = (r[1] * d[0] + r[4] * d[1] + r[7] * d[2]) / E[4];
            double d2 = (r[2] * d[0] + r[5] * d[1] + r[8] * d[2]) / E[5];
            double A = d0 * d0 + d1 * d1 + d2 * d2;
            double B = s0 * d0 + s1 * d1 + s2 * d2;
            double C = s0 * s0 + s1 * s1 + s2 * s2 - 1.0;
            double disc = B * B - A * C;
            if (disc <= 0) continue;
            double sq = std::sqrt(disc);
            double t0 = (-B - sq) / A, t1 = (-B + sq) / A;
            t0 = std::max(t0, a1);
            t1 = std::min(t1, a2);
            if (t1 > t0) acc += E[9] * (t1 - t0) * dl;
          }
        }
        proj[((size_t)p * g->H + v) * g->W + u] = acc;
      }
    }
}

// Space carver, conebeam_spacecarver_kernel (conebeam_projection.cu:822-921):
// the voxel centre (with z negated, :852) is projected into every view and the
// projection is point-sampled (texel floor(u*W), border 0, projections_mask_tex
// at :41-42); views where the sample is nonzero and below `limit` are counted,
// and the mask is 1 where fewer than 3 views were counted.
void oracle_spacecarver(const Geom* g, const float* angles, const float* offs, int P, const double* proj,
                        double limit, unsigned char* mask) {
#pragma omp parallel for collapse(2) schedule(static)
  for (int k = 0; k < g->nz; ++k)
    for (int j = 0; j < g->ny; ++j)
      for (int i = 0; i < g->nx; ++i) {
        const double x = ((i + 0.5) / g->nx - 0.5) * g->lx;
        const double y = ((j + 0.5) / g->ny - 0.5) * g->ly;
        const double z = -((k + 0.5) / g->nz - 0.5) * g->lz;
        int count = 0;
        for (int p = 0; p < P; ++p) {
          const double th = double(angles[p]) * (kPi / 180.0);
          const double c = std::cos(th), s = std::sin(th);
          const double xr = c * x + s * y, yr = -s * x + c * y;
          const double dy = yr + g->SAD;
          const double ex = g->SDD * (xr / dy) - offs[2 * p], ez = g->SDD * (z / dy) - offs[2 * p + 1];
          const double un = ex / g->fov_u + 0.5, vn = ez / g->fov_v + 0.5;
          const long iu = (long)std::floor(un * g->W), iv = (long)std::floor(vn * g->H);
          double t = 0.0;
          if (iu >= 0 && iu < g->W && iv >= 0 && iv < g->H) t = proj[((size_t)p * g->H + iv) * g->W + iu];
          if (t < limit && t != 0.0) ++count;
        }
        mask[((size_t)k * g->ny + j) * g->nx + i] = count < 3 ? 1 : 0;
      }
}

int oracle_num_threads() { return omp_get_max_threads(); }
void oracle_set_num_threads(int n) { omp_set_num_threads(n); }

}  // extern "C"
