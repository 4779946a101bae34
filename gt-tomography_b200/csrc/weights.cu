// weights.cu -- detector-space weights and the FDK row filter for sm_100a.
//
// Offset (Wang) weights: conebeam_projection.cu:233-262 (sin^2, zeroing) and
// :303-331 (sin).  Parker weights: :151-194.  Cosine weights:
// hoCuConebeamProjectionOperator.cpp:64-102.  Row filter: :1504-1511 with
// cb_fft/cb_ifft :87-139.
//
// The reference filters each detector row by zero-padding it to 2W, an R2C
// FFT, a multiply by the real filter H[0..W], a C2R FFT and a division by 2W,
// then crops the centre W samples.  Because input and output both occupy the
// centre W samples of the 2W frame, this is exactly a linear convolution with
// the real even kernel h[j] = IDFT_2W(H)[j], |j| <= W-1 (the wrapped taps are
// never reached).  The kernel below evaluates that convolution with a
// hand-written power-of-two FFT of length L >= 2W-1 in shared memory: two rows
// ride in one complex transform (row a in the real part, row b in the
// imaginary part); since the spectrum of h is real and even, the product's
// inverse keeps the two rows apart.  The spectrum (with the 1/L scale) is
// computed once per filter on the host in FP64.
#include <cmath>
#include <map>
#include <utility>
#include <vector>

#include "device_common.cuh"

namespace cbct {

namespace {

__global__ void offset_weight_kernel(const float* __restrict__ in, float* __restrict__ out,
                                     const ViewParams* __restrict__ views, GridConst gc, int n_views,
                                     int variant) {
  const size_t n = (size_t)gc.W * gc.H * n_views;
  for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < n;
       idx += (size_t)gridDim.x * blockDim.x) {
    const int u = int(idx % gc.W);
    const int p = int(idx / ((size_t)gc.W * gc.H));
    const float o = views[p].ox;
    const float w = variant == 0 ? offset_weight_full(gc.fov_u, gc.W, u, o)
                                 : offset_weight_sqrt(gc.fov_u, gc.W, u, o);
    // The sin^2 variant multiplies by 0 (not a store of 0) where t < -omega,
    // and leaves pixels alone when no branch applies; w = 1 reproduces that.
    out[idx] = in[idx] * w;
  }
}

constexpr int kFftThreads = 256;

// One CTA filters pairs of rows.  rows = H * n_views, row r = (p, v).
//   pre[u + W*v]     cosine weight (nullable)
//   parker[u + W*p]  Parker weight (nullable)
//   post[u + W*p]    sin^2 offset weight (nullable)
// T: storage type of the input projections (float, __half, __nv_bfloat16);
// arithmetic is FP32.  For T = float, in and out may alias.
template <class T>
__global__ void __launch_bounds__(kFftThreads) fdk_filter_kernel(
    const T* in, float* out, int W, int H, long rows, int L, int logL,
    const float* __restrict__ spec, const float2* __restrict__ tw, const float* __restrict__ pre,
    const float* __restrict__ parker, const float* __restrict__ post) {
  extern __shared__ float2 fsm[];
  float2* a = fsm;                  // L
  float2* t = fsm + L;              // L/2 twiddles
  float* hs = reinterpret_cast<float*>(fsm + L + L / 2);  // L spectrum
  const int tid = threadIdx.x;
  for (int i = tid; i < L / 2; i += kFftThreads) t[i] = tw[i];
  for (int i = tid; i < L; i += kFftThreads) hs[i] = spec[i];
  const long npairs = (rows + 1) / 2;
  for (long pr = blockIdx.x; pr < npairs; pr += gridDim.x) {
    const long ra = 2 * pr, rb = 2 * pr + 1;
    const bool hasb = rb < rows;
    const int pa = int(ra / H), va = int(ra % H);
    const int pb = int(rb / H), vb = int(rb % H);
    __syncthreads();
    // Bit-reversed load with the pre-weights fused.
    for (int n = tid; n < L; n += kFftThreads) {
      float xa = 0.f, xb = 0.f;
      if (n < W) {
        xa = sm_f(in[ra * W + n]);
        if (pre) xa *= pre[(size_t)va * W + n];
        if (parker) xa *= parker[(size_t)pa * W + n];
        if (hasb) {
          xb = sm_f(in[rb * W + n]);
          if (pre) xb *= pre[(size_t)vb * W + n];
          if (parker) xb *= parker[(size_t)pb * W + n];
        }
      }
      a[__brev(n) >> (32 - logL)] = make_float2(xa, xb);
    }
    __syncthreads();
    // Forward DIT, twiddle exp(-2 pi i k / L).
    for (int len = 2; len <= L; len <<= 1) {
      const int half = len >> 1, ts = L / len;
      for (int b = tid; b < L / 2; b += kFftThreads) {
        const int grp = b / half, pos = b - grp * half;
        const int i0 = grp * len + pos, i1 = i0 + half;
        const float2 w = t[pos * ts];
        const float2 v = a[i1];
        const float2 x = a[i0];
        const float2 m = make_float2(w.x * v.x - w.y * v.y, w.x * v.y + w.y * v.x);
        a[i0] = make_float2(x.x + m.x, x.y + m.y);
        a[i1] = make_float2(x.x - m.x, x.y - m.y);
      }
      __syncthreads();
    }
    for (int k = tid; k < L; k += kFftThreads) {
      const float h = hs[k];
      a[k] = make_float2(a[k].x * h, a[k].y * h);
    }
    __syncthreads();
    // Inverse DIF (natural order in, bit-reversed order out), twiddle exp(+2 pi i k / L).
    for (int len = L; len >= 2; len >>= 1) {
      const int half = len >> 1, ts = L / len;
      for (int b = tid; b < L / 2; b += kFftThreads) {
        const int grp = b / half, pos = b - grp * half;
        const int i0 = grp * len + pos, i1 = i0 + half;
        const float2 w = t[pos * ts];
        const float2 x = a[i0], v = a[i1];
        const float2 d = make_float2(x.x - v.x, x.y - v.y);
        a[i0] = make_float2(x.x + v.x, x.y + v.y);
        a[i1] = make_float2(w.x * d.x + w.y * d.y, w.x * d.y - w.y * d.x);  // d * conj(w)
      }
      __syncthreads();
    }
    for (int n = tid; n < W; n += kFftThreads) {
      const float2 y = a[__brev(n) >> (32 - logL)];
      float ya = y.x;
      if (post) ya *= post[(size_t)pa * W + n];
      out[ra * W + n] = ya;
      if (hasb) {
        float yb = y.y;
        if (post) yb *= post[(size_t)pb * W + n];
        out[rb * W + n] = yb;
      }
    }
  }
}

// ------------------------------------------------------------ register FFT filter
// The same convolution for L = 32 TL (TL = 16 or 32 lanes per transform, so
// detectors up to 512 wide) as a four-step FFT held in registers: with
// n = TL n1 + n2 and k = k1 + 32 k2, each lane (n2) takes a 32-point DFT over
// n1, multiplies by W_L^(n2 k1), the transform is transposed through shared
// memory, and each lane takes TL-point DFTs over n2 for its k1 (one for TL =
// 32, two for TL = 16); the inverse runs the same steps backwards.  One warp
// filters one pair of rows (TL = 32) or two pairs (TL = 16), with one
// shared-memory transpose per direction instead of log2(L) barrier-separated
// radix-2 passes.
struct Tw32 {
  float2 w[16];  // exp(-2 pi i m / 32), m = 0..15
};

constexpr int kRegFftThreads = 128;

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

constexpr int brev_bits(int i, int bits) {
  int r = 0;
  for (int b = 0; b < bits; ++b) r |= ((i >> b) & 1) << (bits - 1 - b);
  return r;
}

// In-register N-point DFT (N = 16 or 32) of v[off .. off+N), natural order in
// and out; INV takes exp(+2 pi i / N).  Radix-2, decimation in time, all
// indices compile-time.
template <int N, bool INV, int OFF, int NV>
__device__ __forceinline__ void fft_reg(float2 (&v)[NV], const Tw32& tw) {
  constexpr int bits = N == 16 ? 4 : 5;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = brev_bits(i, bits);
    if (j > i) {
      const float2 t = v[OFF + i];
      v[OFF + i] = v[OFF + j];
      v[OFF + j] = t;
    }
  }
#pragma unroll
  for (int len = 2; len <= N; len <<= 1) {
#pragma unroll
    for (int i = 0; i < N; i += len) {
#pragma unroll
      for (int k = 0; k < len / 2; ++k) {
        float2 w = tw.w[k * (32 / len)];
        if (INV) w.y = -w.y;
        const float2 a = v[OFF + i + k];
        const float2 b = cmul(v[OFF + i + k + len / 2], w);
        v[OFF + i + k] = make_float2(a.x + b.x, a.y + b.y);
        v[OFF + i + k + len / 2] = make_float2(a.x - b.x, a.y - b.y);
      }
    }
  }
}

#ifndef CBCT_FDK_MINB
#define CBCT_FDK_MINB 4
#endif

template <class T, int TL>
__global__ void __launch_bounds__(kRegFftThreads, CBCT_FDK_MINB) fdk_filter_reg_kernel(
    const T* in, float* out, int W, int H, long rows, const float* __restrict__ spec,
    const float2* __restrict__ twL, const __grid_constant__ Tw32 tw, const float* __restrict__ pre,
    const float* __restrict__ parker, const float* __restrict__ post) {
  constexpr int G = 32 / TL;          // transforms per warp
  constexpr int S = TL + 1;           // padded row of the transpose buffer
  constexpr int L = 32 * TL;
  extern __shared__ float2 xs[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane / TL, j = lane % TL;
  float2* buf = xs + (size_t)(warp * G + g) * 32 * S;
  // The CTA's copies of the inter-pass twiddles and the spectrum, after the
  // transpose buffers.
  float2* stw = xs + (size_t)(kRegFftThreads / 32) * G * 32 * S;
  float* sspec = reinterpret_cast<float*>(stw + 32 * TL);
  for (int i = threadIdx.x; i < 32 * TL; i += kRegFftThreads) stw[i] = twL[i];
  for (int i = threadIdx.x; i < L; i += kRegFftThreads) sspec[i] = spec[i];
  __syncthreads();
  const long npairs = (rows + 1) / 2;
  const long nwarps = (long)gridDim.x * (kRegFftThreads / 32);
  for (long base = ((long)blockIdx.x * (kRegFftThreads / 32) + warp) * G; base < npairs; base += nwarps * G) {
    const long pr = base + g;
    const bool valid = pr < npairs;
    const long ra = 2 * pr, rb = 2 * pr + 1;
    const bool hasb = valid && rb < rows;
    const int pa = int(ra / H), va = int(ra % H);
    const int pb = int(rb / H), vb = int(rb % H);
    float2 v[32];
    // Load x[TL n1 + j] (row a real, row b imaginary) with the pre-weights.
#pragma unroll
    for (int n1 = 0; n1 < 32; ++n1) {
      const int n = TL * n1 + j;
      float xa = 0.f, xb = 0.f;
      if (valid && n < W) {
        xa = sm_f(in[ra * W + n]);
        if (pre) xa *= pre[(size_t)va * W + n];
        if (parker) xa *= parker[(size_t)pa * W + n];
        if (hasb) {
          xb = sm_f(in[rb * W + n]);
          if (pre) xb *= pre[(size_t)vb * W + n];
          if (parker) xb *= parker[(size_t)pb * W + n];
        }
      }
      v[n1] = make_float2(xa, xb);
    }
    fft_reg<32, false, 0>(v, tw);                       // v[k1]
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) v[k1] = cmul(v[k1], stw[k1 * TL + j]);
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) buf[k1 * S + j] = v[k1];
    __syncwarp();
    // Lane j now takes k1 = j + c TL, c < G: TL-point DFTs over n2.
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int n2 = 0; n2 < TL; ++n2) v[c * TL + n2] = buf[(j + c * TL) * S + n2];
    fft_reg<TL, false, 0>(v, tw);
    if (G > 1) fft_reg<TL, false, (G > 1 ? TL : 0)>(v, tw);
    // Spectrum (real, with the 1/L scale): X[k1 + 32 k2] at v[c TL + k2].
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int k2 = 0; k2 < TL; ++k2) {
        const float h = sspec[(j + c * TL) + 32 * k2];
        v[c * TL + k2] = make_float2(v[c * TL + k2].x * h, v[c * TL + k2].y * h);
      }
    fft_reg<TL, true, 0>(v, tw);
    if (G > 1) fft_reg<TL, true, (G > 1 ? TL : 0)>(v, tw);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int n2 = 0; n2 < TL; ++n2) buf[(j + c * TL) * S + n2] = v[c * TL + n2];
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) {
      const float2 w = stw[k1 * TL + j];
      v[k1] = cmul(buf[k1 * S + j], make_float2(w.x, -w.y));
    }
    fft_reg<32, true, 0>(v, tw);                        // y[TL n1 + j] at v[n1]
#pragma unroll
    for (int n1 = 0; n1 < 32; ++n1) {
      const int n = TL * n1 + j;
      if (valid && n < W) {
        float ya = v[n1].x;
        if (post) ya *= post[(size_t)pa * W + n];
        out[ra * W + n] = ya;
        if (hasb) {
          float yb = v[n1].y;
          if (post) yb *= post[(size_t)pb * W + n];
          out[rb * W + n] = yb;
        }
      }
    }
  }
}

// ------------------------------------------------------------ staged register FFT filter
// The register four-step filter above waits on its own row loads, and its
// 32-point transforms multiply by run-time twiddles, unit ones included.
// This version keeps every warp's next two units of rows in flight: each warp
// owns two shared-memory stages, and one lane issues 1-D bulk copies
// (cp.async.bulk, one per row, completing on the stage's mbarrier) for the
// unit after next as soon as the current unit's rows are in registers, so the
// HBM reads of later rows overlap the transforms of earlier ones.  The
// 32-point transforms use compile-time twiddles (multiplications by 1 and -i
// vanish) and paired FP32 adds (FADD2/FFMA2); the cosine weight is evaluated
// in place (SAD / sqrt(SAD^2 + s^2 + t^2), the formula of
// hoCuConebeamProjectionOperator.cpp:84-97) instead of read from a table; the
// sin^2 offset weights of the output row are fetched before the last inverse
// pass.  A unit is 2G consecutive rows (G transforms of two rows per warp);
// rows sit in the stage with a padded stride so the two half-warps of a
// 16-lane transform read different banks.

// cos(m pi / 16) for 0 <= m <= 8 from its Taylor series (exact at 0 and 8).
constexpr double cos_pi16(int m) {
  if (m == 0) return 1.0;
  if (m == 8) return 0.0;
  const double x = double(m) * (3.14159265358979323846 / 16.0);
  double term = 1.0, sum = 1.0;
  for (int k = 1; k < 16; ++k) {
    term *= -x * x / double((2 * k - 1) * (2 * k));
    sum += term;
  }
  return sum;
}

// a * W_32^M (W_32 = exp(-2 pi i / 32)), or a * conj(W_32^M) when INV.
// Build-time switches of the staged filter's arithmetic: complex products as
// one paired multiply and one paired fused multiply-add (CBCT_FDK_PACKED_CMUL),
// and the first butterfly stage of the zero-padded forward transform as
// copies (CBCT_FDK_ZPAD_STAGE: a + 0 and a - 0 are a, but for the sign of a
// zero input).
#ifndef CBCT_FDK_PACKED_CMUL
#define CBCT_FDK_PACKED_CMUL 0
#endif
#ifndef CBCT_FDK_ZPAD_STAGE
#define CBCT_FDK_ZPAD_STAGE 1
#endif

// a * b as (a.x b.x, a.x b.y) + (-a.y b.y, a.y b.x), paired.
__device__ __forceinline__ float2 cmul_p(float2 a, float2 b) {
  const float2 t = __fmul2_rn(make_float2(a.x, a.x), b);
  return __ffma2_rn(make_float2(-a.y, a.y), make_float2(b.y, b.x), t);
}

__device__ __forceinline__ float2 cmul_async(float2 a, float2 b) {
  return CBCT_FDK_PACKED_CMUL ? cmul_p(a, b) : cmul(a, b);
}

template <int M, bool INV>
__device__ __forceinline__ float2 tw32(float2 a) {
  static_assert(M >= 0 && M < 16, "twiddle index");
  if constexpr (M == 0) {
    return a;
  } else if constexpr (M == 8) {
    return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);   // * (+i) / * (-i)
  } else {
    constexpr float c = float(M <= 8 ? cos_pi16(M) : -cos_pi16(16 - M));
    constexpr float sn = float(M <= 8 ? cos_pi16(8 - M) : cos_pi16(M - 8));   // sin(M pi / 16)
    constexpr float wi = INV ? sn : -sn;
    if constexpr (CBCT_FDK_PACKED_CMUL) return cmul_p(a, make_float2(c, wi));
    return make_float2(fmaf(a.x, c, -a.y * wi), fmaf(a.x, wi, a.y * c));
  }
}

// Butterflies of stage LEN with offset K in every group of an N-point
// decimation-in-time transform held in v[OFF .. OFF + N).
template <int N, bool INV, int OFF, int NV, int LEN, int K>
__device__ __forceinline__ void dit_k(float2 (&v)[NV]) {
#pragma unroll
  for (int i = 0; i < N; i += LEN) {
    const float2 a = v[OFF + i + K];
    const float2 b = tw32<K * (32 / LEN), INV>(v[OFF + i + K + LEN / 2]);
    v[OFF + i + K] = __fadd2_rn(a, b);
    v[OFF + i + K + LEN / 2] = __ffma2_rn(b, make_float2(-1.f, -1.f), a);
  }
}

template <int N, bool INV, int OFF, int NV, int LEN, int... Ks>
__device__ __forceinline__ void dit_stage(float2 (&v)[NV], std::integer_sequence<int, Ks...>) {
  (dit_k<N, INV, OFF, NV, LEN, Ks>(v), ...);
}

template <int N, bool INV, int OFF, int NV, int LEN>
__device__ __forceinline__ void dit_stages(float2 (&v)[NV]) {
  if constexpr (LEN <= N) {
    dit_stage<N, INV, OFF, NV, LEN>(v, std::make_integer_sequence<int, LEN / 2>{});
    dit_stages<N, INV, OFF, NV, LEN * 2>(v);
  }
}

// In-register N-point DFT (N = 16 or 32), natural order in and out.  ZPAD:
// the upper half of the input is zero, so after the bit-reversal every odd
// position holds a zero and the first stage's butterflies are copies.
template <int N, bool INV, int OFF, int NV, bool ZPAD = false>
__device__ __forceinline__ void fft_ct(float2 (&v)[NV]) {
  constexpr int bits = N == 16 ? 4 : 5;
#pragma unroll
  for (int i = 0; i < N; ++i) {
    const int j = brev_bits(i, bits);
    if (j > i) {
      const float2 t = v[OFF + i];
      v[OFF + i] = v[OFF + j];
      v[OFF + j] = t;
    }
  }
  if constexpr (ZPAD) {
#pragma unroll
    for (int i = 0; i < N; i += 2) v[OFF + i + 1] = v[OFF + i];
    dit_stages<N, INV, OFF, NV, 4>(v);
  } else {
    dit_stages<N, INV, OFF, NV, 2>(v);
  }
}

// Cosine weight evaluated in place: w(u, v) = SAD / sqrt(SAD^2 + s^2 + t^2),
// s = su u + bu, t = sv v + bv.
struct CosWeight {
  int on;
  float sad, sad2;
  float su, bu, sv, bv;
};

#ifndef CBCT_FDK_ASYNC_WARPS
#define CBCT_FDK_ASYNC_WARPS 8
#endif
constexpr int kAsyncWarps = CBCT_FDK_ASYNC_WARPS;
// Stages per warp: with two, a unit's rows are in flight for two units'
// compute; with one, for one (the copy is issued as soon as the rows are read).
#ifndef CBCT_FDK_ASYNC_STAGES
#define CBCT_FDK_ASYNC_STAGES 1
#endif
constexpr int kAsyncStages = CBCT_FDK_ASYNC_STAGES;
#ifndef CBCT_FDK_ASYNC_MINB
#define CBCT_FDK_ASYNC_MINB 2
#endif

struct AsyncLayout {
  size_t stage_bytes, stages, tbuf, tw, spec, bars, total;
};

template <class T, int TL>
__host__ __device__ inline AsyncLayout async_layout(int Wp) {
  constexpr int G = 32 / TL, L = 32 * TL;
  AsyncLayout a{};
  a.stage_bytes = (size_t)2 * G * Wp * sizeof(T);
  a.stages = 0;
  a.tbuf = a.stages + (size_t)kAsyncWarps * kAsyncStages * a.stage_bytes;
  a.tw = a.tbuf + sizeof(float2) * (size_t)kAsyncWarps * G * 32 * (TL + 1);
  a.spec = a.tw + sizeof(float2) * 32 * TL;
  a.bars = a.spec + sizeof(float) * L;
  a.total = a.bars + sizeof(uint64_t) * kAsyncStages * kAsyncWarps;
  return a;
}

// Detector row and view of a row index, advanced by a fixed stride without a
// division per step: row r = p H + v.
struct RowPos {
  int p, v;
  __device__ __forceinline__ void advance(int dp, int dv, int H) {
    p += dp;
    v += dv;
    if (v >= H) {
      v -= H;
      ++p;
    }
  }
};

// One transform's two rows, loaded from the stage with the pre-weights:
// x[TL n1 + j] for n1 < 16 (the rest is the zero padding).  Rows past the end
// of the projections, and samples past the row's end, are zero (selects, no
// branches; every shared-memory read stays inside the kernel's allocation).
template <class T, int TL, bool COS, bool PK, bool FULL>
__device__ __forceinline__ void load_pair(float2 (&v)[32], const T* sa, const T* sb, int j, int W, bool oka, bool okb,
                                          const CosWeight& cw, float qa, float qb, const float* pka,
                                          const float* pkb) {
#pragma unroll
  for (int n1 = 0; n1 < 32; ++n1) {
    if (n1 >= 16) {
      v[n1] = make_float2(0.f, 0.f);
      continue;
    }
    const int n = TL * n1 + j;
    float xa = sm_f(sa[n]), xb = sm_f(sb[n]);
    if (COS) {
      const float su = fmaf(float(n), cw.su, cw.bu);
      xa *= cw.sad * rsqrtf(fmaf(su, su, qa));
      xb *= cw.sad * rsqrtf(fmaf(su, su, qb));
    }
    if (PK) {
      const int nc = FULL ? n : min(n, W - 1);
      xa *= __ldg(pka + nc);
      xb *= __ldg(pkb + nc);
    }
    const bool in_row = FULL || n < W;
    v[n1] = make_float2((oka && in_row) ? xa : 0.f, (okb && in_row) ? xb : 0.f);
  }
}

template <class T, int TL, bool COS, bool FULL>
__global__ void __launch_bounds__(kAsyncWarps * 32, CBCT_FDK_ASYNC_MINB) fdk_filter_async_kernel(
    const T* __restrict__ in, float* __restrict__ out, int W, int H, int rows, int Wp,
    const float* __restrict__ spec, const float2* __restrict__ twL, CosWeight cw, const float* __restrict__ parker,
    const float* __restrict__ post, unsigned wait_limit, int* flags) {
  constexpr int G = 32 / TL, L = 32 * TL, S = TL + 1, RU = 2 * G;
  extern __shared__ __align__(128) unsigned char smem[];
  const AsyncLayout lay = async_layout<T, TL>(Wp);
  float2* const tbuf = reinterpret_cast<float2*>(smem + lay.tbuf);
  float2* const stw = reinterpret_cast<float2*>(smem + lay.tw);
  float* const sspec = reinterpret_cast<float*>(smem + lay.spec);
  uint64_t* const bars = reinterpret_cast<uint64_t*>(smem + lay.bars);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int g = lane / TL, j = lane % TL;
  for (int i = threadIdx.x; i < 32 * TL; i += kAsyncWarps * 32) stw[i] = twL[i];
  for (int i = threadIdx.x; i < L; i += kAsyncWarps * 32) sspec[i] = spec[i];
  if (lane == 0) {
    for (int q = 0; q < kAsyncStages; ++q) mbar_init(&bars[kAsyncStages * warp + q], 1);
    fence_mbar_init();
  }
  __syncthreads();
  // From here on every warp works alone.
  unsigned char* const my_st = smem + lay.stages + (size_t)warp * kAsyncStages * lay.stage_bytes;
  float2* const buf = tbuf + ((size_t)warp * G + g) * 32 * S;
  const int nunits = (rows + RU - 1) / RU;
  const int w0 = blockIdx.x * kAsyncWarps + warp, nw = gridDim.x * kAsyncWarps;
  auto issue = [&](int unit, int st) {
    const int r0 = unit * RU;
    const int nr = rows - r0 < RU ? rows - r0 : RU;
    uint64_t* bar = &bars[kAsyncStages * warp + st];
    mbar_arrive_expect_tx(bar, uint32_t(nr) * uint32_t(W * sizeof(T)));
    for (int r = 0; r < nr; ++r)
      bulk_load(my_st + st * lay.stage_bytes + (size_t)r * Wp * sizeof(T), in + (size_t)(r0 + r) * W,
                uint32_t(W * sizeof(T)), bar);
  };
  if (lane == 0)
    for (int q = 0; q < kAsyncStages; ++q)
      if (w0 + q * nw < nunits) issue(w0 + q * nw, q);
  // Row a of this lane's transform and its stride per unit step.
  RowPos pos{(w0 * RU + 2 * g) / H, (w0 * RU + 2 * g) % H};
  const int step_p = (nw * RU) / H, step_v = (nw * RU) % H;
  int it = 0;
  for (int unit = w0; unit < nunits; unit += nw, ++it, pos.advance(step_p, step_v, H)) {
    const int st = it % kAsyncStages;
    const uint32_t par = (it / kAsyncStages) & 1;
    const bool ok = mbar_wait_bounded(&bars[kAsyncStages * warp + st], par, wait_limit);
    if (__any_sync(0xffffffffu, !ok)) {
      // Give up: record it, let the copies in flight land (default limit), leave.
      if (lane == 0) {
        atomicAdd(&flags[1], 1);
        for (int q = 0; q < kAsyncStages; ++q) {
          const int iq = it + q;
          if (unit + q * nw < nunits)
            (void)mbar_wait_bounded(&bars[kAsyncStages * warp + iq % kAsyncStages], (iq / kAsyncStages) & 1,
                                    kWaitLimit);
        }
      }
      __syncwarp();
      return;
    }
    const int ra = unit * RU + 2 * g;
    const bool oka = ra < rows, okb = ra + 1 < rows;
    const int pa = pos.p, vra = pos.v;
    const int pb = vra + 1 < H ? pa : pa + 1, vrb = vra + 1 < H ? vra + 1 : 0;
    const T* sa = reinterpret_cast<const T*>(my_st + st * lay.stage_bytes) + (size_t)(2 * g) * Wp;
    const T* sb = sa + Wp;
    const float ta = fmaf(float(vra), cw.sv, cw.bv), tb = fmaf(float(vrb), cw.sv, cw.bv);
    const float qa = fmaf(ta, ta, cw.sad2), qb = fmaf(tb, tb, cw.sad2);
    float2 v[32];
    if (parker) {
      // Parker rows of the pair's views (rows outside the projections read view 0's).
      const float* pka = parker + (size_t)(oka ? pa : 0) * W;
      const float* pkb = parker + (size_t)(okb ? pb : 0) * W;
      load_pair<T, TL, COS, true, FULL>(v, sa, sb, j, W, oka, okb, cw, qa, qb, pka, pkb);
    } else {
      load_pair<T, TL, COS, false, FULL>(v, sa, sb, j, W, oka, okb, cw, qa, qb, nullptr, nullptr);
    }
    __syncwarp();
    if (lane == 0 && unit + kAsyncStages * nw < nunits) {
      fence_proxy_async();   // the stage's reads above come before the copy that refills it
      issue(unit + kAsyncStages * nw, st);
    }
    fft_ct<32, false, 0, 32, CBCT_FDK_ZPAD_STAGE != 0>(v);   // v[k1]
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) v[k1] = cmul_async(v[k1], stw[k1 * TL + j]);
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) buf[k1 * S + j] = v[k1];
    __syncwarp();
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int n2 = 0; n2 < TL; ++n2) v[c * TL + n2] = buf[(j + c * TL) * S + n2];
    fft_ct<TL, false, 0>(v);
    if constexpr (G > 1) fft_ct<TL, false, TL>(v);
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int k2 = 0; k2 < TL; ++k2) {
        const float h = sspec[(j + c * TL) + 32 * k2];
        v[c * TL + k2] = __fmul2_rn(v[c * TL + k2], make_float2(h, h));
      }
    fft_ct<TL, true, 0>(v);
    if constexpr (G > 1) fft_ct<TL, true, TL>(v);
    __syncwarp();
#pragma unroll
    for (int c = 0; c < G; ++c)
#pragma unroll
      for (int n2 = 0; n2 < TL; ++n2) buf[(j + c * TL) * S + n2] = v[c * TL + n2];
    __syncwarp();
    // Offset weights of the output row a, fetched ahead of the last pass (row b
    // shares them unless the pair straddles two views).
    float pwa[16];
    const float* pob = post ? post + (size_t)(okb ? pb : 0) * W : nullptr;
    if (post) {
      const float* poa = post + (size_t)(oka ? pa : 0) * W;
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) pwa[n1] = __ldg(poa + (FULL ? TL * n1 + j : min(TL * n1 + j, W - 1)));
    } else {
#pragma unroll
      for (int n1 = 0; n1 < 16; ++n1) pwa[n1] = 1.f;
    }
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) {
      const float2 w = stw[k1 * TL + j];
      v[k1] = cmul_async(buf[k1 * S + j], make_float2(w.x, -w.y));
    }
    __syncwarp();
    fft_ct<32, true, 0>(v);                              // y[TL n1 + j] at v[n1]
    float* oa = out + (size_t)ra * W;
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) {
      const int n = TL * n1 + j;
      if (FULL || n < W) {
        if (oka) oa[n] = v[n1].x * pwa[n1];
        if (okb) oa[W + n] = v[n1].y * (pb == pa || !pob ? pwa[n1] : __ldg(pob + n));
      }
    }
  }
}

// In-place radix-2 FFT in double on the host (n a power of two), forward sign.
static void fft_host(std::vector<double>& re, std::vector<double>& im) {
  const size_t n = re.size();
  for (size_t i = 1, j = 0; i < n; ++i) {
    size_t bit = n >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      std::swap(re[i], re[j]);
      std::swap(im[i], im[j]);
    }
  }
  const double pi = 3.14159265358979323846;
  for (size_t len = 2; len <= n; len <<= 1) {
    const double ang = -2.0 * pi / double(len);
    for (size_t k = 0; k < len / 2; ++k) {
      const double wr = std::cos(ang * double(k)), wi = std::sin(ang * double(k));
      for (size_t i = k; i < n; i += len) {
        const size_t q = i + len / 2;
        const double xr = re[q] * wr - im[q] * wi, xi = re[q] * wi + im[q] * wr;
        re[q] = re[i] - xr;
        im[q] = im[i] - xi;
        re[i] += xr;
        im[i] += xi;
      }
    }
  }
}

// FP64 spectrum of the row filter on an L-point grid, scaled by 1/L.
// h[j] = (1/2W) (H[0] + (-1)^j H[W] + 2 sum_k H[k] cos(pi j k / W)), |j| < W, is
// summed with the angle-addition recurrence (exact cosines every 32 steps),
// and the spectrum of the even kernel on L points is one FFT of length L.
std::vector<float> filter_spectrum(const float* H, int W, int L) {
  std::vector<double> h(W);
  const double pi = 3.14159265358979323846;
  for (int j = 0; j < W; ++j) {
    double s = H[0] + ((j & 1) ? -1.0 : 1.0) * H[W];
    const double th = pi * double(j) / W, c1 = std::cos(th), s1 = std::sin(th);
    double c = c1, sn = s1;
    for (int k = 1; k < W; ++k) {
      if ((k & 31) == 0) {
        const double a = pi * double((long)j * k % (2L * W)) / W;
        c = std::cos(a);
        sn = std::sin(a);
      }
      s += 2.0 * H[k] * c;
      const double cn = c * c1 - sn * s1;
      sn = sn * c1 + c * s1;
      c = cn;
    }
    h[j] = s / (2.0 * W);
  }
  std::vector<double> re(L, 0.0), im(L, 0.0);
  re[0] = h[0];
  for (int j = 1; j < W; ++j) re[j] = re[L - j] = h[j];
  fft_host(re, im);
  std::vector<float> spec(L);
  for (int k = 0; k < L; ++k) spec[k] = float(re[k] / L);
  return spec;
}

struct FdkTables {
  float* spec = nullptr;
  float2* tw = nullptr;
  float2* twL = nullptr;    // register FFT: W_L^(n2 k1) at [k1 * TL + n2]
  float* cosw = nullptr;
  float* parker = nullptr;  // per view of the plan
  float* post = nullptr;    // per view of the plan
};

}  // namespace

// Per-plan FDK tables, created on first use (host-side allocation; not inside
// stream capture).
struct FdkState {
  FdkTables t;
  std::vector<float> filter;
  int L = 0, logL = 0;
  Tw32 tw32{};
};

void fdk_state_free(cbct_plan* p) {
  FdkState* f = static_cast<FdkState*>(p->fdk_state);
  if (!f) return;
  plan_dealloc(p, f->t.spec);
  plan_dealloc(p, f->t.tw);
  plan_dealloc(p, f->t.twL);
  plan_dealloc(p, f->t.cosw);
  plan_dealloc(p, f->t.parker);
  plan_dealloc(p, f->t.post);
  delete f;
  p->fdk_state = nullptr;
}

// Parker weights per (view, u) in FP64 (conebeam_projection.cu:169-194); the
// fan angle of each column is evaluated once per column.
static void build_parker(cbct_plan* p, FdkState* f) {
  if (f->t.parker) return;
  const int W = p->g.width, P = p->n_views;
  const double pi = 3.14159265358979323846, eps = 0.001, q = 0.1;
  const double delta = std::atan(p->g.fov_u / (2.0 * double(p->g.SDD)));
  const double tand = std::tan(delta);
  auto S = [&](double b) { return b <= -0.5 ? 0.0 : (b < 0.5 ? 0.5 * (1 + std::sin(pi * b)) : 1.0); };
  std::vector<double> alpha(W), bp(W), bm(W);
  for (int u = 0; u < W; ++u) {
    alpha[u] = -std::atan((double(u) / W - 0.5) * 2.0 * tand);
    bp[u] = q * (2 * (delta - alpha[u]) + eps);
    bm[u] = q * (2 * (delta + alpha[u]) + eps);
  }
  std::vector<float> pk((size_t)W * P);
  parallel_for(P, [&](int lo, int hi, int) {
    for (int v = lo; v < hi; ++v) {
      const double beta = p->angles[v] * (pi / 180.0);
      for (int u = 0; u < W; ++u) {
        const double a = alpha[u];
        const double om = 0.5 * (S(beta / bp[u] - 0.5) + S((beta + 2 * (a - delta) - eps) / bp[u] + 0.5) -
                                 S((beta - pi + 2 * a) / bm[u] - 0.5) - S((beta - pi - 2 * delta - eps) / bm[u] + 0.5));
        pk[(size_t)v * W + u] = float(om);
      }
    }
  });
  f->t.parker = plan_alloc_n<float>(p, pk.size());
  plan_upload(p, f->t.parker, pk.data(), sizeof(float) * pk.size());
}

// sin^2 offset weights per (view, u) in FP64 (conebeam_projection.cu:245-259);
// views with the same offset share one computed row.
static void build_post(cbct_plan* p, FdkState* f) {
  if (f->t.post) return;
  const int W = p->g.width, P = p->n_views;
  const double pi = 3.14159265358979323846, fov = p->g.fov_u;
  std::vector<float> po((size_t)W * P);
  std::map<float, int> row_of;
  for (int v = 0; v < P; ++v) {
    const float key = p->offsets[2 * (size_t)v];
    auto it = row_of.find(key);
    if (it != row_of.end()) {
      std::copy(po.begin() + (size_t)it->second * W, po.begin() + (size_t)(it->second + 1) * W, po.begin() + (size_t)v * W);
      continue;
    }
    row_of[key] = v;
    const double o = key, sg = o / std::fabs(o), omega = fov / 2.0 - std::fabs(o);
    for (int u = 0; u < W; ++u) {
      const double t = (fov * (double(u) / W - 0.5) + o) * sg;
      double w = 1.0;
      if (std::fabs(t) <= omega) {
        const double sw = std::sin(pi * (t + omega) / (4 * omega));
        w = sw * sw;
      }
      if (t < -omega) w = 0.0;
      po[(size_t)v * W + u] = float(w);
    }
  }
  f->t.post = plan_alloc_n<float>(p, po.size());
  plan_upload(p, f->t.post, po.data(), sizeof(float) * po.size());
}

static FdkState* fdk_state(cbct_plan* p, const float* filter) {
  const int W = p->g.width, H = p->g.height, P = p->n_views;
  FdkState* f = static_cast<FdkState*>(p->fdk_state);
  if (!f) {
    f = new FdkState();
    p->fdk_state = f;
    int L = 1, logL = 0;
    while (L < 2 * W - 1) { L <<= 1; ++logL; }
    if (L < 2) { L = 2; logL = 1; }
    f->L = L;
    f->logL = logL;
    std::vector<float2> tw(L / 2);
    const double pi = 3.14159265358979323846;
    for (int k = 0; k < L / 2; ++k)
      tw[k] = make_float2(float(std::cos(2 * pi * k / L)), float(-std::sin(2 * pi * k / L)));
    f->t.tw = plan_alloc_n<float2>(p, tw.size());
    plan_upload(p, f->t.tw, tw.data(), sizeof(float2) * tw.size());
    for (int m = 0; m < 16; ++m)
      f->tw32.w[m] = make_float2(float(std::cos(2 * pi * m / 32)), float(-std::sin(2 * pi * m / 32)));
    if (L == 512 || L == 1024) {
      const int TL = L / 32;
      std::vector<float2> twl((size_t)32 * TL);
      for (int k1 = 0; k1 < 32; ++k1)
        for (int n2 = 0; n2 < TL; ++n2) {
          const long e = (long)k1 * n2 % L;
          twl[(size_t)k1 * TL + n2] = make_float2(float(std::cos(2 * pi * e / L)), float(-std::sin(2 * pi * e / L)));
        }
      f->t.twL = plan_alloc_n<float2>(p, twl.size());
      plan_upload(p, f->t.twL, twl.data(), sizeof(float2) * twl.size());
    }
    f->t.spec = plan_alloc_n<float>(p, L);
    // Cosine weights (hoCuConebeamProjectionOperator.cpp:84-97): double, stored float.
    std::vector<float> cw((size_t)W * H);
    const double SAD = p->g.SAD, SDD = p->g.SDD;
    for (int y = 0; y < H; ++y)
      for (int x = 0; x < W; ++x) {
        const double xx = (double(x) / W - 0.5) * p->g.fov_u, yy = (double(y) / H - 0.5) * p->g.fov_v;
        const double s = SAD * xx / SDD, v = SAD * yy / SDD;
        cw[(size_t)y * W + x] = float(SAD / std::sqrt(SAD * SAD + s * s + v * v));
      }
    f->t.cosw = plan_alloc_n<float>(p, cw.size());
    plan_upload(p, f->t.cosw, cw.data(), sizeof(float) * cw.size());
    // The weight tables this plan's geometry calls for are made now (plan
    // set-up, outside any stream capture); others on first use.
    if (short_scan_rule(p->g, p->angles.data(), P)) build_parker(p, f);
    for (int v = 0; v < P; ++v)
      if (p->offsets[2 * (size_t)v] != 0.f) {
        build_post(p, f);
        break;
      }
  }
  std::vector<float> want(W + 1);
  if (filter) std::copy(filter, filter + W + 1, want.begin());
  else default_filter(W, want.data());
  if (want != f->filter) {
    std::vector<float> spec = filter_spectrum(want.data(), W, f->L);
    plan_upload(p, f->t.spec, spec.data(), sizeof(float) * f->L);
    f->filter = want;
  }
  return f;
}

void offset_weight_launch(cbct_plan* p, int s, const float* in, float* out, int variant,
                          cudaStream_t st) {
  const int first = p->first[s], cnt = p->count[s];
  const size_t n = (size_t)p->g.width * p->g.height * cnt;
  if (n == 0) return;
  const int blocks = (int)std::min<size_t>((n + 255) / 256, 148 * 16);
  offset_weight_kernel<<<blocks, 256, 0, st>>>(in, out, p->d_views + first, p->gc, cnt, variant);
  check_launch("offset_weight_kernel");
}

void fdk_prepare(cbct_plan* p, const float* filter) { fdk_state(p, filter); }

template <class T, int TL>
static void fdk_filter_reg(const void* in, float* out, int W, int H, long rows, const FdkState* f, const float* pre,
                           const float* pk, const float* post, cudaStream_t st) {
  // transpose buffers (32 x (TL + 1) per transform, 32 / TL transforms per
  // warp), twiddles (32 TL) and spectrum (32 TL floats)
  const size_t smem = sizeof(float2) * ((size_t)(kRegFftThreads / 32) * 32 * 32 * (TL + 1) / TL + 32 * TL) +
                      sizeof(float) * 32 * TL;
  auto k = fdk_filter_reg_kernel<T, TL>;
  ensure_smem_attr((const void*)k, smem);
  const long npairs = (rows + 1) / 2;
  const long per_block = (kRegFftThreads / 32) * (32 / TL);
  const int blocks = (int)std::min<long>((npairs + per_block - 1) / per_block, 148L * 16);
  k<<<blocks, kRegFftThreads, smem, st>>>(static_cast<const T*>(in), out, W, H, rows, f->t.spec, f->t.twL, f->tw32,
                                          pre, pk, post);
  check_launch("fdk_filter_reg_kernel");
}

// Row stride (elements) of a stage: W plus padding that keeps rows 16-byte
// aligned and puts the two rows read together by the half-warps of a 16-lane
// transform 16 banks apart.
template <class T>
static int async_row_stride(int W, int TL) {
  if (TL == 32) return W;   // one transform per warp: its two rows are read one at a time
  const int step = 16 / (int)sizeof(T);
  for (int pad = step; pad <= 8 * step; pad += step) {
    const int words = int(2 * (W + pad) * sizeof(T) / 4);
    if (words % 32 == 16) return W + pad;
  }
  return W + step;
}

// The staged filter for L = 512 / 1024 when rows can be bulk-copied (16-byte
// aligned rows); returns false to fall back to the register filter.
template <class T, int TL>
static bool fdk_filter_async(cbct_plan* p, const void* in, float* out, int W, int H, long rows, const FdkState* f,
                             bool cosine, const float* pk, const float* post, cudaStream_t st) {
  if ((W * sizeof(T)) % 16 != 0 || (reinterpret_cast<uintptr_t>(in) % 16) != 0) return false;
  const int Wp = async_row_stride<T>(W, TL);
  const AsyncLayout lay = async_layout<T, TL>(Wp);
  if (lay.total > (size_t)kSmemBudget) return false;
  if (rows > (long)INT32_MAX / 2) return false;
  const bool full = W == 16 * TL;
  auto k = cosine ? (full ? fdk_filter_async_kernel<T, TL, true, true> : fdk_filter_async_kernel<T, TL, true, false>)
                  : (full ? fdk_filter_async_kernel<T, TL, false, true> : fdk_filter_async_kernel<T, TL, false, false>);
  ensure_smem_attr((const void*)k, lay.total);
  int dev = 0, sms = 0, per_sm = 0;
  CBCT_CUDA(cudaGetDevice(&dev));
  CBCT_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
  CBCT_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, kAsyncWarps * 32, lay.total));
  if (per_sm < 1) return false;
  const long units = (rows + 2 * (32 / TL) - 1) / (2 * (32 / TL));
  const int blocks = (int)std::max<long>(1, std::min<long>((long)sms * per_sm, (units + kAsyncWarps - 1) / kAsyncWarps));
  CosWeight cw{};
  const cbct_geometry& g = p->g;
  cw.on = cosine ? 1 : 0;
  cw.sad = g.SAD;
  cw.sad2 = float(double(g.SAD) * g.SAD);
  cw.su = float(double(g.SAD) * g.fov_u / (double(g.SDD) * W));
  cw.bu = float(-0.5 * double(g.SAD) * g.fov_u / g.SDD);
  cw.sv = float(double(g.SAD) * g.fov_v / (double(g.SDD) * H));
  cw.bv = float(-0.5 * double(g.SAD) * g.fov_v / g.SDD);
  k<<<blocks, kAsyncWarps * 32, lay.total, st>>>(static_cast<const T*>(in), out, W, H, (int)rows, Wp, f->t.spec,
                                                  f->t.twL, cw, pk, post, p->gc.wait_limit, p->d_flags);
  check_launch("fdk_filter_async_kernel");
  return true;
}

template <class T>
static void fdk_filter_typed(cbct_plan* p, const void* in, float* out, int W, int H, long rows, const FdkState* f,
                             const float* pre, const float* pk, const float* post, cudaStream_t st) {
  const int L = f->L;
#ifndef CBCT_FDK_RADIX2_ONLY
#ifndef CBCT_FDK_NO_ASYNC
  if (L == 1024 && fdk_filter_async<T, 32>(p, in, out, W, H, rows, f, pre != nullptr, pk, post, st)) return;
  if (L == 512 && fdk_filter_async<T, 16>(p, in, out, W, H, rows, f, pre != nullptr, pk, post, st)) return;
#endif
  if (L == 1024) return fdk_filter_reg<T, 32>(in, out, W, H, rows, f, pre, pk, post, st);
  if (L == 512) return fdk_filter_reg<T, 16>(in, out, W, H, rows, f, pre, pk, post, st);
#endif
  const size_t smem = sizeof(float2) * (L + L / 2) + sizeof(float) * L;
  if (smem > 200 * 1024) throw Error(CBCT_ERR_UNSUPPORTED, "detector too wide for the FDK filter");
  ensure_smem_attr((const void*)fdk_filter_kernel<T>, smem);
  const long npairs = (rows + 1) / 2;
  const int blocks = (int)std::min<long>(npairs, 148L * 8);
  fdk_filter_kernel<T><<<blocks, kFftThreads, smem, st>>>(static_cast<const T*>(in), out, W, H, rows, L, f->logL,
                                                          f->t.spec, f->t.tw, pre, pk, post);
  check_launch("fdk_filter_kernel");
}

void fdk_filter_launch(cbct_plan* p, int s, const void* in, float* out, const float* filter,
                       uint32_t flags, cudaStream_t st, cbct_dtype in_dtype) {
  const int first = p->first[s], cnt = p->count[s];
  const int W = p->g.width, H = p->g.height;
  if (cnt == 0) return;
  FdkState* f = fdk_state(p, filter);
  const long rows = (long)H * cnt;
  const float* pre = (flags & CBCT_FDK_COSINE) ? f->t.cosw : nullptr;
  if (flags & CBCT_FDK_PARKER) build_parker(p, f);
  if (flags & CBCT_FDK_OFFSET) build_post(p, f);
  const float* pk = (flags & CBCT_FDK_PARKER) ? f->t.parker + (size_t)first * W : nullptr;
  const float* post = (flags & CBCT_FDK_OFFSET) ? f->t.post + (size_t)first * W : nullptr;
  if (!(flags & CBCT_FDK_RAMP)) {
    // Weights only: run the filter with a unit spectrum would waste work; use
    // the element-wise path instead.
    throw Error(CBCT_ERR_UNSUPPORTED, "cbct_fdk_filter without CBCT_FDK_RAMP is not implemented");
  }
  switch (in_dtype) {
    case CBCT_F32: fdk_filter_typed<float>(p, in, out, W, H, rows, f, pre, pk, post, st); break;
    case CBCT_F16: fdk_filter_typed<__half>(p, in, out, W, H, rows, f, pre, pk, post, st); break;
    case CBCT_BF16: fdk_filter_typed<__nv_bfloat16>(p, in, out, W, H, rows, f, pre, pk, post, st); break;
    default: throw Error(CBCT_ERR_INVALID_ARGUMENT, "unknown projection storage type");
  }
}

}  // namespace cbct
