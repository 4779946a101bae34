// autotune.cu -- choose the projector variants of a plan by timing them.
//
// Which forward projector is fastest depends on the geometry: the slab kernel
// (16x16 ray tiles, per-ray trilinear samples from TMA boxes), the row-pair
// and row-quad kernels (two or four rays of a column per thread sharing their
// in-plane interpolation), the fan kernel (8x32 tiles, e/d interpolation shared by a
// detector column; larger boxes), or the gather kernel (no staging); likewise
// the TMA-staged and the plain back-projector.  The autotuner runs every
// candidate the plan can use on the plan's largest subset (one warm-up and
// three timed launches each, CUDA events on the caller's stream) and keeps the
// fastest.  All candidates give
// results within FP32 rounding of each other (slab, pair, quad and fan bitwise
// equal).
// No counterpart in the reference.
#include <vector>

#include "cbct_internal.h"

namespace cbct {

void fill_launch(float* x, size_t n, float v, cudaStream_t st);

namespace {

template <class F>
float time_ms(cudaStream_t st, F&& f) {
  cudaEvent_t a, b;
  CBCT_CUDA(cudaEventCreate(&a));
  CBCT_CUDA(cudaEventCreate(&b));
  f();  // warm-up
  CBCT_CUDA(cudaEventRecord(a, st));
  for (int i = 0; i < 3; ++i) f();
  CBCT_CUDA(cudaEventRecord(b, st));
  CBCT_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  CBCT_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  return ms / 3.f;
}

}  // namespace

void plan_autotune(cbct_plan* p, float* times, cudaStream_t st) {
  CBCT_REQUIRE(p != nullptr, "plan is NULL");
  for (int i = 0; i < 7; ++i) times[i] = -1.f;
  int s = 0;
  for (int k = 1; k < p->n_subsets; ++k)
    if (p->count[k] > p->count[s]) s = k;
  const size_t nv = (size_t)p->g.nx * p->g.ny * p->g.nz;
  const size_t np = (size_t)p->g.width * p->g.height * p->count[s];
  float* vol = plan_alloc_n<float>(p, nv);
  float* proj = plan_alloc_n<float>(p, np);
  try {
    fill_launch(vol, nv, 0.01f, st);
    fill_launch(proj, np, 0.01f, st);
    // forward: slab (1), fan (3), gather (2), pairs (4), quads (5); the variant
    // must be the one asked for; slot = its entry of times[]
    const int prefs[5] = {1, 3, 2, 4, 5}, want[5] = {1, 2, 0, 3, 4}, slot[5] = {0, 1, 2, 5, 6};
    const int saved_pref = p->fwd_pref;
    int best = -1;
    float best_ms = 0.f;
    for (int c = 0; c < 5; ++c) {
      p->fwd_pref = prefs[c];
      forward_choose_variant(p);
      forward_prepare(p);
      if (p->fwd_variant != want[c]) continue;
      const float ms = time_ms(st, [&] {
        forward_launch(p, s, CBCT_F32, vol, proj, nullptr, 1.f, 0, 0, 0, nullptr, st);
      });
      times[slot[c]] = ms;
      if (best < 0 || ms < best_ms) { best = c; best_ms = ms; }
    }
    p->fwd_pref = best >= 0 ? prefs[best] : saved_pref;
    forward_choose_variant(p);
    forward_prepare(p);
    // back-projection: TMA-staged boxes (pref 0) or global loads (pref 1)
    const int saved_bp = p->bp_pref;
    int bbest = -1;
    float bbest_ms = 0.f;
    for (int c = 0; c < 2; ++c) {
      p->bp_pref = c;
      backproject_choose_variant(p);
      backproject_prepare(p);
      if (c == 0 && p->bp_variant != 1) continue;
      times[3 + c] = time_ms(st, [&] { backproject_launch(p, s, proj, vol, 0, 0, 1.f, st); });
      if (bbest < 0 || times[3 + c] < bbest_ms) { bbest = c; bbest_ms = times[3 + c]; }
    }
    p->bp_pref = bbest >= 0 ? bbest : saved_bp;
    backproject_choose_variant(p);
    backproject_prepare(p);
  } catch (...) {
    plan_dealloc(p, vol);
    plan_dealloc(p, proj);
    throw;
  }
  CBCT_CUDA(cudaStreamSynchronize(st));
  plan_dealloc(p, vol);
  plan_dealloc(p, proj);
  graph_cache_free(p);
  plan_check_flags(p, st);   // a variant that failed on the device must not pass as a timing
}

}  // namespace cbct
