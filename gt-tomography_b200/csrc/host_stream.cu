// host_stream.cu -- host-array operators streamed through the device in
// batches of views: hoCuConebeamProjectionOperator::mult_M / mult_MH
// (hoCuConebeamProjectionOperator.cpp:104-265) over the reference's host-array
// projectors (conebeam_projection.cu:640-819 forward, :1300-1649 backward and
// FDK).  As there, the volume of one bin stays on the device and the bin's
// projections pass through two device batch buffers, so projection data of
// any size (host memory permitting) streams through a fixed device
// footprint.  Here the plan's subsets are the batches, one compute stream
// runs the kernels and one copy stream moves batches, with events between
// them: while batch i is projected (or back-projected), batch i-1 leaves (or
// batch i+1 arrives).  Copies between a batch buffer (plan view order) and the
// host array (acquisition order) take one transfer per run of consecutive
// acquisition indices (conebeam_projection.cu:744-761).  Host arrays should be
// page-locked for the transfers to overlap the kernels; the calls return once
// the host outputs are written.
#include <vector>

#include "cbct_internal.h"

namespace cbct {

void offset_weight_launch(cbct_plan* p, int s, const float* in, float* out, int variant, cudaStream_t st);
void backproject_launch(cbct_plan* p, int s, const float* proj, float* vol, int fdk_weight, int accumulate,
                        float out_scale, cudaStream_t st);

namespace {

// Two streams and the events between them, released on every exit path.
struct Pipe {
  cudaStream_t compute = nullptr, copy = nullptr;
  std::vector<cudaEvent_t> events;
  Pipe() {
    CBCT_CUDA(cudaStreamCreateWithFlags(&compute, cudaStreamNonBlocking));
    CBCT_CUDA(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
  }
  ~Pipe() {
    if (compute) cudaStreamSynchronize(compute);
    if (copy) cudaStreamSynchronize(copy);
    for (cudaEvent_t e : events) cudaEventDestroy(e);
    if (compute) cudaStreamDestroy(compute);
    if (copy) cudaStreamDestroy(copy);
  }
  cudaEvent_t record(cudaStream_t s) {
    cudaEvent_t e;
    CBCT_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    events.push_back(e);
    CBCT_CUDA(cudaEventRecord(e, s));
    return e;
  }
};

void copy_views(float* dev, float* host, const int* view_index, int first, int count, size_t plane,
                cudaMemcpyKind kind, cudaStream_t st) {
  for (int i = 0; i < count;) {
    int n = 1;
    while (i + n < count && view_index[first + i + n] == view_index[first + i + n - 1] + 1) ++n;
    float* h = host + (size_t)view_index[first + i] * plane;
    float* d = dev + (size_t)i * plane;
    const size_t bytes = (size_t)n * plane * sizeof(float);
    if (kind == cudaMemcpyDeviceToHost) CBCT_CUDA(cudaMemcpyAsync(h, d, bytes, kind, st));
    else CBCT_CUDA(cudaMemcpyAsync(d, h, bytes, kind, st));
    i += n;
  }
}

// Plan-owned batch buffers and bin volume (grown on demand, reused).
void stream_buffers(cbct_plan* p, size_t batch_elems, float** buf, float** vol) {
  if (p->stream_buf_elems < batch_elems) {
    plan_dealloc(p, p->d_stream_buf[0]);
    plan_dealloc(p, p->d_stream_buf[1]);
    p->d_stream_buf[0] = p->d_stream_buf[1] = nullptr;
    p->stream_buf_elems = 0;
    p->d_stream_buf[0] = plan_alloc_n<float>(p, batch_elems);
    p->d_stream_buf[1] = plan_alloc_n<float>(p, batch_elems);
    p->stream_buf_elems = batch_elems;
  }
  if (!p->d_stream_vol) p->d_stream_vol = plan_alloc_n<float>(p, (size_t)p->g.nx * p->g.ny * p->g.nz);
  buf[0] = p->d_stream_buf[0];
  buf[1] = p->d_stream_buf[1];
  *vol = p->d_stream_vol;
}

void check_range(const cbct_plan* p, int s0, int ns, const int* view_index) {
  CBCT_REQUIRE(p != nullptr && view_index != nullptr, "NULL argument");
  CBCT_REQUIRE(s0 >= 0 && ns >= 0 && s0 + ns <= p->n_subsets, "batch range outside the plan's subsets");
  for (int i = 0; i < p->n_views; ++i) CBCT_REQUIRE(view_index[i] >= 0, "negative view index");
}

size_t largest_batch(const cbct_plan* p, int s0, int ns) {
  int m = 0;
  for (int s = s0; s < s0 + ns; ++s) m = std::max(m, p->count[s]);
  return (size_t)m * p->g.width * p->g.height;
}

}  // namespace

void host_forward(cbct_plan* p, int s0, int ns, const float* vol_host, float* proj_host, const int* view_index,
                  int offset_sqrt, cudaStream_t caller) {
  check_range(p, s0, ns, view_index);
  CBCT_REQUIRE(vol_host && proj_host, "NULL array");
  if (ns == 0) return;
  const size_t plane = (size_t)p->g.width * p->g.height, nv = (size_t)p->g.nx * p->g.ny * p->g.nz;
  float* buf[2];
  float* vol;
  stream_buffers(p, largest_batch(p, s0, ns), buf, &vol);
  Pipe pipe;
  cudaEvent_t start;
  CBCT_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  pipe.events.push_back(start);
  CBCT_CUDA(cudaEventRecord(start, caller));
  CBCT_CUDA(cudaStreamWaitEvent(pipe.compute, start, 0));
  CBCT_CUDA(cudaStreamWaitEvent(pipe.copy, start, 0));
  CBCT_CUDA(cudaMemcpyAsync(vol, vol_host, nv * sizeof(float), cudaMemcpyHostToDevice, pipe.compute));
  std::vector<cudaEvent_t> copied(ns);
  for (int i = 0; i < ns; ++i) {
    const int s = s0 + i;
    float* b = buf[i & 1];
    if (i >= 2) CBCT_CUDA(cudaStreamWaitEvent(pipe.compute, copied[i - 2], 0));  // buffer drained
    forward_launch_ex(p, s, CBCT_F32, vol, b, nullptr, nullptr, 1.f, 0, 0, 0, nullptr, pipe.compute);
    // mult_M's offset weight (sqrt variant) when not in FBP mode (.cpp:168-169)
    if (offset_sqrt) offset_weight_launch(p, s, b, b, 1, pipe.compute);
    CBCT_CUDA(cudaStreamWaitEvent(pipe.copy, pipe.record(pipe.compute), 0));
    copy_views(b, proj_host, view_index, p->first[s], p->count[s], plane, cudaMemcpyDeviceToHost, pipe.copy);
    copied[i] = pipe.record(pipe.copy);
  }
  CBCT_CUDA(cudaStreamSynchronize(pipe.copy));
  CBCT_CUDA(cudaStreamSynchronize(pipe.compute));
  plan_check_flags(p, pipe.compute);
}

void host_backproject(cbct_plan* p, int s0, int ns, const float* proj_host, float* vol_host, const int* view_index,
                      int fbp, const float* filter, uint32_t fdk_flags, int offset_sqrt, float scale, int accumulate,
                      cudaStream_t caller) {
  check_range(p, s0, ns, view_index);
  CBCT_REQUIRE(vol_host && proj_host, "NULL array");
  const size_t plane = (size_t)p->g.width * p->g.height, nv = (size_t)p->g.nx * p->g.ny * p->g.nz;
  float* buf[2];
  float* vol;
  stream_buffers(p, std::max<size_t>(largest_batch(p, s0, ns), plane), buf, &vol);
  if (fbp) fdk_prepare(p, filter);
  Pipe pipe;
  cudaEvent_t start;
  CBCT_CUDA(cudaEventCreateWithFlags(&start, cudaEventDisableTiming));
  pipe.events.push_back(start);
  CBCT_CUDA(cudaEventRecord(start, caller));
  CBCT_CUDA(cudaStreamWaitEvent(pipe.compute, start, 0));
  CBCT_CUDA(cudaStreamWaitEvent(pipe.copy, start, 0));
  if (accumulate) CBCT_CUDA(cudaMemcpyAsync(vol, vol_host, nv * sizeof(float), cudaMemcpyHostToDevice, pipe.compute));
  else if (ns == 0) CBCT_CUDA(cudaMemsetAsync(vol, 0, nv * sizeof(float), pipe.compute));
  std::vector<cudaEvent_t> consumed(ns);
  for (int i = 0; i < ns; ++i) {
    const int s = s0 + i;
    float* b = buf[i & 1];
    if (i >= 2) CBCT_CUDA(cudaStreamWaitEvent(pipe.copy, consumed[i - 2], 0));  // buffer free again
    copy_views(b, const_cast<float*>(proj_host), view_index, p->first[s], p->count[s], plane,
               cudaMemcpyHostToDevice, pipe.copy);
    CBCT_CUDA(cudaStreamWaitEvent(pipe.compute, pipe.record(pipe.copy), 0));
    if (fbp) {
      // cosine -> [Parker] -> ramp -> [sin^2 offset] per batch (conebeam_projection.cu:1483-1521)
      fdk_filter_launch(p, s, b, b, filter, fdk_flags | CBCT_FDK_RAMP | CBCT_FDK_COSINE, pipe.compute);
    } else if (offset_sqrt) {
      offset_weight_launch(p, s, b, b, 1, pipe.compute);  // offset_correct_sqrt (:1528-1529)
    }
    // vol = scale * (vol + batch): the bin's 2/P scale (.cpp:253) rides on the last batch.
    backproject_launch(p, s, b, vol, fbp, (i > 0 || accumulate) ? 1 : 0, i == ns - 1 ? scale : 1.f, pipe.compute);
    consumed[i] = pipe.record(pipe.compute);
  }
  CBCT_CUDA(cudaMemcpyAsync(vol_host, vol, nv * sizeof(float), cudaMemcpyDeviceToHost, pipe.compute));
  CBCT_CUDA(cudaStreamSynchronize(pipe.compute));
  CBCT_CUDA(cudaStreamSynchronize(pipe.copy));
  plan_check_flags(p, pipe.compute);
}

}  // namespace cbct
