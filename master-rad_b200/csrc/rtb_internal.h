// Host-side internals shared by the library's translation units.
#pragma once
#include <cuda_runtime.h>

#include <atomic>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/rtb200.h"
#include "rtb_device.cuh"

struct rtb_context {
  int device = 0;
  int sm_count = 0;
  int cc_major = 0, cc_minor = 0;
  char name[256] = {0};
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // Orders all device work of the context across streams: the work queue, counters and
  // staging buffers below are shared, so a launch on one stream must not overlap the
  // context's previous launch on another.
  cudaEvent_t order_ev = nullptr;
  bool order_pending = false;
  std::mutex mu;
  std::string last_error;
  rtb_frame_stats last{};
  // Small device scratch: [0] pixel queue head (u64), [1..] status words, counters.
  unsigned long long* d_work = nullptr;
  // Abort words in device memory (see abort_raised): [0] generation, [1] generation at
  // submit, [2] stopped.  abort_generation is the last generation on the device; abort_mu
  // serialises rtb_request_abort calls.
  int* d_abort = nullptr;
  std::atomic<int> abort_generation{0};
  std::mutex abort_mu;
  // Replay / output staging reused across calls.
  void* d_stage = nullptr;
  size_t stage_bytes = 0;
  void* h_pinned = nullptr;
  size_t pinned_bytes = 0;
  // Per-sample radiance of the frame's last pixels (rendered one sample per lane).
  float* d_tail = nullptr;
  size_t tail_bytes = 0;
  // Path state of the wavefront form, grown to the largest frame rendered in that form.
  void* d_wave = nullptr;
  size_t wave_bytes = 0;
  int render_launches = 0;  // kernels the last render_frame launched
};

struct rtb_scene {
  // One arena holds every device array of the scene.
  void* arena = nullptr;
  size_t arena_bytes = 0;
  rtb::DevScene dev{};
  // Reference-layout BVH kept on the device for download (topology checks).
  float* ref_node_bounds = nullptr;
  int* ref_node_data = nullptr;
  int* ref_refs = nullptr;
  int* ref_roots = nullptr;
  int ref_node_count = 0, ref_ref_count = 0, ref_root_count = 0;
  bool has_bvh = false;
  int device = 0;  // the device the scene is resident on
  std::vector<void*> extra;  // additional allocations freed with the scene
};

namespace rtb {

// Makes `s` wait for the context's previous device work, and marks `s` as holding the
// latest.  Every entry point that enqueues work brackets it with these.
inline void ctx_acquire(rtb_context* ctx, cudaStream_t s) {
  if (ctx->order_pending) cudaStreamWaitEvent(s, ctx->order_ev, 0);
}
inline void ctx_release(rtb_context* ctx, cudaStream_t s) {
  cudaEventRecord(ctx->order_ev, s);
  ctx->order_pending = true;
}

// Enqueues, on `s`, the write of the current abort generation as the submitted work's own
// and the clearing of the stopped word.  Every launch of a persistent kernel is preceded by
// it (outside any graph capture: the generation is a kernel argument).
void arm_abort(rtb_context* ctx, cudaStream_t s);

// Status helpers.
rtb_status fail(rtb_context* ctx, rtb_status s, const std::string& msg);
rtb_status cuda_fail(rtb_context* ctx, cudaError_t e, const char* what);

// Device staging buffer of at least `bytes` (grown on demand, owned by the context).
void* stage(rtb_context* ctx, size_t bytes);
void* pinned(rtb_context* ctx, size_t bytes);

// rtb_scene.cu
rtb_status scene_create(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_bvh_desc* host_bvh,
                        const float* d_node_bounds, const int* d_node_data, int node_count,
                        const int* d_refs, int ref_count, const int* d_roots, int root_count,
                        rtb_scene** out);
void scene_free(rtb_scene* s, cudaStream_t stream);

// rtb_render.cu
// Rows row0, row0 + row_stride, ... of the frame, packed densely into d_rgb (0, 1: the
// whole frame).
rtb_status render_frame(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                        const rtb_render_params* p, float* d_rgb, cudaStream_t stream,
                        bool timed, int row0 = 0, int row_stride = 1);
// The same frame in the wavefront form (whole frames, no metrics build).
rtb_status render_frame_wavefront(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                                  const rtb_render_params* p, float* d_rgb, cudaStream_t stream);
// One frame's launch, planned apart from where it runs (the batch's frames mode launches
// many into one graph).  plan_frame validates and sizes; bind_frame gives it a queue head
// (zeroed before launch), a sample buffer of frame_tail_bytes (nullptr: no single-sample
// tail), the abort flag and 14 counters; launch_frame enqueues its kernels and returns how
// many.
struct FramePlan;
FramePlan* new_frame_plan();
void delete_frame_plan(FramePlan* f);
// tail_per_thread: pixels per resident thread queued one sample per item at the frame's
// end (0: the default).
rtb_status plan_frame(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                      const rtb_render_params* p, float* d_rgb, FramePlan* f, int row0 = 0,
                      int row_stride = 1, int tail_per_thread = 0);
size_t frame_tail_bytes(const FramePlan* f);
void bind_frame(FramePlan* f, unsigned long long* queue, float* tail, int* abort_flag,
                unsigned long long* counters);
int launch_frame(const FramePlan* f, cudaStream_t stream);
// Closest-hit launch without a context (no counters, no allocation).
cudaError_t launch_trace(const DevScene& scene, int use_bvh, const float* d_rays, int n, int* d_flags,
                         float* d_t, int* d_order, int* d_mat, float* d_normal, cudaStream_t stream);
rtb_status trace_rays(rtb_context* ctx, rtb_scene* scene, const float* d_rays, int n, int use_bvh,
                      int collect_metrics, int* d_flags, float* d_t, int* d_order, int* d_mat,
                      float* d_normal, cudaStream_t stream);

// rtb_build.cu
rtb_status build_bvh(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                     rtb_scene** out, rtb_bvh_stats* stats);
rtb_status build_bvh_options(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                             const rtb_build_options* options, rtb_scene** out, rtb_bvh_stats* stats);

// rtb_sbvh.cu: the SBVH modes (4, 5), built on the host in depth-first order.
rtb_status build_bvh_sbvh(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                          const rtb_build_options* options, rtb_scene** out, rtb_bvh_stats* stats);

// rtb_binned.cu
rtb_status build_bvh_binned(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                            int bins, rtb_scene** out, rtb_bvh_stats* stats);

}  // namespace rtb
