// The C ABI (include/rtb200.h): contexts, scene residency, render and replay entry points.
// Every entry point locks the context, makes its device current and returns a status;
// errors carry a message retrievable with rtb_last_error.
#include <chrono>
#include <cstdio>
#include <cstring>

#include "rtb_internal.h"

namespace rtb {

rtb_status fail(rtb_context* ctx, rtb_status s, const std::string& msg) {
  if (ctx) ctx->last_error = msg;
  return s;
}

rtb_status cuda_fail(rtb_context* ctx, cudaError_t e, const char* what) {
  if (ctx) ctx->last_error = std::string(what) + ": " + cudaGetErrorString(e);
  return e == cudaErrorMemoryAllocation ? RTB_ERR_OUT_OF_MEMORY : RTB_ERR_CUDA;
}

void* stage(rtb_context* ctx, size_t bytes) {
  if (bytes > ctx->stage_bytes) {
    cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_stage);
    ctx->d_stage = nullptr;
    ctx->stage_bytes = 0;
    size_t want = bytes + bytes / 4 + 4096;
    if (cudaMalloc(&ctx->d_stage, want) != cudaSuccess) return nullptr;
    ctx->stage_bytes = want;
  }
  return ctx->d_stage;
}

void* pinned(rtb_context* ctx, size_t bytes) {
  if (bytes > ctx->pinned_bytes) {
    cudaStreamSynchronize(ctx->stream);
    cudaFreeHost(ctx->h_pinned);
    ctx->h_pinned = nullptr;
    ctx->pinned_bytes = 0;
    if (cudaMallocHost(&ctx->h_pinned, bytes) != cudaSuccess) return nullptr;
    ctx->pinned_bytes = bytes;
  }
  return ctx->h_pinned;
}

}  // namespace rtb

using namespace rtb;

namespace {
using Clock = std::chrono::steady_clock;
long long ns_since(Clock::time_point t0) {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(Clock::now() - t0).count();
}

struct Guard {
  rtb_context* ctx;
  std::lock_guard<std::mutex> lock;
  explicit Guard(rtb_context* c) : ctx(c), lock(c->mu) {
    cudaSetDevice(c->device);
    c->last_error.clear();
  }
};

rtb_status read_counters(rtb_context* ctx, long long* dst) {
  unsigned long long h[14];
  cudaError_t e = cudaMemcpy(h, ctx->d_work + 8, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "counter read-back");
  for (int k = 0; k < 14; ++k) dst[k] = (long long)h[k];
  return RTB_OK;
}
}  // namespace

namespace rtb {
namespace {
__global__ void k_arm_abort(int* words, int generation) {
  words[1] = generation;
  words[2] = 0;
}
}  // namespace

void arm_abort(rtb_context* ctx, cudaStream_t s) {
  k_arm_abort<<<1, 1, 0, s>>>(ctx->d_abort, ctx->abort_generation.load());
}
}  // namespace rtb

extern "C" {

const char* rtb_status_string(rtb_status s) {
  switch (s) {
    case RTB_OK: return "ok";
    case RTB_ERR_INVALID_ARGUMENT: return "invalid argument";
    case RTB_ERR_UNAVAILABLE: return "CUDA device unavailable";
    case RTB_ERR_CUDA: return "CUDA error";
    case RTB_ERR_OUT_OF_MEMORY: return "out of device memory";
    case RTB_ERR_UNSUPPORTED: return "unsupported configuration";
    case RTB_ERR_DEVICE_CHECK: return "device-side check failed";
    case RTB_ERR_WATCHDOG: return "kernel stopped by its work budget or an abort request";
    case RTB_ERR_LIMIT: return "size limit exceeded";
  }
  return "unknown status";
}

const char* rtb_last_error(const rtb_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

rtb_status rtb_context_create(int device, rtb_context** out) {
  if (!out) return RTB_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess || n <= 0) {
    cudaGetLastError();
    return RTB_ERR_UNAVAILABLE;
  }
  if (device < 0 || device >= n) return RTB_ERR_INVALID_ARGUMENT;
  rtb_context* ctx = new rtb_context();
  ctx->device = device;
  cudaError_t e = cudaSetDevice(device);
  cudaDeviceProp prop;
  if (e == cudaSuccess) e = cudaGetDeviceProperties(&prop, device);
  if (e != cudaSuccess) {
    delete ctx;
    return RTB_ERR_UNAVAILABLE;
  }
  ctx->sm_count = prop.multiProcessorCount;
  ctx->cc_major = prop.major;
  ctx->cc_minor = prop.minor;
  std::snprintf(ctx->name, sizeof(ctx->name), "%s", prop.name);
  if (prop.major < 10) {
    delete ctx;
    return RTB_ERR_UNAVAILABLE;  // built for sm_100a only
  }
  // Keep freed stream-ordered allocations in this process's default pool (the builder and
  // scene arenas allocate from it on every build).
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev0);
  if (e == cudaSuccess) e = cudaEventCreate(&ctx->ev1);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ctx->order_ev, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_work, 32 * sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaMalloc(&ctx->d_abort, 4 * sizeof(int));
  if (e == cudaSuccess) e = cudaMemset(ctx->d_abort, 0, 4 * sizeof(int));
  if (e != cudaSuccess) {
    rtb_context_destroy(ctx);
    return RTB_ERR_CUDA;
  }
  *out = ctx;
  return RTB_OK;
}

rtb_status rtb_context_destroy(rtb_context* ctx) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    cudaFree(ctx->d_work);
    cudaFree(ctx->d_abort);
    cudaFree(ctx->d_stage);
    cudaFree(ctx->d_tail);
    cudaFree(ctx->d_wave);
    cudaFreeHost(ctx->h_pinned);
    if (ctx->ev0) cudaEventDestroy(ctx->ev0);
    if (ctx->ev1) cudaEventDestroy(ctx->ev1);
    if (ctx->order_ev) cudaEventDestroy(ctx->order_ev);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
  }
  delete ctx;
  return RTB_OK;
}

rtb_status rtb_device_info(rtb_context* ctx, char* name, int name_len, int* cc_major, int* cc_minor,
                           int* sm_count) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  if (name && name_len > 0) std::snprintf(name, name_len, "%s", ctx->name);
  if (cc_major) *cc_major = ctx->cc_major;
  if (cc_minor) *cc_minor = ctx->cc_minor;
  if (sm_count) *sm_count = ctx->sm_count;
  return RTB_OK;
}

rtb_status rtb_scene_upload(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_bvh_desc* bvh,
                            rtb_scene** out) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  auto t0 = Clock::now();
  ctx_acquire(ctx, ctx->stream);
  rtb_status s = scene_create(ctx, desc, bvh, nullptr, nullptr, 0, nullptr, 0, nullptr, 0, out);
  ctx_release(ctx, ctx->stream);
  if (s == RTB_OK) ctx->last.upload_ns = ns_since(t0);
  return s;
}

rtb_status rtb_scene_build(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* config,
                           rtb_scene** out, rtb_bvh_stats* stats) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  auto t0 = Clock::now();
  ctx_acquire(ctx, ctx->stream);
  rtb_status s = build_bvh(ctx, desc, config, out, stats);
  ctx_release(ctx, ctx->stream);
  if (s == RTB_OK) ctx->last.upload_ns = ns_since(t0);
  return s;
}

rtb_status rtb_scene_build_with_options(rtb_context* ctx, const rtb_scene_desc* desc,
                                        const rtb_build_config* config,
                                        const rtb_build_options* options, rtb_scene** out,
                                        rtb_bvh_stats* stats) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  auto t0 = Clock::now();
  ctx_acquire(ctx, ctx->stream);
  rtb_status s = build_bvh_options(ctx, desc, config, options, out, stats);
  ctx_release(ctx, ctx->stream);
  if (s == RTB_OK) ctx->last.upload_ns = ns_since(t0);
  return s;
}

rtb_status rtb_scene_build_binned(rtb_context* ctx, const rtb_scene_desc* desc,
                                  const rtb_build_config* config, int bins, rtb_scene** out,
                                  rtb_bvh_stats* stats) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  auto t0 = Clock::now();
  ctx_acquire(ctx, ctx->stream);
  rtb_status s = build_bvh_binned(ctx, desc, config, bins, out, stats);
  ctx_release(ctx, ctx->stream);
  if (s == RTB_OK) ctx->last.upload_ns = ns_since(t0);
  return s;
}

rtb_status rtb_scene_bvh_sizes(rtb_context* ctx, const rtb_scene* scene, int* node_count,
                               int* ref_count, int* root_count) {
  if (!ctx || !scene) return RTB_ERR_INVALID_ARGUMENT;
  if (node_count) *node_count = scene->ref_node_count;
  if (ref_count) *ref_count = scene->ref_ref_count;
  if (root_count) *root_count = scene->ref_root_count;
  return RTB_OK;
}

rtb_status rtb_scene_download_bvh(rtb_context* ctx, const rtb_scene* scene, float* node_bounds,
                                  int* node_data, int* refs, int* roots) {
  if (!ctx || !scene) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  cudaError_t e = cudaSuccess;
  if (node_bounds && scene->ref_node_count)
    e = cudaMemcpy(node_bounds, scene->ref_node_bounds, (size_t)scene->ref_node_count * 24, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && node_data && scene->ref_node_count)
    e = cudaMemcpy(node_data, scene->ref_node_data, (size_t)scene->ref_node_count * 16, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && refs && scene->ref_ref_count)
    e = cudaMemcpy(refs, scene->ref_refs, (size_t)scene->ref_ref_count * 4, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && roots && scene->ref_root_count)
    e = cudaMemcpy(roots, scene->ref_roots, (size_t)scene->ref_root_count * 4, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH download");
  return RTB_OK;
}

rtb_status rtb_scene_destroy(rtb_context* ctx, rtb_scene* scene) {
  if (!ctx || !scene) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  ctx_acquire(ctx, ctx->stream);
  scene_free(scene, ctx->stream);
  ctx_release(ctx, ctx->stream);
  return RTB_OK;
}

rtb_status rtb_trace_replay(rtb_context* ctx, rtb_scene* scene, const float* rays, int ray_count,
                            int use_bvh, int collect_metrics, int* hit_flags, float* hit_distances,
                            int* hit_orders, int* hit_materials, float* hit_normals) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  if (!scene || !rays || ray_count <= 0 || !hit_flags || !hit_distances || !hit_orders ||
      !hit_materials || !hit_normals)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "Replay rays must contain origin.xyz and direction.xyz.");
  auto t0 = Clock::now();
  size_t n = (size_t)ray_count;
  size_t bytes = n * (24 + 4 + 4 + 4 + 4 + 12) + 6 * 256;
  char* sb = (char*)stage(ctx, bytes);
  if (!sb) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "replay staging");
  auto al = [](size_t v) { return (v + 255) & ~size_t(255); };
  float* d_rays = (float*)sb;
  size_t o = al(n * 24);
  int* d_f = (int*)(sb + o);
  o += al(n * 4);
  float* d_t = (float*)(sb + o);
  o += al(n * 4);
  int* d_o = (int*)(sb + o);
  o += al(n * 4);
  int* d_m = (int*)(sb + o);
  o += al(n * 4);
  float* d_n = (float*)(sb + o);
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  cudaMemcpyAsync(d_rays, rays, n * 24, cudaMemcpyHostToDevice, sm);
  cudaEventRecord(ctx->ev0, sm);
  rtb_status s = trace_rays(ctx, scene, d_rays, ray_count, use_bvh, collect_metrics, d_f, d_t, d_o, d_m, d_n, sm);
  if (s != RTB_OK) return s;
  cudaEventRecord(ctx->ev1, sm);
  cudaMemcpyAsync(hit_flags, d_f, n * 4, cudaMemcpyDeviceToHost, sm);
  cudaMemcpyAsync(hit_distances, d_t, n * 4, cudaMemcpyDeviceToHost, sm);
  cudaMemcpyAsync(hit_orders, d_o, n * 4, cudaMemcpyDeviceToHost, sm);
  cudaMemcpyAsync(hit_materials, d_m, n * 4, cudaMemcpyDeviceToHost, sm);
  cudaMemcpyAsync(hit_normals, d_n, n * 12, cudaMemcpyDeviceToHost, sm);
  ctx_release(ctx, sm);
  cudaError_t e = cudaStreamSynchronize(sm);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trace replay");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  ctx->last = rtb_frame_stats{};
  ctx->last.kernel_ns = (long long)(ms * 1e6);
  ctx->last.max_physical_kernel_ns = ctx->last.kernel_ns;
  ctx->last.physical_launches = 1;
  if (collect_metrics) {
    s = read_counters(ctx, ctx->last.counters);
    if (s != RTB_OK) return s;
  }
  ctx->last.total_ns = ns_since(t0);
  return RTB_OK;
}

rtb_status rtb_render_device(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                             const rtb_render_params* params, float* rgb_device, void* stream) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  cudaStream_t sm = stream ? (cudaStream_t)stream : ctx->stream;
  ctx_acquire(ctx, sm);
  arm_abort(ctx, sm);
  rtb_status s = render_frame(ctx, scene, camera, params, rgb_device, sm, false);
  ctx_release(ctx, sm);
  return s;
}

rtb_status rtb_render_device_wavefront(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                                       const rtb_render_params* params, float* rgb_device,
                                       void* stream) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  cudaStream_t sm = stream ? (cudaStream_t)stream : ctx->stream;
  ctx_acquire(ctx, sm);
  arm_abort(ctx, sm);
  rtb_status s = render_frame_wavefront(ctx, scene, camera, params, rgb_device, sm);
  ctx_release(ctx, sm);
  return s;
}

rtb_status rtb_render_rows_device(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                                  const rtb_render_params* params, int first_row, int row_stride,
                                  float* rgb_device, void* stream) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  cudaStream_t sm = stream ? (cudaStream_t)stream : ctx->stream;
  ctx_acquire(ctx, sm);
  arm_abort(ctx, sm);
  rtb_status s = render_frame(ctx, scene, camera, params, rgb_device, sm, false, first_row,
                              row_stride);
  ctx_release(ctx, sm);
  return s;
}

rtb_status rtb_render_sample(rtb_context* ctx, rtb_scene* scene, const rtb_camera* camera,
                             const rtb_render_params* params, float* rgb) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  Guard g(ctx);
  if (!rgb || !params) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "RGB output is required");
  auto t0 = Clock::now();
  size_t bytes = (size_t)params->width * params->height * 12;
  float* d_rgb = (float*)stage(ctx, bytes);
  if (!d_rgb) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "output staging");
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  arm_abort(ctx, sm);
  rtb_status s = render_frame(ctx, scene, camera, params, d_rgb, sm, true);
  ctx_release(ctx, sm);
  if (s != RTB_OK) return s;
  cudaError_t e = cudaEventSynchronize(ctx->ev1);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render");
  int aborted = 0;  // abort word [2]: the kernel stopped fetching work
  cudaMemcpy(&aborted, ctx->d_abort + 2, sizeof(int), cudaMemcpyDeviceToHost);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  auto tc = Clock::now();
  e = cudaMemcpy(rgb, d_rgb, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "image read-back");
  rtb_frame_stats st{};
  st.copy_ns = ns_since(tc);
  st.kernel_ns = (long long)(ms * 1e6);
  st.max_physical_kernel_ns = st.kernel_ns;
  st.physical_launches = ctx->render_launches;
  st.upload_ns = 0;
  if (params->collect_metrics) {
    s = read_counters(ctx, st.counters);
    if (s != RTB_OK) return s;
  }
  st.total_ns = ns_since(t0);
  ctx->last = st;
  if (aborted) return fail(ctx, RTB_ERR_WATCHDOG, "render aborted on request");
  return RTB_OK;
}

rtb_status rtb_last_frame_stats(rtb_context* ctx, rtb_frame_stats* out) {
  if (!ctx || !out) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  *out = ctx->last;
  return RTB_OK;
}

rtb_status rtb_request_abort(rtb_context* ctx) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  // Not under the context mutex: it must reach a render that holds it.  Requests are
  // serialised among themselves so that generations land in increasing order, and a
  // generation is published (taken by later submissions) only once it is on the device:
  // work submitted before this call sees a generation above its own and stops; work
  // submitted after it never does.
  std::lock_guard<std::mutex> lock(ctx->abort_mu);
  int next = ctx->abort_generation.load() + 1;
  cudaSetDevice(ctx->device);
  cudaStream_t s;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return RTB_ERR_CUDA;
  cudaError_t e = cudaMemcpyAsync(ctx->d_abort, &next, sizeof(int), cudaMemcpyHostToDevice, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  cudaStreamDestroy(s);
  if (e != cudaSuccess || e2 != cudaSuccess) return RTB_ERR_CUDA;
  ctx->abort_generation.store(next);
  return RTB_OK;
}

}  // extern "C"
