// Oracle (test infrastructure only): a launcher for the reference's own CUDA kernels.
//
// The reference compiles gfxlab/gpu/GpuKernelSources.java's PATH_TRACER string with NVRTC
// and launches renderKernel / traceReplayKernel through JCuda (gfxlab/gpu/GpuRayTracer.java).
// build_oracle.py extracts that string verbatim into oracle/_ref/ref_kernel.cu (git-ignored)
// and compiles this file against it with nvcc for sm_100a.  The launch plans restate
// GpuRayTracer's:
//   renderSample        GpuRayTracer.java:317-432  (16x16 blocks, one launch per
//                       (sample, tile), tiles of <= 262,144 pixels from
//                       GpuLaunchProvenance.renderTileLayout, GpuLaunchProvenance.java:44-60)
//   renderKernel params GpuRayTracer.java:478-538
//   traceReplay         GpuRayTracer.java:615-716  (1-D launches of 256 threads,
//                       <= 262,144 rays per launch)
// Only tests/ and bench.py (as a comparison arm) load the resulting library.
#include "ref_kernel.cu"

#include <cuda_runtime.h>
#include <stdint.h>

namespace {

struct DevScene {
  float *spheres = nullptr, *boxes = nullptr, *planes = nullptr, *aspheres = nullptr,
        *aboxes = nullptr, *materials = nullptr, *node_bounds = nullptr;
  int *node_data = nullptr, *refs = nullptr, *roots = nullptr;
  int counts[6] = {0, 0, 0, 0, 0, 0};
  int node_count = 0, ref_count = 0, root_count = 0, use_bvh = 0;
};

int upload(const float* h, size_t n, float** d) {
  size_t bytes = (n > 0 ? n : 1) * sizeof(float);
  if (cudaMalloc((void**)d, bytes) != cudaSuccess) return -1;
  if (n > 0 && cudaMemcpy(*d, h, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  return 0;
}
int upload_i(const int* h, size_t n, int** d) {
  size_t bytes = (n > 0 ? n : 1) * sizeof(int);
  if (cudaMalloc((void**)d, bytes) != cudaSuccess) return -1;
  if (n > 0 && cudaMemcpy(*d, h, n * sizeof(int), cudaMemcpyHostToDevice) != cudaSuccess) return -1;
  return 0;
}

const int kFloatsPer[6] = {5, 7, 26, 22, 22, 13};

int make_scene(DevScene* s, const float* const* arrays, const int* counts, const int* bvh_ints,
               const float* node_bounds, const int* node_data, const int* refs, const int* roots) {
  float** dst[6] = {&s->spheres, &s->boxes, &s->planes, &s->aspheres, &s->aboxes, &s->materials};
  for (int k = 0; k < 6; ++k) {
    s->counts[k] = counts[k];
    if (upload(arrays[k], (size_t)counts[k] * kFloatsPer[k], dst[k])) return -1;
  }
  s->use_bvh = bvh_ints[3];
  s->node_count = s->use_bvh ? bvh_ints[0] : 0;
  s->ref_count = s->use_bvh ? bvh_ints[1] : 0;
  s->root_count = s->use_bvh ? bvh_ints[2] : 0;
  if (upload(node_bounds, (size_t)s->node_count * 6, &s->node_bounds)) return -1;
  if (upload_i(node_data, (size_t)s->node_count * 4, &s->node_data)) return -1;
  if (upload_i(refs, (size_t)s->ref_count, &s->refs)) return -1;
  if (upload_i(roots, (size_t)s->root_count, &s->roots)) return -1;
  return 0;
}

void free_scene(DevScene* s) {
  cudaFree(s->spheres);
  cudaFree(s->boxes);
  cudaFree(s->planes);
  cudaFree(s->aspheres);
  cudaFree(s->aboxes);
  cudaFree(s->materials);
  cudaFree(s->node_bounds);
  cudaFree(s->node_data);
  cudaFree(s->refs);
  cudaFree(s->roots);
}

// GpuLaunchProvenance.renderTileLayout (GpuLaunchProvenance.java:44-60).
void tile_layout(int width, int height, int pixels_per_launch, int* tw, int* th, int* cols,
                 int* rows) {
  *tw = width < pixels_per_launch ? width : pixels_per_launch;
  int q = pixels_per_launch / *tw;
  if (q < 1) q = 1;
  *th = height < q ? height : q;
  *cols = 1 + (width - 1) / *tw;
  *rows = 1 + (height - 1) / *th;
}

}  // namespace

extern "C" {

// Closest-hit replay through traceReplayKernel.  Layouts as in the oracle's orc_trace.
int ref_trace(const float* const* arrays, const int* counts, const int* bvh_ints,
              const float* node_bounds, const int* node_data, const int* refs, const int* roots,
              const float* rays, int n, int* hit_flags, float* hit_t, int* hit_order,
              int* hit_material, float* hit_normal, unsigned long long* stats) {
  DevScene s;
  int rc = make_scene(&s, arrays, counts, bvh_ints, node_bounds, node_data, refs, roots);
  float *d_rays = nullptr, *d_t = nullptr, *d_n = nullptr;
  int *d_f = nullptr, *d_o = nullptr, *d_m = nullptr;
  unsigned long long* d_stats = nullptr;
  if (!rc) rc = upload(rays, (size_t)n * 6, &d_rays);
  if (!rc && cudaMalloc(&d_t, (size_t)n * 4) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_n, (size_t)n * 12) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_f, (size_t)n * 4) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_o, (size_t)n * 4) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_m, (size_t)n * 4) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_stats, 14 * 8) != cudaSuccess) rc = -1;
  if (!rc) cudaMemset(d_stats, 0, 14 * 8);
  const int per_launch = 262144;
  for (int off = 0; !rc && off < n; off += per_launch) {
    int cnt = n - off < per_launch ? n - off : per_launch;
    int grid = (cnt + 255) / 256;
    traceReplayKernel<<<grid, 256>>>(
        d_rays + (size_t)off * 6, cnt, s.spheres, s.counts[0], s.boxes, s.counts[1], s.planes,
        s.counts[2], s.aspheres, s.counts[3], s.aboxes, s.counts[4], s.node_bounds, s.node_count,
        s.node_data, s.refs, s.ref_count, s.roots, s.root_count, s.use_bvh, s.materials,
        d_f + off, d_t + off, d_o + off, d_m + off, d_n + (size_t)off * 3, stats ? 1 : 0,
        d_stats);
    if (cudaGetLastError() != cudaSuccess) rc = -2;
  }
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = -3;
  if (!rc) {
    cudaMemcpy(hit_flags, d_f, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hit_t, d_t, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hit_order, d_o, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hit_material, d_m, (size_t)n * 4, cudaMemcpyDeviceToHost);
    cudaMemcpy(hit_normal, d_n, (size_t)n * 12, cudaMemcpyDeviceToHost);
    if (stats) cudaMemcpy(stats, d_stats, 14 * 8, cudaMemcpyDeviceToHost);
  }
  cudaFree(d_rays);
  cudaFree(d_t);
  cudaFree(d_n);
  cudaFree(d_f);
  cudaFree(d_o);
  cudaFree(d_m);
  cudaFree(d_stats);
  free_scene(&s);
  return rc;
}

// One logical frame through renderKernel with renderSample's launch plan, repeated
// `frames` times after `warmup` untimed frames; returns the CUDA-event time of the
// timed frames (ms, summed) in *kernel_ms and the last frame's image in rgb (3 floats
// per pixel, may be null).  camera: pos, forward, right, up; params: width, height,
// spp, max_depth, frame_index.
// With flush_bytes > 0 each timed frame has its own event pair, and a buffer of that many
// bytes is written before it, outside the events (an L2 flush, as the library's bench does).
static int render_frames(const float* const* arrays, const int* counts, const int* bvh_ints,
                         const float* node_bounds, const int* node_data, const int* refs,
                         const int* roots, const float* camera, const float* background,
                         const int* params, unsigned long long frame_seed, int warmup, int frames,
                         float* rgb, double* kernel_ms, unsigned long long* stats,
                         size_t flush_bytes = 0) {
  DevScene s;
  int rc = make_scene(&s, arrays, counts, bvh_ints, node_bounds, node_data, refs, roots);
  int width = params[0], height = params[1], spp = params[2], max_depth = params[3];
  int frame_index = params[4];
  float* d_out = nullptr;
  unsigned long long* d_stats = nullptr;
  if (!rc && cudaMalloc(&d_out, (size_t)width * height * 12) != cudaSuccess) rc = -1;
  if (!rc && cudaMalloc(&d_stats, 14 * 8) != cudaSuccess) rc = -1;
  if (!rc) cudaMemset(d_stats, 0, 14 * 8);
  int tw, th, cols, rows;
  tile_layout(width, height, 262144, &tw, &th, &cols, &rows);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  double total = 0.0;
  void* d_flush = nullptr;
  if (!rc && flush_bytes > 0 && cudaMalloc(&d_flush, flush_bytes) != cudaSuccess) rc = -1;
  for (int f = 0; !rc && f < warmup + frames; ++f) {
    if (d_flush && f >= warmup) {
      cudaMemsetAsync(d_flush, f & 0xFF, flush_bytes);
      cudaEventRecord(e0);
    } else if (f == warmup) {
      cudaEventRecord(e0);
    }
    for (int so = 0; so < spp; ++so) {
      for (int t = 0; t < cols * rows; ++t) {
        int c = t % cols, r = t / cols;
        int x = c * tw, y = r * th;
        int w = tw < width - x ? tw : width - x;
        int h = th < height - y ? th : height - y;
        dim3 grid((w + 15) / 16, (h + 15) / 16);
        renderKernel<<<grid, dim3(16, 16)>>>(
            d_out, width, height, x, y, w, h, camera[0], camera[1], camera[2], camera[3],
            camera[4], camera[5], camera[6], camera[7], camera[8], camera[9], camera[10],
            camera[11], s.spheres, s.counts[0], s.boxes, s.counts[1], s.planes, s.counts[2],
            s.aspheres, s.counts[3], s.aboxes, s.counts[4], s.node_bounds, s.node_count,
            s.node_data, s.refs, s.ref_count, s.roots, s.root_count, s.use_bvh, s.materials,
            s.counts[5], background[0], background[1], background[2], max_depth, frame_index,
            frame_seed, so, spp, d_stats, stats ? 1 : 0);
      }
    }
    if (cudaGetLastError() != cudaSuccess) rc = -2;
    if (!rc && d_flush && f >= warmup) {
      cudaEventRecord(e1);
      cudaEventSynchronize(e1);
      float ms = 0.0f;
      cudaEventElapsedTime(&ms, e0, e1);
      total += ms;
    }
  }
  if (!rc && frames > 0 && !d_flush) {
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    total = ms;
  }
  if (!rc && cudaDeviceSynchronize() != cudaSuccess) rc = -3;
  if (!rc && rgb) cudaMemcpy(rgb, d_out, (size_t)width * height * 12, cudaMemcpyDeviceToHost);
  if (!rc && stats) cudaMemcpy(stats, d_stats, 14 * 8, cudaMemcpyDeviceToHost);
  if (kernel_ms) *kernel_ms = total;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d_flush);
  cudaFree(d_out);
  cudaFree(d_stats);
  free_scene(&s);
  return rc;
}

int ref_render(const float* const* arrays, const int* counts, const int* bvh_ints,
               const float* node_bounds, const int* node_data, const int* refs, const int* roots,
               const float* camera, const float* background, const int* params,
               unsigned long long frame_seed, int warmup, int frames, float* rgb,
               double* kernel_ms) {
  return render_frames(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots, camera,
                       background, params, frame_seed, warmup, frames, rgb, kernel_ms, nullptr);
}

// As ref_render, with each timed frame timed on its own and an L2 flush of flush_bytes
// written before it outside the events; *kernel_ms is the sum over the timed frames.
int ref_render_flushed(const float* const* arrays, const int* counts, const int* bvh_ints,
                       const float* node_bounds, const int* node_data, const int* refs,
                       const int* roots, const float* camera, const float* background,
                       const int* params, unsigned long long frame_seed, int warmup, int frames,
                       unsigned long long flush_bytes, float* rgb, double* kernel_ms) {
  return render_frames(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots, camera,
                       background, params, frame_seed, warmup, frames, rgb, kernel_ms, nullptr,
                       (size_t)flush_bytes);
}

// One frame with the kernel's metrics enabled (a build with GFXLAB_RENDER_METRICS): the 14
// frame counters (K:30-43) summed over the frame's launches.
int ref_render_stats(const float* const* arrays, const int* counts, const int* bvh_ints,
                     const float* node_bounds, const int* node_data, const int* refs,
                     const int* roots, const float* camera, const float* background,
                     const int* params, unsigned long long frame_seed, float* rgb,
                     unsigned long long* stats) {
  return render_frames(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots, camera,
                       background, params, frame_seed, 0, 1, rgb, nullptr, stats);
}

}  // extern "C"
