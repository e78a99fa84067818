// Batched rendering: many resident scenes, each with its own camera, resolution, sample count
// and depth, rendered by ONE persistent launch over a shared pixel queue and replayed from a
// captured CUDA graph.
//
// The per-scene form launches one frame per scene; small frames (256x256 = 65,536 pixels)
// cannot fill 148 SMs and every launch ends in its own tail.  Here the pixels of all jobs form
// one index space: a lane that finishes a pixel takes the next index of the batch queue, which
// may belong to another scene, so the GPU stays full until the whole batch's last pixels.
// Each pixel still runs its samples in order with the reference's random streams and FP32
// running sum (GpuKernelSources.java:1231-1293, tracePath K:1061-1165), so every job's image
// is bit-identical to its per-scene frame.
//
// The batch's last pixels (about two per resident thread) are queued one sample per item,
// as in the per-scene frame: their radiance goes to the batch's sample buffer and
// k_sum_batch_tail adds each pixel's samples in sample order, so images stay bit-identical.
//
// Frames mode: with the scene read from a job table instead of kernel parameters, the shared
// queue costs every sample a little; the alternative is each job's own persistent frame
// (k_render with its single-sample tail), the frames spread over concurrent branches of the
// same graph so that one frame's last blocks overlap the next frame's first.  Each frame has
// its own queue head and sample buffer, so its image is exactly its per-scene frame's.
//
// Launch parameters (mode, threads per block, job order, branches) come from
// rtb_batch_autotune, which times the candidates on the batch itself.
#include <algorithm>
#include <numeric>
#include <vector>

#include "rtb_internal.h"

struct rtb_batch {
  std::vector<rtb_batch_job> jobs;  // in the caller's order
  void* d_jobs = nullptr;           // device job table (in the tuned order)
  long long total_pixels = 0;
  long long total_items = 0;        // whole pixels + single samples of the queue
  int tail_pixels = 0;              // pixels rendered one sample per item, over all jobs
  float* d_tail = nullptr;          // their samples' RGB
  size_t tail_bytes = 0;
  rtb_batch_tuning tuning{};
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int device = 0;
  // frames mode
  std::vector<rtb::FramePlan*> frames;   // in the tuned order
  unsigned long long* d_queues = nullptr;  // one queue head per frame
  size_t queue_count = 0;
  float* d_frame_tails = nullptr;          // one sample buffer per branch
  size_t frame_tail_bytes = 0;
  cudaStream_t branch[4] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[4] = {nullptr, nullptr, nullptr, nullptr};
};

namespace rtb {
namespace {

constexpr int kMaxSharedJobs = 256;

struct BatchJob {
  DevScene S;
  float3 cam_pos, cam_f, cam_r, cam_u;
  int width, height, spp, max_depth, frame_index;
  unsigned long long frame_seed;
  float* out;
  long long begin;  // first queue item of this job
  long long split;  // pixels [split, width*height) are queued one sample per item
  long long tail_off;  // first sample-buffer slot of the job's single-sample items
  int tail_begin;      // first tail pixel (over all jobs) of this job
};

// At most 16M single-sample items (192 MB of radiance) per batch.
constexpr long long kMaxBatchTailItems = 1LL << 24;

__device__ __forceinline__ float luminance(float3 c) {  // K:181-183
  return c.x * 0.212655f + c.y * 0.715158f + c.z * 0.072187f;
}
__device__ __forceinline__ float3 reflect_dir(float3 n, float3 i) {  // K:1022-1024
  return sub(mul(n, 2.0f * dot(i, n)), i);
}
static __device__ __noinline__ float3 refract_dir(float3 incoming, float3 n, float eta) {  // K:1026-1039
  float3 i = normalize_safe(incoming);
  float c1 = dot(i, n);
  float ri = (c1 >= 0.0f) ? eta : -1.0f / eta;
  float inv_ri2 = 1.0f / (ri * ri);
  float c2 = 1.0f - (1.0f - c1 * c1) * inv_ri2;
  if (c2 <= 0.0f) return normalize_safe(reflect_dir(n, i));
  float sq = sqrtf(c2);
  return normalize_safe(sub(mul(n, c1 - sq * ri), i));
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 1024 / THREADS) k_batch(const BatchJob* jobs, int njobs,
                                                                   long long total, float* tail,
                                                                   unsigned long long* queue,
                                                                   int* abort_flag) {
  __shared__ long long s_begin[kMaxSharedJobs];
  const int nshared = njobs < kMaxSharedJobs ? njobs : kMaxSharedJobs;
  for (int j = threadIdx.x; j < nshared; j += THREADS) s_begin[j] = jobs[j].begin;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  int job = 0;
  long long pixel = -1;
  int x = 0, y = 0, so = 0;
  long long titem = -1;  // sample-buffer slot of a single-sample lane, -1 for a whole pixel
  uint32_t base_seed = 0, rng = 0;
  float3 acc = v3(0, 0, 0), thr = v3(0, 0, 0), rad = v3(0, 0, 0), o = v3(0, 0, 0), d = v3(0, 0, 0);
  int depth = 0;
  bool path = false, done = false;
  while (true) {
    // ---- fetch a batch pixel (warp-aggregated) and find its job
    bool need = !done && pixel < 0;
    unsigned need_mask = __ballot_sync(0xFFFFFFFFu, need);
    if (need_mask) {
      unsigned long long basep = 0;
      int leader = __ffs(need_mask) - 1;
      if (lane == leader)
        basep = abort_raised(abort_flag) ? (unsigned long long)total
                                         : atomicAdd(queue, (unsigned long long)__popc(need_mask));
      basep = __shfl_sync(0xFFFFFFFFu, basep, leader);
      if (need) {
        long long g = (long long)basep + __popc(need_mask & ((1u << lane) - 1u));
        if (g >= total) {
          done = true;
        } else {
          int lo = 0, hi = njobs - 1;  // last job with begin <= g
          while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            long long b = mid < kMaxSharedJobs ? s_begin[mid] : jobs[mid].begin;
            if (b <= g) lo = mid; else hi = mid - 1;
          }
          job = lo;
          const BatchJob& J = jobs[job];
          pixel = g - J.begin;
          if (pixel < J.split) {
            so = 0;
            titem = -1;
          } else {
            unsigned t = (unsigned)(pixel - J.split);
            so = (int)(t % (unsigned)J.spp);
            pixel = J.split + (long long)(t / (unsigned)J.spp);
            titem = J.tail_off + t;
          }
          x = (int)(pixel % J.width);
          y = (int)(pixel / J.width);
          uint32_t s = hash_u32((uint32_t)(J.frame_seed & 0xFFFFFFFFULL));  // K:1231-1236
          s ^= hash_u32((uint32_t)(J.frame_seed >> 32));
          s ^= hash_u32((uint32_t)J.frame_index);
          s ^= hash_u32((uint32_t)y * (uint32_t)J.width + (uint32_t)x);
          base_seed = hash_u32(s);
        }
      }
    }
    if (__all_sync(0xFFFFFFFFu, done)) break;
    const BatchJob& J = jobs[job];
    // ---- start a sample (K:1251-1264)
    if (!done && !path) {
      uint32_t seed = base_seed ^ hash_u32((uint32_t)so);
      seed ^= hash_u32((uint32_t)(so * 0x9E3779B9u));
      rng = hash_u32(seed);
      float jx = rand01(&rng) - 0.5f;
      float jy = rand01(&rng) - 0.5f;
      float aspect = (float)J.width / (float)J.height;
      float u = ((((float)x + 0.5f) + jx) * (2.0f / (float)J.width) - 1.0f) * aspect;
      float v = 1.0f - ((((float)y + 0.5f) + jy) * (2.0f / (float)J.height));
      o = J.cam_pos;
      d = add(add(J.cam_f, mul(J.cam_r, u)), mul(J.cam_u, v));
      thr = v3(1.0f, 1.0f, 1.0f);
      rad = v3(0.0f, 0.0f, 0.0f);
      depth = 0;
      path = J.max_depth > 0;
    }
    // ---- one path segment (K:1098-1162)
    bool finished = !done && !path;
    bool tracing = !done && path;
    Best b;
    bool hit = trace_closest<false>(J.S, o, d, tracing, b, nullptr, nullptr);
    if (tracing) {
      if (!hit) {
        rad = add(rad, mulv(thr, J.S.background));
        finished = true;
      } else {
        float3 pos, n;
        int mi;
        hit_record(J.S, b, o, d, &pos, &n, &mi);
        float4 m0 = make_float4(0, 0, 0, 0), m1 = m0, m2 = m0, m3 = m0;
        if (mi >= 0) {
          const float4* mp = J.S.materials + 4 * mi;
          m0 = __ldg(mp);
          m1 = __ldg(mp + 1);
          m2 = __ldg(mp + 2);
          m3 = __ldg(mp + 3);
        }
        float3 cd = v3(m0.x, m0.y, m0.z), cr = v3(m1.x, m1.y, m1.z), ct = v3(m2.x, m2.y, m2.z);
        rad = add(rad, mulv(thr, v3(m3.x, m3.y, m3.z)));
        float3 inc = neg(d);
        float wd = luminance(cd), wr = luminance(cr), wt = luminance(ct);
        float sum = wd + wr + wt;
        if (sum <= 0.0f) {
          finished = true;
        } else {
          float xi = rand01(&rng) * sum;
          float3 nd, wc;
          if (xi < wd) {
            float pc = wd / sum;
            float z = rand01(&rng) * 2.0f - 1.0f;
            float t = rand01(&rng) * 2.0f * CUDART_PI_F;
            float r = sqrtf(fmaxf(0.0f, 1.0f - z * z));
            nd = add(v3(r * cosf(t), r * sinf(t), z), n);
            wc = divs(cd, pc);
          } else if (xi < wd + wr) {
            float pc = wr / sum;
            nd = reflect_dir(n, inc);
            wc = divs(cr, pc);
          } else {
            float pc = wt / sum;
            nd = refract_dir(inc, n, m0.w);
            wc = divs(ct, pc);
          }
          o = add(pos, mul(nd, kEps));
          thr = mulv(thr, wc);
          d = nd;
          depth++;
          if (depth >= J.max_depth) finished = true;
        }
      }
    }
    if (finished && titem >= 0) {
      path = false;
      float* t = tail + 3 * titem;
      t[0] = rad.x;
      t[1] = rad.y;
      t[2] = rad.z;
      pixel = -1;
    } else if (finished) {
      path = false;
      acc = so == 0 ? rad : add(acc, rad);
      so++;
      if (so == J.spp) {
        acc = mul(acc, 1.0f / (float)J.spp);
        float* out = J.out + 3 * pixel;
        out[0] = acc.x;
        out[1] = acc.y;
        out[2] = acc.z;
        pixel = -1;
      }
    }
  }
}

// One thread per tail pixel of the batch: the in-order FP32 sum of its samples, scaled as in
// k_batch.  A batch whose kernel stopped on an abort leaves its tail pixels unwritten.
__global__ void __launch_bounds__(256) k_sum_batch_tail(const BatchJob* jobs, int njobs,
                                                        const float* __restrict__ tail,
                                                        int tail_pixels, const int* abort_flag) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= tail_pixels || abort_stopped(abort_flag)) return;
  int lo = 0, hi = njobs - 1;  // last job with tail_begin <= q
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].tail_begin <= q) lo = mid; else hi = mid - 1;
  }
  const BatchJob& J = jobs[lo];
  long long k = q - J.tail_begin;  // tail pixel within the job
  const float* s = tail + 3 * (J.tail_off + k * J.spp);
  float3 acc = v3(s[0], s[1], s[2]);
  for (int i = 1; i < J.spp; i++) acc = add(acc, v3(s[3 * i], s[3 * i + 1], s[3 * i + 2]));
  acc = mul(acc, 1.0f / (float)J.spp);
  float* o = J.out + 3 * (J.split + k);
  o[0] = acc.x;
  o[1] = acc.y;
  o[2] = acc.z;
}

int blocks_per_sm(int threads) {
  int bps = 1;
  const void* fn = threads == 64 ? (const void*)k_batch<64>
                 : threads == 256 ? (const void*)k_batch<256> : (const void*)k_batch<128>;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, fn, threads, 0);
  return bps < 1 ? 1 : bps;
}

int launch_grid(rtb_context* ctx, int threads, long long total) {
  long long want = (total + threads - 1) / threads;
  return (int)std::max<long long>(
      1, std::min<long long>((long long)ctx->sm_count * blocks_per_sm(threads), want));
}

constexpr int kMaxBranches = 4;

// Frames mode: every job's frame, round-robin over the branches, forked from and joined back
// into `sm` (inside a capture this builds the graph's parallel branches).
rtb_status enqueue_frames(rtb_context* ctx, rtb_batch* B, cudaStream_t sm) {
  int n = (int)B->frames.size();
  int K = std::min(B->tuning.branches, n);
  cudaMemsetAsync(B->d_queues, 0, sizeof(unsigned long long) * n, sm);
  if (K <= 1) {
    for (FramePlan* f : B->frames) launch_frame(f, sm);
  } else {
    cudaEventRecord(B->fork, sm);
    for (int b = 0; b < K; ++b) cudaStreamWaitEvent(B->branch[b], B->fork, 0);
    for (int i = 0; i < n; ++i) launch_frame(B->frames[i], B->branch[i % K]);
    for (int b = 0; b < K; ++b) {
      cudaEventRecord(B->join[b], B->branch[b]);
      cudaStreamWaitEvent(sm, B->join[b], 0);
    }
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? RTB_OK : cuda_fail(ctx, e, "batch frame launches");
}

rtb_status enqueue(rtb_context* ctx, rtb_batch* B, cudaStream_t sm) {
  if (B->tuning.branches > 0) return enqueue_frames(ctx, B, sm);
  int threads = B->tuning.threads_per_block;
  int grid = launch_grid(ctx, threads, B->total_items);
  cudaMemsetAsync(ctx->d_work, 0, sizeof(unsigned long long), sm);
  const BatchJob* J = (const BatchJob*)B->d_jobs;
  int n = (int)B->jobs.size();
  long long total = B->total_items;
  if (threads == 64)
    k_batch<64><<<grid, 64, 0, sm>>>(J, n, total, B->d_tail, ctx->d_work, ctx->d_abort);
  else if (threads == 256)
    k_batch<256><<<grid, 256, 0, sm>>>(J, n, total, B->d_tail, ctx->d_work, ctx->d_abort);
  else
    k_batch<128><<<grid, 128, 0, sm>>>(J, n, total, B->d_tail, ctx->d_work, ctx->d_abort);
  if (B->tail_pixels > 0)
    k_sum_batch_tail<<<(B->tail_pixels + 255) / 256, 256, 0, sm>>>(J, n, B->d_tail, B->tail_pixels,
                                                                     ctx->d_abort);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? RTB_OK : cuda_fail(ctx, e, "batch launch");
}

void free_frames(rtb_batch* B) {
  for (FramePlan* f : B->frames) delete_frame_plan(f);
  B->frames.clear();
}

// Frames mode: one planned frame per job in `order`, its queue head, and one sample buffer
// per branch sized for the largest tail among that branch's frames.
rtb_status plan_frames(rtb_context* ctx, rtb_batch* B, const std::vector<int>& order) {
  free_frames(B);
  int n = (int)order.size();
  int K = std::max(1, std::min(B->tuning.branches, n));
  std::vector<size_t> branch_bytes(K, 0);
  for (int i = 0; i < n; ++i) {
    const rtb_batch_job& j = B->jobs[order[i]];
    rtb_render_params p = j.params;
    p.collect_metrics = 0;
    if (B->tuning.shared_stack_entries != 0) p.shared_stack_entries = B->tuning.shared_stack_entries;
    FramePlan* f = new_frame_plan();
    rtb_status s = plan_frame(ctx, j.scene, &j.camera, &p, j.rgb_device, f, 0, 1,
                              B->tuning.tail_pixels_per_thread);
    if (s != RTB_OK) {
      delete_frame_plan(f);
      free_frames(B);
      return s;
    }
    B->frames.push_back(f);
    branch_bytes[i % K] = std::max(branch_bytes[i % K], rtb::frame_tail_bytes(f));
  }
  std::vector<size_t> off(K, 0);
  size_t total = 0;
  for (int b = 0; b < K; ++b) {
    off[b] = total;
    total += (branch_bytes[b] + 255) & ~(size_t)255;
  }
  if (total > B->frame_tail_bytes) {
    cudaFree(B->d_frame_tails);
    B->d_frame_tails = nullptr;
    B->frame_tail_bytes = 0;
    cudaError_t e = cudaMalloc(&B->d_frame_tails, total);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch frame sample buffers");
    B->frame_tail_bytes = total;
  }
  if ((size_t)n > B->queue_count) {
    cudaFree(B->d_queues);
    B->d_queues = nullptr;
    B->queue_count = 0;
    cudaError_t e = cudaMalloc(&B->d_queues, sizeof(unsigned long long) * n);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch frame queues");
    B->queue_count = n;
  }
  for (int i = 0; i < n; ++i) {
    float* tail = branch_bytes[i % K] ? (float*)((char*)B->d_frame_tails + off[i % K]) : nullptr;
    bind_frame(B->frames[i], B->d_queues + i, tail, ctx->d_abort, ctx->d_work + 8);
  }
  return RTB_OK;
}

// Job table in the tuned order: order 0 keeps the caller's order, order 1 puts the most
// expensive jobs (pixels x spp x depth) first so the batch does not end on a large frame.
rtb_status upload_jobs(rtb_context* ctx, rtb_batch* B) {
  std::vector<int> order(B->jobs.size());
  std::iota(order.begin(), order.end(), 0);
  if (B->tuning.job_order == 1) {
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
      const rtb_render_params& pa = B->jobs[a].params;
      const rtb_render_params& pb = B->jobs[b].params;
      double ca = (double)pa.width * pa.height * pa.samples_per_frame * std::max(1, pa.max_depth);
      double cb = (double)pb.width * pb.height * pb.samples_per_frame * std::max(1, pb.max_depth);
      return ca > cb;
    });
  }
  // Job tables and sample buffers change only while no batch kernel runs.
  cudaDeviceSynchronize();
  if (B->tuning.branches > 0) return plan_frames(ctx, B, order);
  // Tail: the last jobs' last pixels, about two per resident thread, as single samples.
  std::vector<long long> tail(order.size(), 0);
  {
    long long per_thread = B->tuning.tail_pixels_per_thread > 0 ? B->tuning.tail_pixels_per_thread : 2;
    long long want = per_thread * ctx->sm_count * blocks_per_sm(B->tuning.threads_per_block) *
                     B->tuning.threads_per_block;
    long long items_left = kMaxBatchTailItems;
    for (size_t k = order.size(); k-- > 0 && want > 0;) {
      const rtb_render_params& p = B->jobs[order[k]].params;
      long long px = (long long)p.width * p.height;
      long long tp = std::min(std::min(px, want), items_left / p.samples_per_frame);
      if (tp <= 0) break;
      tail[k] = tp;
      want -= tp;
      items_left -= tp * p.samples_per_frame;
      if (tp < px) break;
    }
  }
  long long tail_items = 0, tail_pixels = 0;
  for (size_t k = 0; k < order.size(); ++k)
    tail_items += tail[k] * B->jobs[order[k]].params.samples_per_frame;
  for (long long t : tail) tail_pixels += t;
  size_t tail_bytes = (size_t)tail_items * 3 * sizeof(float);
  if (tail_bytes > B->tail_bytes) {
    cudaFree(B->d_tail);
    B->d_tail = nullptr;
    B->tail_bytes = 0;
    cudaError_t e = cudaMalloc(&B->d_tail, tail_bytes);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch sample buffer");
    B->tail_bytes = tail_bytes;
  }
  std::vector<BatchJob> h(order.size());
  long long begin = 0, tail_off = 0;
  int tail_begin = 0;
  for (size_t k = 0; k < order.size(); ++k) {
    const rtb_batch_job& j = B->jobs[order[k]];
    BatchJob& b = h[k];
    b.S = j.scene->dev;
    b.S.use_bvh = (j.params.use_bvh && j.scene->has_bvh) ? 1 : 0;
    b.cam_pos = make_float3(j.camera.position[0], j.camera.position[1], j.camera.position[2]);
    b.cam_f = make_float3(j.camera.forward[0], j.camera.forward[1], j.camera.forward[2]);
    b.cam_r = make_float3(j.camera.right[0], j.camera.right[1], j.camera.right[2]);
    b.cam_u = make_float3(j.camera.up[0], j.camera.up[1], j.camera.up[2]);
    b.width = j.params.width;
    b.height = j.params.height;
    b.spp = j.params.samples_per_frame;
    b.max_depth = j.params.max_depth;
    b.frame_index = j.params.frame_index;
    b.frame_seed = j.params.frame_seed;
    b.out = j.rgb_device;
    b.begin = begin;
    long long px = (long long)j.params.width * j.params.height;
    b.split = px - tail[k];
    b.tail_off = tail_off;
    b.tail_begin = tail_begin;
    begin += b.split + tail[k] * b.spp;
    tail_off += tail[k] * b.spp;
    tail_begin += (int)tail[k];
  }
  if (!B->d_jobs) {
    cudaError_t e = cudaMalloc(&B->d_jobs, sizeof(BatchJob) * h.size());
    if (e != cudaSuccess) return cuda_fail(ctx, e, "batch job table");
  }
  cudaError_t e = cudaMemcpy(B->d_jobs, h.data(), sizeof(BatchJob) * h.size(), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch job table upload");
  B->total_items = begin;
  B->tail_pixels = (int)tail_pixels;
  B->total_pixels = 0;
  for (const rtb_batch_job& j : B->jobs) B->total_pixels += (long long)j.params.width * j.params.height;
  return RTB_OK;
}

void release_batch(rtb_batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  free_frames(B);
  cudaFree(B->d_jobs);
  cudaFree(B->d_tail);
  cudaFree(B->d_queues);
  cudaFree(B->d_frame_tails);
  for (int b = 0; b < kMaxBranches; ++b) {
    if (B->branch[b]) cudaStreamDestroy(B->branch[b]);
    if (B->join[b]) cudaEventDestroy(B->join[b]);
  }
  if (B->fork) cudaEventDestroy(B->fork);
  delete B;
}

rtb_status capture(rtb_context* ctx, rtb_batch* B) {
  if (B->exec) cudaGraphExecDestroy(B->exec);
  if (B->graph) cudaGraphDestroy(B->graph);
  B->exec = nullptr;
  B->graph = nullptr;
  cudaStream_t sm = ctx->stream;
  cudaError_t e = cudaStreamBeginCapture(sm, cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture");
  rtb_status s = enqueue(ctx, B, sm);
  e = cudaStreamEndCapture(sm, &B->graph);
  if (s != RTB_OK) return s;
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph capture");
  e = cudaGraphInstantiate(&B->exec, B->graph, 0);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph instantiate");
  return RTB_OK;
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

rtb_status rtb_batch_create(rtb_context* ctx, const rtb_batch_job* jobs, int job_count,
                            const rtb_batch_tuning* tuning, rtb_batch** out) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  if (!jobs || job_count < 1 || !out) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "a batch needs jobs");
  for (int k = 0; k < job_count; ++k) {
    const rtb_batch_job& j = jobs[k];
    const rtb_render_params& p = j.params;
    if (!j.scene || !j.rgb_device || p.width < 1 || p.height < 1 || p.samples_per_frame < 1 ||
        p.max_depth < 0 || p.max_depth > 32)
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "invalid batch job " + std::to_string(k));
    if (j.scene->device != ctx->device)
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "batch job scene is on another device");
  }
  rtb_batch* B = new rtb_batch();
  B->device = ctx->device;
  B->jobs.assign(jobs, jobs + job_count);
  B->tuning.threads_per_block = 128;
  B->tuning.job_order = 1;
  B->tuning.branches = 4;
  if (tuning) B->tuning = *tuning;
  if (B->tuning.threads_per_block != 64 && B->tuning.threads_per_block != 128 &&
      B->tuning.threads_per_block != 256) {
    delete B;
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "threads_per_block must be 64, 128 or 256");
  }
  if (B->tuning.branches < 0 || B->tuning.branches > kMaxBranches) {
    delete B;
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "branches must be in [0, 4]");
  }
  int se = B->tuning.shared_stack_entries;
  if ((se != 0 && se != -1 && se != 8 && se != 16) || B->tuning.tail_pixels_per_thread < 0 ||
      B->tuning.tail_pixels_per_thread > 16) {
    delete B;
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT,
                "shared_stack_entries must be 0, -1, 8 or 16 and tail_pixels_per_thread in [0, 16]");
  }
  cudaError_t e = cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming);
  for (int b = 0; b < kMaxBranches && e == cudaSuccess; ++b) {
    e = cudaStreamCreateWithFlags(&B->branch[b], cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&B->join[b], cudaEventDisableTiming);
  }
  if (e != cudaSuccess) {
    release_batch(B);
    return cuda_fail(ctx, e, "batch streams");
  }
  rtb_status s = upload_jobs(ctx, B);
  if (s == RTB_OK) s = capture(ctx, B);
  if (s != RTB_OK) {
    release_batch(B);
    return s;
  }
  *out = B;
  return RTB_OK;
}

rtb_status rtb_batch_render(rtb_context* ctx, rtb_batch* B, void* stream) {
  if (!ctx || !B) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaStream_t sm = stream ? (cudaStream_t)stream : ctx->stream;
  ctx_acquire(ctx, sm);
  arm_abort(ctx, sm);  // outside the graph: its kernels read the words, never write [1]
  cudaError_t e = cudaGraphLaunch(B->exec, sm);
  ctx_release(ctx, sm);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "batch graph launch");
  return RTB_OK;
}

rtb_status rtb_batch_autotune(rtb_context* ctx, rtb_batch* B, int repeats, rtb_batch_tuning* best,
                              double* best_ms) {
  if (!ctx || !B) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  if (repeats < 1) repeats = 1;
  double best_time = 1e300;
  rtb_batch_tuning pick = B->tuning;
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  rtb_status s = RTB_OK;
  auto try_all = [&](const std::vector<rtb_batch_tuning>& cands) {
    for (const rtb_batch_tuning& c : cands) {
      B->tuning = c;
      s = upload_jobs(ctx, B);
      if (s != RTB_OK) return;
      double total = 0.0;
      for (int r = 0; r <= repeats && s == RTB_OK; ++r) {  // first run warms up
        arm_abort(ctx, sm);
        cudaEventRecord(ctx->ev0, sm);
        s = enqueue(ctx, B, sm);
        if (s != RTB_OK) return;
        cudaEventRecord(ctx->ev1, sm);
        cudaError_t e = cudaEventSynchronize(ctx->ev1);
        if (e != cudaSuccess) {
          s = cuda_fail(ctx, e, "batch autotune");
          return;
        }
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
        if (r > 0) total += ms;
      }
      double mean = total / repeats;
      if (mean < best_time) {
        best_time = mean;
        pick = c;
      }
    }
  };
  // Stage 1: the kernel form -- the shared-queue kernel at 64/128/256 threads, or per-job
  // frames over 1/2/4 graph branches -- each in the caller's order and most expensive first.
  std::vector<rtb_batch_tuning> cands;
  for (int order = 0; order < 2; ++order) {
    for (int t : {64, 128, 256}) cands.push_back({t, order, 0, 0, 0});
    for (int k : {1, 2, 4}) cands.push_back({128, order, k, 0, 0});
  }
  try_all(cands);
  // Stage 2: queue granularity at the end of the frames (or of the shared queue).
  if (s == RTB_OK) {
    cands.clear();
    for (int t : {1, 2, 4, 8}) {
      rtb_batch_tuning c = pick;
      c.tail_pixels_per_thread = t;
      cands.push_back(c);
    }
    try_all(cands);
  }
  // Stage 3: for per-job frames, the traversal-stack entries kept in shared memory.
  if (s == RTB_OK && pick.branches > 0) {
    cands.clear();
    for (int e : {-1, 8, 16}) {
      rtb_batch_tuning c = pick;
      c.shared_stack_entries = e;
      cands.push_back(c);
    }
    try_all(cands);
  }
  ctx_release(ctx, sm);
  B->tuning = pick;
  rtb_status s2 = upload_jobs(ctx, B);
  if (s2 == RTB_OK) s2 = capture(ctx, B);
  if (s != RTB_OK) return s;
  if (s2 != RTB_OK) return s2;
  if (best) *best = pick;
  if (best_ms) *best_ms = best_time;
  return RTB_OK;
}

rtb_status rtb_batch_destroy(rtb_context* ctx, rtb_batch* B) {
  if (!ctx || !B) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  cudaDeviceSynchronize();
  release_batch(B);
  return RTB_OK;
}

}  // extern "C"
