// Adjoint of the path tracer with respect to per-material albedo (diffuse colour) and
// emission: path replay.  No counterpart in the reference.
//
// For one sample the kernel's radiance is  L = sum_k thr_k (*) E_k  (+ thr_K (*) background on
// a miss), with thr_{k+1} = thr_k (*) W_k and W_k the lobe weight colour (for the diffuse lobe
// W = albedo / p, p the lobe probability).  Given the image adjoint a = dLoss/dI of the
// pixel, the backward kernel re-traces each sample from its random seed -- the same traversal
// and the same random stream as the forward frame, so the same path -- keeping the vertices
// (material, thr, W, 1/p, lobe) in a per-thread stack, then walks them backward with the
// incoming radiance Li (background or 0 after the last vertex, Li <- E_k + W_k (*) Li):
//     dLoss/dE_k      += (a / spp) (*) thr_k
//     dLoss/dalbedo_k += (a / spp) (*) thr_k (*) Li_after_k / p_k      (diffuse lobe chosen)
// The lobe probability is treated as fixed (the sampling decision is not differentiated); for
// materials with only a diffuse lobe -- the differentiable workload's -- p = 1 and the result
// is the exact derivative of the rendered image.  Emission gradients are exact for all
// materials.  Gradients accumulate in FP32: first in a per-block shared-memory table keyed by
// material (walls and emitters are hit by most paths), then with one global atomic per entry.
#include <algorithm>

#include "rtb_internal.h"

namespace rtb {
namespace {

constexpr int kTable = 512;       // shared-memory gradient entries per block
constexpr int kMaxVertices = 32;  // max_depth limit of the renderer

struct AdjointArgs {
  DevScene S;
  float3 cam_pos, cam_f, cam_r, cam_u;
  int width, height, spp, max_depth, frame_index;
  unsigned long long frame_seed;
  const float* adjoint;  // dLoss/dI, 3 floats per pixel
  float* grad_albedo;    // 3 per material
  float* grad_emission;  // 3 per material
  long long pixels;
  unsigned long long* queue;
  int* abort_flag;  // the context's abort words (abort_raised)
};

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

struct GradTable {
  int key[kTable];
  float val[kTable][6];
};

__device__ __forceinline__ void accumulate(GradTable& T, const AdjointArgs& a, int m, float3 ga,
                                           float3 ge) {
  unsigned h = ((unsigned)m * 2654435761u) & (kTable - 1);
  for (int probe = 0; probe < 8; ++probe) {
    int slot = (h + probe) & (kTable - 1);
    int k = atomicCAS(&T.key[slot], -1, m);
    if (k == -1 || k == m) {
      atomicAdd(&T.val[slot][0], ga.x);
      atomicAdd(&T.val[slot][1], ga.y);
      atomicAdd(&T.val[slot][2], ga.z);
      atomicAdd(&T.val[slot][3], ge.x);
      atomicAdd(&T.val[slot][4], ge.y);
      atomicAdd(&T.val[slot][5], ge.z);
      return;
    }
  }
  atomicAdd(a.grad_albedo + 3 * m, ga.x);
  atomicAdd(a.grad_albedo + 3 * m + 1, ga.y);
  atomicAdd(a.grad_albedo + 3 * m + 2, ga.z);
  atomicAdd(a.grad_emission + 3 * m, ge.x);
  atomicAdd(a.grad_emission + 3 * m + 1, ge.y);
  atomicAdd(a.grad_emission + 3 * m + 2, ge.z);
}

__global__ void __launch_bounds__(128, 6) k_adjoint(AdjointArgs a) {
  __shared__ GradTable T;
  for (int i = threadIdx.x; i < kTable; i += blockDim.x) {
    T.key[i] = -1;
    for (int k = 0; k < 6; ++k) T.val[i][k] = 0.0f;
  }
  __syncthreads();
  const DevScene& S = a.S;
  const int lane = threadIdx.x & 31;
  long long pixel = -1;
  int x = 0, y = 0, so = 0;
  uint32_t base_seed = 0, rng = 0;
  float3 adj = v3(0, 0, 0), thr = v3(0, 0, 0), o = v3(0, 0, 0), d = v3(0, 0, 0);
  int depth = 0;
  bool path = false, done = false;
  // Vertex stack of the current sample.
  int vm[kMaxVertices];
  float3 vthr[kMaxVertices], vw[kMaxVertices];
  float vinvp[kMaxVertices];
  int nv = 0;
  bool escaped = false;
  const float aspect = (float)a.width / (float)a.height;
  while (true) {
    bool need = !done && pixel < 0;
    unsigned need_mask = __ballot_sync(0xFFFFFFFFu, need);
    if (need_mask) {
      unsigned long long basep = 0;
      int leader = __ffs(need_mask) - 1;
      if (lane == leader)
        basep = abort_raised(a.abort_flag) ? (unsigned long long)a.pixels
                                           : atomicAdd(a.queue, (unsigned long long)__popc(need_mask));
      basep = __shfl_sync(0xFFFFFFFFu, basep, leader);
      if (need) {
        long long p = (long long)basep + __popc(need_mask & ((1u << lane) - 1u));
        if (p >= a.pixels) {
          done = true;
        } else {
          pixel = p;
          x = (int)(p % a.width);
          y = (int)(p / a.width);
          so = 0;
          uint32_t s = hash_u32((uint32_t)(a.frame_seed & 0xFFFFFFFFULL));
          s ^= hash_u32((uint32_t)(a.frame_seed >> 32));
          s ^= hash_u32((uint32_t)a.frame_index);
          s ^= hash_u32((uint32_t)y * (uint32_t)a.width + (uint32_t)x);
          base_seed = hash_u32(s);
          float inv_spp = 1.0f / (float)a.spp;
          const float* ap = a.adjoint + 3 * p;
          adj = v3(ap[0] * inv_spp, ap[1] * inv_spp, ap[2] * inv_spp);
        }
      }
    }
    if (__all_sync(0xFFFFFFFFu, done)) break;
    if (!done && !path) {  // replay the sample's camera ray (K:1251-1264)
      uint32_t seed = base_seed ^ hash_u32((uint32_t)so);
      seed ^= hash_u32((uint32_t)(so * 0x9E3779B9u));
      rng = hash_u32(seed);
      float jx = rand01(&rng) - 0.5f;
      float jy = rand01(&rng) - 0.5f;
      float u = ((((float)x + 0.5f) + jx) * (2.0f / (float)a.width) - 1.0f) * aspect;
      float v = 1.0f - ((((float)y + 0.5f) + jy) * (2.0f / (float)a.height));
      o = a.cam_pos;
      d = add(add(a.cam_f, mul(a.cam_r, u)), mul(a.cam_u, v));
      thr = v3(1.0f, 1.0f, 1.0f);
      depth = 0;
      nv = 0;
      escaped = false;
      path = a.max_depth > 0;
    }
    bool finished = !done && !path;
    bool tracing = !done && path;
    Best b;
    bool hit = trace_closest<false>(S, o, d, tracing, b, nullptr, nullptr);
    if (tracing) {
      if (!hit) {
        escaped = true;
        finished = true;
      } else {
        float3 pos, n;
        int mi;
        hit_record(S, b, o, d, &pos, &n, &mi);
        float4 m0 = make_float4(0, 0, 0, 0), m1 = m0, m2 = m0;
        if (mi >= 0) {
          const float4* mp = S.materials + 4 * mi;
          m0 = __ldg(mp);
          m1 = __ldg(mp + 1);
          m2 = __ldg(mp + 2);
        }
        float3 cd = v3(m0.x, m0.y, m0.z), cr = v3(m1.x, m1.y, m1.z), ct = v3(m2.x, m2.y, m2.z);
        float3 inc = neg(d);
        float wd = luminance(cd), wr = luminance(cr), wt = luminance(ct);
        float sum = wd + wr + wt;
        vm[nv] = mi;
        vthr[nv] = thr;
        vw[nv] = v3(0.0f, 0.0f, 0.0f);
        vinvp[nv] = 0.0f;  // 0: no albedo gradient through this vertex
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
            vinvp[nv] = 1.0f / pc;
          } else if (xi < wd + wr) {
            float pc = wr / sum;
            nd = reflect_dir(n, inc);
            wc = divs(cr, pc);
          } else {
            float pc = wt / sum;
            nd = refract_dir(inc, n, m0.w);
            wc = divs(ct, pc);
          }
          vw[nv] = wc;
          o = add(pos, mul(nd, kEps));
          thr = mulv(thr, wc);
          d = nd;
          depth++;
          if (depth >= a.max_depth) finished = true;
        }
        nv++;
      }
    }
    if (finished) {
      path = false;
      if (nv > 0) {
        // Backward over the sample's vertices.
        float3 li = escaped ? S.background : v3(0.0f, 0.0f, 0.0f);
        for (int k = nv - 1; k >= 0; --k) {
          int m = vm[k];
          float3 e = v3(0.0f, 0.0f, 0.0f);
          if (m >= 0) {
            float4 m3 = __ldg(S.materials + 4 * m + 3);
            e = v3(m3.x, m3.y, m3.z);
            float3 base = mulv(adj, vthr[k]);
            float3 ga = mul(mulv(base, li), vinvp[k]);
            accumulate(T, a, m, ga, base);
          }
          li = add(e, mulv(vw[k], li));
        }
      }
      so++;
      if (so == a.spp) pixel = -1;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTable; i += blockDim.x) {
    int m = T.key[i];
    if (m < 0) continue;
    atomicAdd(a.grad_albedo + 3 * m, T.val[i][0]);
    atomicAdd(a.grad_albedo + 3 * m + 1, T.val[i][1]);
    atomicAdd(a.grad_albedo + 3 * m + 2, T.val[i][2]);
    atomicAdd(a.grad_emission + 3 * m, T.val[i][3]);
    atomicAdd(a.grad_emission + 3 * m + 1, T.val[i][4]);
    atomicAdd(a.grad_emission + 3 * m + 2, T.val[i][5]);
  }
}

__global__ void k_repack_materials(const float* raw, int n, float4* out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float* r = raw + 13 * (size_t)s;
  out[4 * s] = make_float4(r[0], r[1], r[2], r[12]);
  out[4 * s + 1] = make_float4(r[3], r[4], r[5], 0.0f);
  out[4 * s + 2] = make_float4(r[6], r[7], r[8], 0.0f);
  out[4 * s + 3] = make_float4(r[9], r[10], r[11], 0.0f);
}

}  // namespace
}  // namespace rtb

using namespace rtb;

extern "C" {

rtb_status rtb_scene_set_materials(rtb_context* ctx, rtb_scene* scene, const float* materials,
                                   int material_count) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  if (!scene || !materials || material_count != scene->dev.material_count)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "material table must keep the scene's material count");
  size_t bytes = (size_t)material_count * 13 * sizeof(float);
  float* raw = (float*)stage(ctx, bytes);
  if (!raw) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "material staging");
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  cudaMemcpyAsync(raw, materials, bytes, cudaMemcpyHostToDevice, sm);
  k_repack_materials<<<(material_count + 255) / 256, 256, 0, sm>>>(
      raw, material_count, const_cast<float4*>(scene->dev.materials));
  ctx_release(ctx, sm);
  cudaError_t e = cudaStreamSynchronize(sm);
  if (e == cudaSuccess) e = cudaGetLastError();
  return e == cudaSuccess ? RTB_OK : cuda_fail(ctx, e, "material update");
}

// The backward launch; the caller holds the context lock with its device current.
static rtb_status render_backward(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                                  const rtb_render_params* p, const float* adjoint_device,
                                  float* grad_albedo_device, float* grad_emission_device,
                                  cudaStream_t stream) {
  if (!scene || !cam || !p || !adjoint_device || !grad_albedo_device || !grad_emission_device)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (p->width < 1 || p->height < 1 || p->samples_per_frame < 1)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "image size and samples must be positive");
  if (p->max_depth < 0 || p->max_depth > kMaxVertices)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "GPU full-path depth must be in [0, 32]");
  cudaStream_t sm = stream ? stream : ctx->stream;
  ctx_acquire(ctx, sm);
  AdjointArgs a;
  a.S = scene->dev;
  a.S.use_bvh = (p->use_bvh && scene->has_bvh) ? 1 : 0;
  a.cam_pos = make_float3(cam->position[0], cam->position[1], cam->position[2]);
  a.cam_f = make_float3(cam->forward[0], cam->forward[1], cam->forward[2]);
  a.cam_r = make_float3(cam->right[0], cam->right[1], cam->right[2]);
  a.cam_u = make_float3(cam->up[0], cam->up[1], cam->up[2]);
  a.width = p->width;
  a.height = p->height;
  a.spp = p->samples_per_frame;
  a.max_depth = p->max_depth;
  a.frame_index = p->frame_index;
  a.frame_seed = p->frame_seed;
  a.adjoint = adjoint_device;
  a.grad_albedo = grad_albedo_device;
  a.grad_emission = grad_emission_device;
  a.pixels = (long long)p->width * p->height;
  a.queue = ctx->d_work;
  a.abort_flag = ctx->d_abort;
  size_t gbytes = (size_t)scene->dev.material_count * 3 * sizeof(float);
  cudaMemsetAsync(ctx->d_work, 0, sizeof(unsigned long long), sm);
  arm_abort(ctx, sm);
  cudaMemsetAsync(grad_albedo_device, 0, gbytes, sm);
  cudaMemsetAsync(grad_emission_device, 0, gbytes, sm);
  int bps = 1;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, (const void*)k_adjoint, 128, 0);
  if (bps < 1) bps = 1;
  long long grid = std::min<long long>((long long)ctx->sm_count * bps, (a.pixels + 127) / 128);
  cudaEventRecord(ctx->ev0, sm);
  k_adjoint<<<(unsigned)std::max<long long>(1, grid), 128, 0, sm>>>(a);
  cudaEventRecord(ctx->ev1, sm);
  ctx_release(ctx, sm);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint launch");
  return RTB_OK;
}

rtb_status rtb_render_backward(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                               const rtb_render_params* p, const float* adjoint_device,
                               float* grad_albedo_device, float* grad_emission_device, void* stream) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  return render_backward(ctx, scene, cam, p, adjoint_device, grad_albedo_device,
                         grad_emission_device, (cudaStream_t)stream);
}

rtb_status rtb_render_backward_sample(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                                      const rtb_render_params* p, const float* adjoint,
                                      float* grad_albedo, float* grad_emission) {
  if (!ctx) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  if (!scene || !p || !adjoint || !grad_albedo || !grad_emission)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (p->width < 1 || p->height < 1)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "image size and samples must be positive");
  size_t img = (size_t)p->width * p->height * 3 * sizeof(float);
  size_t grads = (size_t)scene->dev.material_count * 3 * sizeof(float);
  size_t img_pad = (img + 255) & ~(size_t)255, grads_pad = (grads + 255) & ~(size_t)255;
  char* d = (char*)stage(ctx, img_pad + 2 * grads_pad);
  if (!d) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "adjoint staging");
  float* d_adj = (float*)d;
  float* d_ga = (float*)(d + img_pad);
  float* d_ge = (float*)(d + img_pad + grads_pad);
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  cudaMemcpyAsync(d_adj, adjoint, img, cudaMemcpyHostToDevice, sm);
  ctx_release(ctx, sm);
  rtb_status s = render_backward(ctx, scene, cam, p, d_adj, d_ga, d_ge, sm);
  if (s != RTB_OK) return s;
  ctx_acquire(ctx, sm);
  cudaMemcpyAsync(grad_albedo, d_ga, grads, cudaMemcpyDeviceToHost, sm);
  cudaMemcpyAsync(grad_emission, d_ge, grads, cudaMemcpyDeviceToHost, sm);
  ctx_release(ctx, sm);
  cudaError_t e = cudaStreamSynchronize(sm);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "adjoint");
  int aborted = 0;
  cudaMemcpy(&aborted, ctx->d_abort + 2, sizeof(int), cudaMemcpyDeviceToHost);
  if (aborted) return fail(ctx, RTB_ERR_WATCHDOG, "backward pass aborted on request");
  return RTB_OK;
}

}  // extern "C"
