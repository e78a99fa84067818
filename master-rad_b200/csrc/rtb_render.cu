// Path-tracing and closest-hit kernels.
//
// Render: one persistent launch per frame (the reference issues one launch per sample and
// tile, GpuRayTracer.java:356-376).  Each resident thread owns one pixel at a time and runs
// its samples in order, one path segment per loop iteration; a lane whose path ends starts
// the next sample (or fetches the next pixel from a warp-aggregated queue) while the other
// lanes continue, so warps stay full across uneven path lengths.  The per-pixel sum is the
// reference's FP32 running sum over samples 0..spp-1 scaled by 1/spp after the last one
// (GpuKernelSources.java:1284-1293), and each sample consumes the reference's random
// stream (seed K:1231-1254, jitter and camera K:1256-1264, tracePath K:1061-1165), so the
// image matches the reference's renderKernel bit for bit under the same arithmetic.
//
// The frame's last pixels (about four per resident thread, or all of a small frame) are
// handed out one sample per queue item instead, so the end of the frame does not wait on
// a few lanes that each still hold a whole pixel.  Those samples' radiance goes to a
// buffer in item order and k_sum_tail adds each pixel's samples in sample order, the same
// FP32 additions as the in-register sum.
#include "rtb_internal.h"

namespace rtb {
namespace {

struct RenderArgs {
  DevScene S;
  float3 cam_pos, cam_f, cam_r, cam_u;
  int width, height, spp, max_depth, frame_index;
  unsigned long long frame_seed;
  float* out;
  long long pixels;                // pixels of the output (the frame, or a set of its rows)
  int row0, row_stride;            // output row k is frame row row0 + k * row_stride
  long long split;                 // pixels [split, pixels) are queued one sample per item
  long long items;                 // split + (pixels - split) * spp queue items
  float* tail;                     // RGB of each tail item, item - split order
  unsigned long long* queue;       // work queue head
  int* abort_flag;                 // the context's abort words (abort_raised)
  unsigned long long* counters;    // 14 counters (metrics build) + overflow count
};

__device__ __forceinline__ float luminance(float3 c) {  // K:181-183
  return c.x * 0.212655f + c.y * 0.715158f + c.z * 0.072187f;
}
__device__ __forceinline__ float3 reflect_dir(float3 n, float3 i) {  // K:1022-1024
  return sub(mul(n, 2.0f * dot(i, n)), i);
}
// Out of line: the refraction lobe is rare, and its code stays out of the frame loop.
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

__device__ __forceinline__ uint32_t pixel_base_seed(unsigned long long frame_seed, int frame_index,
                                                    uint32_t pixel) {  // K:1231-1236
  uint32_t s = hash_u32((uint32_t)(frame_seed & 0xFFFFFFFFULL));
  s ^= hash_u32((uint32_t)(frame_seed >> 32));
  s ^= hash_u32((uint32_t)frame_index);
  s ^= hash_u32(pixel);
  return hash_u32(s);
}

// One path segment after its closest-hit query (tracePath loop body, K:1098-1162): the
// background on a miss; else the hit's emission, the lobe chosen by luminance, and the
// next ray with its throughput.  Returns true when the path ends.  The wavefront kernels
// shade through this function; k_render keeps the same statements inline (as a function
// they cost it 1.5-3.6 % of its speed), and the tests hold the two forms' frames equal bit
// for bit.
__device__ __forceinline__ bool shade_segment(const DevScene& S, bool hit, const Best& b, float3& o,
                                              float3& d, float3& thr, float3& rad, uint32_t& rng,
                                              int& depth, int max_depth) {
  if (!hit) {
    rad = add(rad, mulv(thr, S.background));
    return true;
  }
  float3 pos, n;
  int mi;
  hit_record(S, b, o, d, &pos, &n, &mi);
  float4 m0 = make_float4(0, 0, 0, 0), m1 = m0, m2 = m0, m3 = m0;
  if (mi >= 0) {
    const float4* mp = S.materials + 4 * mi;
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
  if (sum <= 0.0f) return true;
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
  return depth >= max_depth;
}

// The camera ray of sample `so` of pixel (x, y) and its random stream (renderKernel
// prologue, K:1251-1264), for the wavefront kernels (k_render's prologue is inline).
__device__ __forceinline__ void camera_sample(const RenderArgs& a, int x, int y, int so,
                                              uint32_t base_seed, uint32_t& rng, float3& o,
                                              float3& d) {
  uint32_t seed = base_seed ^ hash_u32((uint32_t)so);
  seed ^= hash_u32((uint32_t)(so * 0x9E3779B9u));
  rng = hash_u32(seed);
  const float aspect = (float)a.width / (float)a.height;
  float jx = rand01(&rng) - 0.5f;
  float jy = rand01(&rng) - 0.5f;
  float u = ((((float)x + 0.5f) + jx) * (2.0f / (float)a.width) - 1.0f) * aspect;
  float v = 1.0f - ((((float)y + 0.5f) + jy) * (2.0f / (float)a.height));
  o = a.cam_pos;
  d = add(add(a.cam_f, mul(a.cam_r, u)), mul(a.cam_u, v));
}

// SDEPTH traversal-stack entries per thread in shared memory (16 KB a block at 16), for
// scenes far larger than the caches: there the local-memory stack's lines compete with the
// scene for L1 and L2.  A scene that the caches hold keeps the whole stack in local memory
// and the caches for itself.
#ifndef RTB_RENDER_BLOCKS_PER_SM
#define RTB_RENDER_BLOCKS_PER_SM 8  // 64 registers a thread; 6, 7 and 9 measured slower
#endif
template <bool METRICS, int SDEPTH>
__global__ void __launch_bounds__(128, RTB_RENDER_BLOCKS_PER_SM) k_render(RenderArgs a) {
  __shared__ int2 s_stack[SDEPTH > 0 ? SDEPTH : 1][128];
  const DevScene& S = a.S;
  const int lane = threadIdx.x & 31;
  TraceCounters c{};
  unsigned long long rays = 0;
  // Per-lane state.
  long long pixel = -1;
  int x = 0, y = 0, so = 0;
  int titem = -1;  // tail item of a single-sample lane, -1 while the lane holds a whole pixel
  uint32_t base_seed = 0, rng = 0;
  float3 acc = v3(0, 0, 0), thr = v3(0, 0, 0), rad = v3(0, 0, 0), o = v3(0, 0, 0), d = v3(0, 0, 0);
  int depth = 0;
  bool path = false;
  bool done = false;
  const float aspect = (float)a.width / (float)a.height;
  while (true) {
    // ---- fetch a pixel (warp-aggregated) for lanes that need one
    bool need = !done && pixel < 0;
    unsigned need_mask = __ballot_sync(0xFFFFFFFFu, need);
    if (need_mask) {
      unsigned long long basep = 0;
      int leader = __ffs(need_mask) - 1;
      if (lane == leader) {
        basep = abort_raised(a.abort_flag) ? (unsigned long long)a.items
                                           : atomicAdd(a.queue, (unsigned long long)__popc(need_mask));
      }
      basep = __shfl_sync(0xFFFFFFFFu, basep, leader);
      if (need) {
        long long p = (long long)basep + __popc(need_mask & ((1u << lane) - 1u));
        if (p >= a.items) {
          done = true;
        } else {
          if (p < a.split) {
            so = 0;
            titem = -1;
          } else {
            titem = (int)(p - a.split);
            so = (int)((unsigned)titem % (unsigned)a.spp);
            p = a.split + (long long)((unsigned)titem / (unsigned)a.spp);
          }
          pixel = p;
          x = (int)(p % a.width);
          y = a.row0 + (int)(p / a.width) * a.row_stride;
          base_seed = pixel_base_seed(a.frame_seed, a.frame_index,
                                      (uint32_t)y * (uint32_t)a.width + (uint32_t)x);
        }
      }
    }
    if (__all_sync(0xFFFFFFFFu, done)) break;
    // ---- start a sample (renderKernel prologue, K:1251-1264)
    if (!done && !path) {
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
      rad = v3(0.0f, 0.0f, 0.0f);
      depth = 0;
      path = a.max_depth > 0;
    }
    // ---- one path segment (tracePath loop body, K:1098-1162)
    bool finished = !done && !path;  // max_depth == 0: the sample is black
    bool tracing = !done && path;
    Best b;
    bool hit = trace_closest<METRICS, SDEPTH, 128>(S, o, d, tracing, b, &c, nullptr,
                                                  &s_stack[0][threadIdx.x]);
    if (tracing) {
      if (METRICS) rays++;
      if (!hit) {
        rad = add(rad, mulv(thr, S.background));
        finished = true;
      } else {
        float3 pos, n;
        int mi;
        hit_record(S, b, o, d, &pos, &n, &mi);
        float4 m0 = make_float4(0, 0, 0, 0), m1 = m0, m2 = m0, m3 = m0;
        if (mi >= 0) {
          const float4* mp = S.materials + 4 * mi;
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
          if (depth >= a.max_depth) finished = true;
        }
      }
    }
    if (finished && titem >= 0) {
      path = false;
      float* t = a.tail + 3 * (size_t)titem;
      t[0] = rad.x;
      t[1] = rad.y;
      t[2] = rad.z;
      pixel = -1;
    } else if (finished) {
      path = false;
      acc = so == 0 ? rad : add(acc, rad);
      so++;
      if (so == a.spp) {
        acc = mul(acc, 1.0f / (float)a.spp);
        float* out = a.out + 3 * pixel;
        out[0] = acc.x;
        out[1] = acc.y;
        out[2] = acc.z;
        pixel = -1;
      }
    }
  }
  if (METRICS) {
    unsigned long long* k = a.counters;
    atomicAdd(k + 0, rays);
    atomicAdd(k + 1, c.aabb);
    atomicAdd(k + 2, c.prim);
    atomicAdd(k + 3, c.type[0]);
    atomicAdd(k + 4, c.type[1]);
    atomicAdd(k + 5, c.type[2]);
    atomicAdd(k + 6, c.type[3]);
    atomicAdd(k + 7, c.type[4]);
    atomicAdd(k + 8, c.overflow);
    atomicMax(k + 9, c.maxstack);
    atomicAdd(k + 10, c.internal);
    atomicAdd(k + 11, c.leaf);
    atomicAdd(k + 12, c.homo);
    atomicAdd(k + 13, c.mixed);
  }
}

// One thread per tail pixel: the in-order FP32 sum of its samples, scaled as in k_render.
// A frame whose render stopped on an abort leaves tail pixels unwritten, like the pixels it
// never fetched.
__global__ void __launch_bounds__(256) k_sum_tail(const float* __restrict__ tail, float* out,
                                                 long long split, int tail_pixels, int spp,
                                                 const int* abort_flag) {
  int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= tail_pixels || abort_stopped(abort_flag)) return;
  const float* s = tail + 3 * (size_t)q * spp;
  float3 acc = v3(s[0], s[1], s[2]);
  for (int i = 1; i < spp; i++) acc = add(acc, v3(s[3 * i], s[3 * i + 1], s[3 * i + 2]));
  acc = mul(acc, 1.0f / (float)spp);
  float* o = out + 3 * (split + q);
  o[0] = acc.x;
  o[1] = acc.y;
  o[2] = acc.z;
}

template <bool METRICS>
__global__ void __launch_bounds__(256) k_trace(DevScene S, const float* rays, int n, int* flags,
                                               float* dist, int* order, int* mat, float* normal,
                                               unsigned long long* counters) {
  int r = blockIdx.x * blockDim.x + threadIdx.x;
  bool active = r < n;  // every lane stays for the warp-cooperative traversal
  float3 o = v3(0.0f, 0.0f, 0.0f), d = v3(0.0f, 0.0f, 1.0f);
  if (active) {
    const float* ry = rays + 6 * (size_t)r;
    o = v3(ry[0], ry[1], ry[2]);
    d = v3(ry[3], ry[4], ry[5]);
  }
  TraceCounters c{};
  Best b;
  bool hit = trace_closest<METRICS>(S, o, d, active, b, &c, nullptr);
  if (!active) return;
  float3 pos, nn = v3(0, 0, 0);
  int mi = -1;
  if (hit) hit_record(S, b, o, d, &pos, &nn, &mi);
  flags[r] = hit ? 1 : 0;
  dist[r] = hit ? b.t : CUDART_INF_F;
  order[r] = hit ? b.order : -1;
  mat[r] = hit ? mi : -1;
  normal[3 * (size_t)r] = nn.x;
  normal[3 * (size_t)r + 1] = nn.y;
  normal[3 * (size_t)r + 2] = nn.z;
  if (METRICS) {
    atomicAdd(counters + 0, 1ULL);
    atomicAdd(counters + 1, c.aabb);
    atomicAdd(counters + 2, c.prim);
    atomicAdd(counters + 3, c.type[0]);
    atomicAdd(counters + 4, c.type[1]);
    atomicAdd(counters + 5, c.type[2]);
    atomicAdd(counters + 6, c.type[3]);
    atomicAdd(counters + 7, c.type[4]);
    atomicAdd(counters + 8, c.overflow);
    atomicMax(counters + 9, c.maxstack);
    atomicAdd(counters + 10, c.internal);
    atomicAdd(counters + 11, c.leaf);
    atomicAdd(counters + 12, c.homo);
    atomicAdd(counters + 13, c.mixed);
  }
}

int g_render_blocks_per_sm[2][3] = {{0, 0, 0}, {0, 0, 0}};

// Scenes whose traversal data (nodes, references, primitive records) exceed this many bytes
// use the shared-memory stack: on the 1M-primitive scene (about 150 MB) it was 5 % faster,
// on the 10k scene (about 2 MB) 1.7 % slower.
constexpr long long kSharedStackSceneBytes = 16LL << 20;
constexpr int kSharedStackDepth = 16;

#ifndef RTB_TAIL_FACTOR
#define RTB_TAIL_FACTOR 4.0
#endif
// At most 64M tail samples (768 MB of radiance, held by the context); frames whose last
// four pixels per resident thread hold more samples split fewer pixels.
constexpr long long kMaxTailItems = 1LL << 26;

// ---- the wavefront form of a frame (rtb_render_device_wavefront)
//
// One wave per sample index over every pixel of the frame; per bounce, k_wf_trace runs the
// closest-hit query of every live path of the wave (the compacted list) and k_wf_shade
// shades it through shade_segment (k_render's segment statements), appending the paths
// that go on to the next list.  Path state lives in HBM, 16-byte records per path: origin, direction,
// throughput with the random stream's state, radiance with the depth, and the hit.  A
// pixel's samples are summed in sample order, one wave after the other, as k_render sums
// them, so the image is bit-identical.  It exists as the A/B counterpart of the persistent
// kernel: on the B200 it is slower (the state round trips and the per-bounce launches cost
// more than the warps' coherence buys).
struct WaveState {
  float4* o;    // origin (w unused)
  float4* d;    // direction (w unused)
  float4* thr;  // throughput; w holds the random stream's state
  float4* rad;  // radiance; w holds the depth
  Best* hit;
  int* list[2];
  int* count;   // sizes of list[0] and list[1]
};

__global__ void __launch_bounds__(256) k_wf_start(RenderArgs a, WaveState W, int so, int cur) {
  const long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= a.pixels) return;
  const int x = (int)(p % a.width), y = (int)(p / a.width);
  if (p == 0) W.count[cur] = (a.max_depth > 0 && !abort_raised(a.abort_flag)) ? (int)a.pixels : 0;
  if (a.max_depth <= 0) {  // a black sample, summed like k_render's
    float* out = a.out + 3 * p;
    float3 acc = so == 0 ? v3(0, 0, 0) : add(v3(out[0], out[1], out[2]), v3(0, 0, 0));
    if (so + 1 == a.spp) acc = mul(acc, 1.0f / (float)a.spp);
    out[0] = acc.x;
    out[1] = acc.y;
    out[2] = acc.z;
    return;
  }
  uint32_t rng;
  float3 o, d;
  camera_sample(a, x, y, so,
                pixel_base_seed(a.frame_seed, a.frame_index, (uint32_t)y * (uint32_t)a.width + (uint32_t)x),
                rng, o, d);
  W.o[p] = make_float4(o.x, o.y, o.z, 0.0f);
  W.d[p] = make_float4(d.x, d.y, d.z, 0.0f);
  W.thr[p] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(rng));
  W.rad[p] = make_float4(0.0f, 0.0f, 0.0f, __int_as_float(0));
  W.list[cur][p] = (int)p;
}

template <int SDEPTH>
__global__ void __launch_bounds__(128, RTB_RENDER_BLOCKS_PER_SM) k_wf_trace(RenderArgs a, WaveState W,
                                                                           int cur) {
  __shared__ int2 s_stack[SDEPTH > 0 ? SDEPTH : 1][128];
  const int n = W.count[cur];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if ((i & ~31) >= n) return;  // whole warps only: the traversal is warp-cooperative
  const bool active = i < n;
  const int p = active ? W.list[cur][i] : 0;
  float3 o = v3(0, 0, 0), d = v3(0, 0, 0);
  if (active) {
    const float4 o4 = W.o[p], d4 = W.d[p];
    o = v3(o4.x, o4.y, o4.z);
    d = v3(d4.x, d4.y, d4.z);
  }
  Best b;
  TraceCounters c{};
  const bool hit = trace_closest<false, SDEPTH, 128>(a.S, o, d, active, b, &c, nullptr,
                                                    &s_stack[0][threadIdx.x]);
  if (active) {
    if (!hit) b.type = -1;
    W.hit[p] = b;
  }
}

__global__ void __launch_bounds__(256) k_wf_shade(RenderArgs a, WaveState W, int so, int cur) {
  const int n = W.count[cur];
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  if ((i & ~31) >= n) return;
  bool more = false;
  int p = 0;
  if (i < n) {
    p = W.list[cur][i];
    const float4 o4 = W.o[p], d4 = W.d[p], t4 = W.thr[p], r4 = W.rad[p];
    float3 o = v3(o4.x, o4.y, o4.z), d = v3(d4.x, d4.y, d4.z);
    float3 thr = v3(t4.x, t4.y, t4.z), rad = v3(r4.x, r4.y, r4.z);
    uint32_t rng = __float_as_uint(t4.w);
    int depth = __float_as_int(r4.w);
    const Best b = W.hit[p];
    if (shade_segment(a.S, b.type >= 0, b, o, d, thr, rad, rng, depth, a.max_depth)) {
      float* out = a.out + 3 * (size_t)p;
      float3 acc = so == 0 ? rad : add(v3(out[0], out[1], out[2]), rad);
      if (so + 1 == a.spp) acc = mul(acc, 1.0f / (float)a.spp);
      out[0] = acc.x;
      out[1] = acc.y;
      out[2] = acc.z;
    } else {
      W.o[p] = make_float4(o.x, o.y, o.z, 0.0f);
      W.d[p] = make_float4(d.x, d.y, d.z, 0.0f);
      W.thr[p] = make_float4(thr.x, thr.y, thr.z, __uint_as_float(rng));
      W.rad[p] = make_float4(rad.x, rad.y, rad.z, __int_as_float(depth));
      more = true;
    }
  }
  // warp-aggregated append to the next bounce's list
  const unsigned m = __ballot_sync(0xFFFFFFFFu, more);
  if (m) {
    const int leader = __ffs(m) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(W.count + (cur ^ 1), __popc(m));
    base = __shfl_sync(0xFFFFFFFFu, base, leader);
    if (more) W.list[cur ^ 1][base + __popc(m & ((1u << lane) - 1u))] = p;
  }
}

}  // namespace

// One frame's launch: arguments, grid, and how many of its last pixels run one sample per
// item.  Built by plan_frame; the caller binds the queue, sample buffer and flags.
struct FramePlan {
  RenderArgs a;
  int metrics = 0;
  int shared_stack = 0;       // k_render's SDEPTH: 0, 8 or kSharedStackDepth
  long long resident = 0;     // threads of a full-occupancy grid
  long long tail_pixels = 0;  // the frame's last pixels, queued one sample per item
  long long grid = 0;
};

namespace {

const void* render_kernel(int metrics, int shared_stack) {
  if (shared_stack == kSharedStackDepth)
    return metrics ? (const void*)k_render<true, kSharedStackDepth>
                   : (const void*)k_render<false, kSharedStackDepth>;
  if (shared_stack == 8)
    return metrics ? (const void*)k_render<true, 8> : (const void*)k_render<false, 8>;
  return metrics ? (const void*)k_render<true, 0> : (const void*)k_render<false, 0>;
}

int frame_blocks_per_sm(int metrics, int shared_stack) {
  int& bps = g_render_blocks_per_sm[metrics][shared_stack == 0 ? 0 : shared_stack == 8 ? 1 : 2];
  if (bps == 0) {
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, render_kernel(metrics, shared_stack), 128, 0);
    if (bps < 1) bps = 1;
  }
  return bps;
}

long long traversal_bytes(const DevScene& S) {
  return (long long)S.node_count * 64 + (long long)S.ref_count * 4 + (long long)S.count[kSphere] * 16 +
         (long long)S.count[kBox] * 32 + ((long long)S.count[kAffineSphere] + S.count[kAffineBox]) * 48;
}

void set_tail(FramePlan* f, long long tail_pixels) {
  RenderArgs& a = f->a;
  f->tail_pixels = tail_pixels;
  a.split = a.pixels - tail_pixels;
  a.items = a.split + tail_pixels * a.spp;
  long long want = (a.items + 127) / 128;
  f->grid = std::min<long long>(f->resident / 128, want);
}

}  // namespace

rtb_status plan_frame(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                      const rtb_render_params* p, float* d_rgb, FramePlan* f, int row0,
                      int row_stride, int tail_per_thread) {
  if (!scene || !cam || !p || !d_rgb) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (p->width < 1 || p->height < 1 || p->samples_per_frame < 1)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "image size and samples must be positive");
  if (p->max_depth < 0 || p->max_depth > 32)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT,
                "GPU full-path depth must be in [0, 32] but was " + std::to_string(p->max_depth));
  RenderArgs& a = f->a;
  a = RenderArgs{};
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
  if (row0 < 0 || row0 >= p->height || row_stride < 1)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "first row must be in [0, height) and the stride positive");
  a.out = d_rgb;
  a.row0 = row0;
  a.row_stride = row_stride;
  a.pixels = (long long)p->width * ((p->height - row0 + row_stride - 1) / row_stride);
  f->metrics = p->collect_metrics ? 1 : 0;
  // rtb_render_params.shared_stack_entries: 0 picks by scene size, -1 none, 8 or 16 entries
  int se = p->shared_stack_entries;
  if (se != 0 && se != -1 && se != 8 && se != kSharedStackDepth)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "shared_stack_entries must be 0, -1, 8 or 16");
  f->shared_stack = se == 0 ? (traversal_bytes(a.S) > kSharedStackSceneBytes ? kSharedStackDepth : 0)
                  : se < 0 ? 0 : se;
  f->resident = (long long)ctx->sm_count * frame_blocks_per_sm(f->metrics, f->shared_stack) * 128;
  // Tail: about four pixels per resident thread are split into single samples.
  double per_thread = tail_per_thread > 0 ? (double)tail_per_thread : RTB_TAIL_FACTOR;
  long long tail_pixels = std::min<long long>(a.pixels, (long long)(per_thread * f->resident));
  set_tail(f, std::min<long long>(tail_pixels, kMaxTailItems / a.spp));
  return RTB_OK;
}

size_t frame_tail_bytes(const FramePlan* f) {
  return (size_t)f->tail_pixels * f->a.spp * 3 * sizeof(float);
}

void bind_frame(FramePlan* f, unsigned long long* queue, float* tail, int* abort_flag,
                unsigned long long* counters) {
  if (!tail) set_tail(f, 0);  // no buffer: every pixel keeps its samples in one lane
  f->a.queue = queue;
  f->a.tail = tail;
  f->a.abort_flag = abort_flag;
  f->a.counters = counters;
}

int launch_frame(const FramePlan* f, cudaStream_t stream) {
  const RenderArgs& a = f->a;
  if (f->shared_stack == kSharedStackDepth) {
    if (f->metrics)
      k_render<true, kSharedStackDepth><<<(unsigned)f->grid, 128, 0, stream>>>(a);
    else
      k_render<false, kSharedStackDepth><<<(unsigned)f->grid, 128, 0, stream>>>(a);
  } else if (f->shared_stack == 8) {
    if (f->metrics)
      k_render<true, 8><<<(unsigned)f->grid, 128, 0, stream>>>(a);
    else
      k_render<false, 8><<<(unsigned)f->grid, 128, 0, stream>>>(a);
  } else {
    if (f->metrics)
      k_render<true, 0><<<(unsigned)f->grid, 128, 0, stream>>>(a);
    else
      k_render<false, 0><<<(unsigned)f->grid, 128, 0, stream>>>(a);
  }
  if (f->tail_pixels == 0) return 1;
  k_sum_tail<<<(unsigned)((f->tail_pixels + 255) / 256), 256, 0, stream>>>(
      a.tail, a.out, a.split, (int)f->tail_pixels, a.spp, a.abort_flag);
  return 2;
}

FramePlan* new_frame_plan() { return new FramePlan(); }
void delete_frame_plan(FramePlan* f) { delete f; }

rtb_status render_frame(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                        const rtb_render_params* p, float* d_rgb, cudaStream_t stream, bool timed,
                        int row0, int row_stride) {
  FramePlan f;
  rtb_status s = plan_frame(ctx, scene, cam, p, d_rgb, &f, row0, row_stride);
  if (s != RTB_OK) return s;
  size_t tail_bytes = frame_tail_bytes(&f);
  if (tail_bytes > ctx->tail_bytes) {
    cudaStreamSynchronize(stream);  // the previous frame's sum may still read the buffer
    cudaFree(ctx->d_tail);
    ctx->d_tail = nullptr;
    ctx->tail_bytes = 0;
    if (cudaMalloc(&ctx->d_tail, tail_bytes) == cudaSuccess) {
      ctx->tail_bytes = tail_bytes;
    } else {
      cudaGetLastError();
      ctx->d_tail = nullptr;
    }
  }
  bind_frame(&f, ctx->d_work, ctx->d_tail, ctx->d_abort, ctx->d_work + 8);
  cudaMemsetAsync(ctx->d_work, 0, 32 * sizeof(unsigned long long), stream);
  if (timed) cudaEventRecord(ctx->ev0, stream);
  ctx->render_launches = launch_frame(&f, stream);
  if (timed) cudaEventRecord(ctx->ev1, stream);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "render launch");
  return RTB_OK;
}

cudaError_t launch_trace(const DevScene& scene, int use_bvh, const float* d_rays, int n, int* d_flags,
                         float* d_t, int* d_order, int* d_mat, float* d_normal, cudaStream_t stream) {
  DevScene S = scene;
  S.use_bvh = use_bvh ? scene.use_bvh : 0;
  if (n > 0)
    k_trace<false><<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(S, d_rays, n, d_flags, d_t, d_order,
                                                                    d_mat, d_normal, nullptr);
  return cudaGetLastError();
}

rtb_status trace_rays(rtb_context* ctx, rtb_scene* scene, const float* d_rays, int n, int use_bvh,
                      int collect_metrics, int* d_flags, float* d_t, int* d_order, int* d_mat,
                      float* d_normal, cudaStream_t stream) {
  DevScene S = scene->dev;
  S.use_bvh = (use_bvh && scene->has_bvh) ? 1 : 0;
  unsigned long long* counters = ctx->d_work + 8;
  cudaMemsetAsync(ctx->d_work, 0, 32 * sizeof(unsigned long long), stream);
  unsigned grid = (unsigned)((n + 255) / 256);
  if (n > 0) {
    if (collect_metrics)
      k_trace<true><<<grid, 256, 0, stream>>>(S, d_rays, n, d_flags, d_t, d_order, d_mat, d_normal, counters);
    else
      k_trace<false><<<grid, 256, 0, stream>>>(S, d_rays, n, d_flags, d_t, d_order, d_mat, d_normal, counters);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "trace launch");
  return RTB_OK;
}

rtb_status render_frame_wavefront(rtb_context* ctx, rtb_scene* scene, const rtb_camera* cam,
                                  const rtb_render_params* p, float* d_rgb, cudaStream_t stream) {
  FramePlan f;
  rtb_status s = plan_frame(ctx, scene, cam, p, d_rgb, &f, 0, 1);
  if (s != RTB_OK) return s;
  if (f.metrics) return fail(ctx, RTB_ERR_UNSUPPORTED, "the wavefront form has no metrics build");
  const long long P = f.a.pixels;
  if (P > 0x7FFFFFFFLL) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "frame too large");
  // path state: four 16-byte records, the hit and two list slots per pixel, two counts
  const size_t bytes = (size_t)P * (4 * sizeof(float4) + sizeof(Best) + 2 * sizeof(int)) + 256;
  if (bytes > ctx->wave_bytes) {
    cudaStreamSynchronize(stream);  // an earlier wavefront frame may still use the buffer
    cudaFree(ctx->d_wave);
    ctx->d_wave = nullptr;
    ctx->wave_bytes = 0;
    if (cudaMalloc(&ctx->d_wave, bytes) != cudaSuccess) {
      cudaGetLastError();
      return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "wavefront path state");
    }
    ctx->wave_bytes = bytes;
  }
  char* q = (char*)ctx->d_wave;
  WaveState W;
  W.o = (float4*)q;
  W.d = W.o + P;
  W.thr = W.d + P;
  W.rad = W.thr + P;
  W.hit = (Best*)(W.rad + P);
  W.list[0] = (int*)(W.hit + P);
  W.list[1] = W.list[0] + P;
  W.count = W.list[1] + P;
  f.a.abort_flag = ctx->d_abort;
  const unsigned g256 = (unsigned)((P + 255) / 256), g128 = (unsigned)((P + 127) / 128);
  int launches = 0;
  for (int so = 0; so < f.a.spp; ++so) {
    int cur = 0;
    k_wf_start<<<g256, 256, 0, stream>>>(f.a, W, so, cur);
    ++launches;
    for (int b = 0; b < f.a.max_depth; ++b) {
      if (f.shared_stack == kSharedStackDepth)
        k_wf_trace<kSharedStackDepth><<<g128, 128, 0, stream>>>(f.a, W, cur);
      else if (f.shared_stack == 8)
        k_wf_trace<8><<<g128, 128, 0, stream>>>(f.a, W, cur);
      else
        k_wf_trace<0><<<g128, 128, 0, stream>>>(f.a, W, cur);
      cudaMemsetAsync(W.count + (cur ^ 1), 0, sizeof(int), stream);
      k_wf_shade<<<g256, 256, 0, stream>>>(f.a, W, so, cur);
      launches += 2;
      cur ^= 1;
    }
  }
  ctx->render_launches = launches;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(ctx, e, "wavefront launch");
  return RTB_OK;
}

}  // namespace rtb
