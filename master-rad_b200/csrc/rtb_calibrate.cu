// Primitive-cost calibration on the device: relative cost of each intersection operation
// of this library's traversal, normalised to the sphere test.  The counterpart of the
// reference's PrimitiveCostBenchmark (gfxlab/gpu/PrimitiveCostBenchmark.java), which
// measured its own kernel on an RTX 3080 and produced the constants of
// PrimitiveCostModel.java:11-19; here the operations are the ones rtb_device.cuh runs.
//
// Protocol (PrimitiveCostBenchmark.java:115-131, 200-266, 345-405):
//  * one launch shape; every thread draws a ray of the current profile and `copies`
//    records per iteration by the counter hash, calls the operation through a
//    non-inlined wrapper and folds the full result into an accumulator, so nothing is
//    removed and the call and consumer cost is the same for every operation;
//  * an observation is `sublaunches` timed launches of the operation alternated with the
//    same launches of the setup operation (the wrapper without a test); its net cost per
//    test is (operation - setup) / tests, the first launch of each pair alternating;
//  * every operation observation is paired with a sphere observation (alternating which
//    comes first) so clock drift cancels in the ratio operation / sphere;
//  * per profile the ratio of the medians over the repeats, then the median over the
//    ray profiles is the recommended weight.
#include <algorithm>
#include <cmath>
#include <vector>

#include "rtb_internal.h"

namespace rtb {
namespace {

struct CalData {
  const float* rays;      // profiles x records x 6 (origin, direction)
  const float4* spheres;  // records
  const float4* boxes;    // 2 x records (lo, hi)
  const float4* affines;  // 3 x records (inverse rows, centre in .w)
  const float4* planes;   // records (unit normal, offset)
  const float4* nodes;    // 4 x records: child-pair nodes (rtb_device.cuh layout)
  int records;            // a power of two
};

// The operation under test; TYPE 0 is the setup wrapper alone.  Labels follow the
// reference: 1 sphere, 2 box, 3 affine sphere, 4 affine box, 5 node AABB, 6 interior
// traversal (both child boxes and their order), 7 plane.
template <int TYPE>
__device__ __noinline__ float2 cost_op(const CalData D, int idx, float3 o, float3 d, float dd, float3 inv) {
  float limit = 64.0f + fabsf(o.x) + fabsf(o.y) + fabsf(o.z);
  float3 n;
  if (TYPE == 0) return make_float2(limit, (float)idx);
  if (TYPE == 1) return make_float2(sphere_test<false>(__ldg(D.spheres + idx), o, d, dd, &n), 0.0f);
  if (TYPE == 2)
    return make_float2(box_test<false>(__ldg(D.boxes + 2 * idx), __ldg(D.boxes + 2 * idx + 1), o, d, &n),
                       0.0f);
  if (TYPE == 3) {
    const float4* r = D.affines + 3 * idx;
    return make_float2(affine_sphere_test<false>(__ldg(r), __ldg(r + 1), __ldg(r + 2), o, d, dd, nullptr, &n),
                       0.0f);
  }
  if (TYPE == 4) {
    const float4* r = D.affines + 3 * idx;
    return make_float2(affine_box_test<false>(__ldg(r), __ldg(r + 1), __ldg(r + 2), o, d, dd, nullptr, &n),
                       0.0f);
  }
  if (TYPE == 5) {
    float4 lo = __ldg(D.boxes + 2 * idx), hi = __ldg(D.boxes + 2 * idx + 1);
    return make_float2(child_entry(lo.x, hi.x, lo.y, hi.y, lo.z, hi.z, o, inv, limit), 0.0f);
  }
  if (TYPE == 6) {
    const float4* np = D.nodes + 4 * idx;
    float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
    float e0 = child_entry(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, limit);
    float e1 = child_entry(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, limit);
    bool swap = e1 < e0;
    return make_float2(swap ? e1 : e0, swap ? 1.0f : 0.0f);
  }
  // TYPE 7: tracePlane's test (K:708-734), as in trace_closest
  float4 p = __ldg(D.planes + idx);
  float3 pn = v3(p.x, p.y, p.z);
  float den = dot(pn, d);
  float t = den == 0.0f ? CUDART_INF_F : -(dot(pn, o) + p.w) / den;
  return make_float2(t <= kEps ? CUDART_INF_F : t, 0.0f);
}

template <int TYPE>
__global__ void __launch_bounds__(256) k_cost(const CalData D, int profile, int it0, int iters, int copies,
                                              float* out) {
  int tid = blockIdx.x * blockDim.x + threadIdx.x;
  float acc = 0.0f;
  const unsigned mask = (unsigned)D.records - 1u;
  for (int i = 0; i < iters; ++i) {
    unsigned sample = hash_u32((unsigned)(it0 + i) * 0x9E3779B9u + (unsigned)tid);
    int ray = (int)(sample & mask);
    const float* r = D.rays + 6 * ((size_t)profile * D.records + ray);
    float3 o = v3(r[0], r[1], r[2]), d = v3(r[3], r[4], r[5]);
    float dd = dot(d, d);
    float3 inv = v3(d.x != 0.0f ? 1.0f / d.x : 1e30f, d.y != 0.0f ? 1.0f / d.y : 1e30f,
                    d.z != 0.0f ? 1.0f / d.z : 1e30f);
    for (int c = 0; c < copies; ++c) {
      unsigned rs = hash_u32(sample ^ ((unsigned)(c + 1) * 0x85EBCA6Bu));
      int idx = (int)(rs & mask);
      float2 h = cost_op<TYPE>(D, idx, o, d, dd, inv);
      float t = isfinite(h.x) ? h.x : 1.0f;
      acc += o.x * 0.00013f + o.y * 0.00017f + o.z * 0.00019f + d.x * 0.00023f + d.y * 0.00029f +
             d.z * 0.00031f + (float)(idx & 7) * 0.0000001f + t * 0.000001f + h.y * 0.000073f;
    }
  }
  out[tid] = acc;
}

using Kernel = void (*)(const CalData, int, int, int, int, float*);
const Kernel kKernels[8] = {k_cost<0>, k_cost<1>, k_cost<2>, k_cost<3>,
                            k_cost<4>, k_cost<5>, k_cost<6>, k_cost<7>};

struct Runner {
  rtb_context* ctx;
  CalData D;
  rtb_calibration_params p;
  float* out;
  cudaStream_t sm;
  cudaError_t err = cudaSuccess;
  bool too_long = false;

  // One timed launch: milliseconds.
  double chunk(int type, int profile, int it0, int iters) {
    cudaEventRecord(ctx->ev0, sm);
    kKernels[type]<<<p.blocks, p.threads, 0, sm>>>(D, profile, it0, iters, p.copies, out);
    cudaEventRecord(ctx->ev1, sm);
    cudaError_t e = cudaEventSynchronize(ctx->ev1);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess && err == cudaSuccess) err = e;
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
    if (ms > p.max_launch_ms) too_long = true;
    return ms;
  }

  // runPair: setup and operation launches alternated; net ns per test.
  double pair(int type, int profile, int repeat) {
    bool setup_first_overall = (repeat & 1) == 0;
    int per = p.iterations / p.sublaunches;
    double setup_ms = 0.0, op_ms = 0.0;
    for (int s = 0; s < p.sublaunches && err == cudaSuccess && !too_long; ++s) {
      int it0 = s * per;
      bool setup_first = ((s & 1) == 0) == setup_first_overall;
      if (setup_first) {
        setup_ms += chunk(0, profile, it0, per);
        op_ms += chunk(type, profile, it0, per);
      } else {
        op_ms += chunk(type, profile, it0, per);
        setup_ms += chunk(0, profile, it0, per);
      }
    }
    double tests = (double)p.blocks * p.threads * (double)per * p.sublaunches * p.copies;
    return (op_ms - setup_ms) * 1.0e6 / tests;
  }
};

double median(std::vector<double> v) {
  std::sort(v.begin(), v.end());
  size_t m = v.size() / 2;
  return v.size() % 2 ? v[m] : 0.5 * (v[m - 1] + v[m]);
}

}  // namespace
}  // namespace rtb

using namespace rtb;

rtb_status rtb_calibrate_costs(rtb_context* ctx, const rtb_calibration_workload* w,
                               const rtb_calibration_params* params, rtb_calibration_result* res) {
  if (!ctx || !w || !params || !res) return RTB_ERR_INVALID_ARGUMENT;
  std::lock_guard<std::mutex> lock(ctx->mu);
  cudaSetDevice(ctx->device);
  ctx->last_error.clear();
  rtb_calibration_params p = *params;
  int R = w->records;
  if (R < 1 || (R & (R - 1)) != 0 || R > (1 << 24) || !w->rays || !w->spheres || !w->boxes ||
      !w->affines || !w->planes || !w->nodes)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "calibration workload: records must be a power of two");
  if (w->profiles < 1 || w->profiles > RTB_CALIBRATION_MAX_PROFILES)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "calibration workload: 1..3 ray profiles");
  if (p.blocks < 1 || p.threads < 32 || p.threads > 256 || p.iterations < 1 || p.copies < 1 ||
      p.sublaunches < 1 || p.iterations % p.sublaunches != 0 || p.repeats < 1 || p.warmups < 0 ||
      !(p.max_launch_ms > 0.0))
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "calibration parameters out of range");
  cudaStream_t sm = ctx->stream;
  ctx_acquire(ctx, sm);
  size_t rays_b = (size_t)w->profiles * R * 6 * 4, sph_b = (size_t)R * 16, box_b = (size_t)R * 32,
         aff_b = (size_t)R * 48, pl_b = (size_t)R * 16, nd_b = (size_t)R * 64,
         out_b = (size_t)p.blocks * p.threads * 4;
  char* buf = nullptr;
  size_t total = rays_b + sph_b + box_b + aff_b + pl_b + nd_b + out_b + 7 * 256;
  cudaError_t e = cudaMallocAsync((void**)&buf, total, sm);
  if (e != cudaSuccess) {
    ctx_release(ctx, sm);
    return cuda_fail(ctx, e, "calibration workload");
  }
  size_t off = 0;
  auto take = [&](size_t b) {
    char* q = buf + off;
    off = (off + b + 255) & ~size_t(255);
    return q;
  };
  CalData D;
  float* d_rays = (float*)take(rays_b);
  float4* d_sph = (float4*)take(sph_b);
  float4* d_box = (float4*)take(box_b);
  float4* d_aff = (float4*)take(aff_b);
  float4* d_pl = (float4*)take(pl_b);
  float4* d_nd = (float4*)take(nd_b);
  float* d_out = (float*)take(out_b);
  cudaMemcpyAsync(d_rays, w->rays, rays_b, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(d_sph, w->spheres, sph_b, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(d_box, w->boxes, box_b, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(d_aff, w->affines, aff_b, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(d_pl, w->planes, pl_b, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(d_nd, w->nodes, nd_b, cudaMemcpyHostToDevice, sm);
  D.rays = d_rays;
  D.spheres = d_sph;
  D.boxes = d_box;
  D.affines = d_aff;
  D.planes = d_pl;
  D.nodes = d_nd;
  D.records = R;

  Runner run{ctx, D, p, d_out, sm};
  *res = rtb_calibration_result{};
  res->profiles = w->profiles;
  std::vector<double> ratios[8];
  // PrimitiveCostBenchmark.operationOrder: a rotation of the operations per context
  int order[7];
  for (int k = 0; k < 7; ++k) order[k] = 1 + (k + p.order_offset % 7 + 7) % 7;
  for (int prof = 0; prof < w->profiles && run.err == cudaSuccess && !run.too_long; ++prof) {
    std::vector<double> sphere_all;
    for (int k = 0; k < 7 && run.err == cudaSuccess && !run.too_long; ++k) {
      int type = order[k];
      for (int r = 0; r < p.warmups; ++r) {
        run.pair(type, prof, r);
        run.pair(1, prof, r + 1);
      }
      std::vector<double> op_net, sphere_net;
      for (int r = 0; r < p.repeats; ++r) {
        bool op_first = (r & 1) == 0;
        double a, s;
        if (op_first) {
          a = run.pair(type, prof, r);
          s = run.pair(1, prof, r + 1);
        } else {
          s = run.pair(1, prof, r + 1);
          a = run.pair(type, prof, r);
        }
        op_net.push_back(a);
        sphere_net.push_back(s);
        sphere_all.push_back(s);
      }
      double net = median(op_net), local = median(sphere_net);
      res->net_ns[prof][type] = net;
      res->sphere_ns[prof][type] = local;
      res->ratio[prof][type] = type == 1 ? 1.0 : net / local;
      ratios[type].push_back(res->ratio[prof][type]);
    }
    res->net_ns[prof][0] = 0.0;
    res->sphere_net_ns[prof] = median(sphere_all);
  }
  cudaFreeAsync(buf, sm);
  cudaError_t e2 = cudaStreamSynchronize(sm);
  ctx_release(ctx, sm);
  if (run.err != cudaSuccess) return cuda_fail(ctx, run.err, "calibration launch");
  if (e2 != cudaSuccess) return cuda_fail(ctx, e2, "calibration");
  if (run.too_long) return fail(ctx, RTB_ERR_LIMIT, "a calibration launch exceeded max_launch_ms");
  for (int t = 1; t < 8; ++t) {
    res->weight[t] = median(ratios[t]);
    if (!(res->weight[t] > 0.0) || !std::isfinite(res->weight[t]))
      return fail(ctx, RTB_ERR_DEVICE_CHECK, "calibration produced a non-positive operation cost");
  }
  res->weight[0] = 0.0;
  res->tests_per_observation =
      (long long)p.blocks * p.threads * (long long)p.iterations * p.copies;
  return RTB_OK;
}
