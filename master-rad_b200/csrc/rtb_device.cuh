// Device-side scene layout, primitive intersection and BVH traversal for sm_100a.
//
// HBM layout of a resident scene (built by rtb_scene.cu):
//   nodes      4 x float4 per node (64 B, 64-B aligned): the bounds of BOTH children,
//              so one node fetch tests two boxes:
//                n0 = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//                n1 = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//                n2 = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//                n3 = (link0, link1, leaf0, leaf1)  as ints
//              link >= 0: interior child node index.  link < 0: leaf with first
//              reference ~link; leafN = count | (type code << 24), code 0..3 = the
//              homogeneous primitive type, 4 = mixed.  Node 0 is a synthetic top node whose
//              children are the reference's roots (unused slots have empty bounds).
//   refs       int per leaf reference: type << 30 | index into that type's arrays.
//              Each type's records are stored in the order its references first appear
//              in leaf order, so the records of a leaf are adjacent in memory.
//   spheres    float4 (centre, radius)                                        16 B
//   boxes      2 x float4 (min.xyz, max.xyz)                                  32 B
//   affines    3 x float4 rows (inverse linear row, world centre component)   48 B
//              plus the 9-float normal matrix and material, read only for the final hit
//   planes     float4 (unit normal, offset) + the reference's 26-float record for the
//              (rare) grid material choice
//   materials  4 x float4 (diffuse+ior, reflective, refractive, emittance)    64 B
//   orig       per type: storage index -> insertion index (global order = type base +
//              insertion index; it breaks equal-distance ties exactly as the reference).
//
// Arithmetic contract: the primitive tests and the path-shading code restate the
// reference kernel (gfxlab/gpu/GpuKernelSources.java, K:lines below) operation for
// operation.  The library is compiled with -fmad=false, so a*b+c is never contracted;
// fmaf() appears exactly where the reference calls fmaf.  Hit distances, primitive ids
// and normals are therefore bit-identical to the reference kernel built without
// contraction.  Node tests are this library's own (reciprocal slab test with widened
// bounds); pruning is conservative, so the closest hit -- the lexicographic minimum of
// (distance, global order) over all primitives -- does not depend on the tree layout.
#pragma once
#include <cuda_runtime.h>
#include <math_constants.h>
#include <stdint.h>

namespace rtb {

constexpr float kEps = 1e-4f;          // K:12
constexpr int kTypeShift = 30;
constexpr int kIndexMask = 0x3FFFFFFF;  // K:20
constexpr int kStackSize = 64;          // covers every tree depth the builders produce
// Leaf tests wait until at most this many lanes of the warp can still walk the tree
// (measured on the 10k and 1M scenes: 4 was best of 0/2/4/8/12/16).
#ifndef RTB_LEAF_POSTPONE_LANES
#define RTB_LEAF_POSTPONE_LANES 4
#endif
constexpr int kLeafPostponeLanes = RTB_LEAF_POSTPONE_LANES;

enum PrimType { kSphere = 0, kBox = 1, kAffineSphere = 2, kAffineBox = 3, kPlane = 4 };

struct DevScene {
  const float4* nodes;
  int node_count;
  const int* refs;
  int ref_count;
  const float4* spheres;
  const float4* boxes;
  const float4* aspheres;
  const float4* aboxes;
  const float* asphere_nm;  // 9 floats per record
  const float* abox_nm;
  const int* mat[4];        // material index per storage record, per type
  const int* orig[4];       // insertion index per storage record, per type
  int count[4];             // spheres, boxes, affine spheres, affine boxes
  int order_base[5];        // global order of the first record of each type (planes last)
  const float4* planes;     // unit normal + offset
  const float* plane_full;  // reference 26-float records
  int plane_count;
  const float4* materials;  // 4 float4 per material
  int material_count;
  float3 background;
  int use_bvh;
};

// ---------------------------------------------------------------- vector helpers (K:45-118)
__device__ __forceinline__ float3 v3(float x, float y, float z) { return make_float3(x, y, z); }
__device__ __forceinline__ float3 add(float3 a, float3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ float3 sub(float3 a, float3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ float3 neg(float3 v) { return v3(-v.x, -v.y, -v.z); }
__device__ __forceinline__ float3 mul(float3 v, float s) { return v3(v.x * s, v.y * s, v.z * s); }
__device__ __forceinline__ float3 mulv(float3 a, float3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ float3 divs(float3 v, float s) {
  float inv = 1.0f / s;
  return v3(v.x * inv, v.y * inv, v.z * inv);
}
__device__ __forceinline__ float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ float3 normalize_safe(float3 v) {  // K:96-99
  float len = sqrtf(fmaxf(dot(v, v), 1e-20f));
  return divs(v, len);
}
__device__ __forceinline__ float3 normalize_transformed(float3 v) {  // K:101-110
  float l2 = dot(v, v);
  if (l2 >= 1.0e-20f && isfinite(l2)) return divs(v, sqrtf(l2));
  float scale = fmaxf(fabsf(v.x), fmaxf(fabsf(v.y), fabsf(v.z)));
  if (!(scale > 0.0f) || !isfinite(scale)) return v3(0.0f, 0.0f, 0.0f);
  float3 s = v3(v.x / scale, v.y / scale, v.z / scale);
  return divs(s, sqrtf(dot(s, s)));
}

// ---------------------------------------------------------------- RNG (K:165-179)
// Host abort words, three ints in device memory owned by the context:
//   [0] the abort generation, raised by rtb_request_abort;
//   [1] the generation that was current when the running work was submitted, written in
//       stream order just before it (kernel argument of k_arm_abort, so a later abort
//       request can never be overwritten by it);
//   [2] set to 1 by a kernel that stopped fetching work because of an abort.
// A persistent kernel calls abort_raised() before each work fetch.
__device__ __forceinline__ bool abort_raised(int* w) {
  if (*(volatile int*)w == *(volatile int*)(w + 1)) return false;
  *(volatile int*)(w + 2) = 1;
  return true;
}
__device__ __forceinline__ bool abort_stopped(const int* w) { return *(volatile const int*)(w + 2) != 0; }

__device__ __forceinline__ uint32_t hash_u32(uint32_t x) {
  x ^= x >> 17;
  x *= 0xed5ad4bbU;
  x ^= x >> 11;
  x *= 0xac4c1b51U;
  x ^= x >> 15;
  x *= 0x31848babU;
  x ^= x >> 14;
  return x;
}
__device__ __forceinline__ float rand01(uint32_t* s) {
  *s = hash_u32(*s + 0x9e3779b9U);
  return (*s >> 8) * 0x1p-24f;
}

// ---------------------------------------------------------------- primitive tests
// Each test returns the hit distance, or +inf for no hit beyond kEps.  With NORMAL set it
// also produces the surface normal the reference stores for that hit.

// traceSphere, K:338-399.
template <bool NORMAL>
__device__ __forceinline__ float sphere_test(float4 s, float3 o, float3 d, float a, float3* n) {
  float3 oc = sub(o, v3(s.x, s.y, s.z));
  float b = dot(oc, d);
  float center_t = -b / a;
  float3 cl = v3(fmaf(d.x, center_t, oc.x), fmaf(d.y, center_t, oc.y), fmaf(d.z, center_t, oc.z));
  float corr = -dot(cl, d) / a;
  center_t += corr;
  cl = v3(fmaf(d.x, corr, cl.x), fmaf(d.y, corr, cl.y), fmaf(d.z, corr, cl.z));
  float radial_sq = fmaf(s.w, s.w, -dot(cl, cl));
  if (radial_sq <= 0.0f) return CUDART_INF_F;
  float half = sqrtf(radial_sq / a);
  float t1 = center_t - half;
  float t2 = center_t + half;
  float t, roff;
  if (t1 > kEps) {
    t = t1;
    roff = -half;
  } else if (t2 > kEps) {
    t = t2;
    roff = half;
  } else {
    return CUDART_INF_F;
  }
  if (NORMAL) {
    float3 radial = v3(fmaf(d.x, roff, cl.x), fmaf(d.y, roff, cl.y), fmaf(d.z, roff, cl.z));
    *n = normalize_safe(radial);
  }
  return t;
}

// Shared slab logic of traceBox (K:588-706) and traceAffineBox (K:463-586).
template <bool NORMAL>
__device__ __forceinline__ float slab_test(float3 o, float3 d, float3 bmin, float3 bmax,
                                           float after, int* axis_out, float* sign_out) {
  float txmin, txmax, tymin, tymax, tzmin, tzmax;
  if (d.x == 0.0f) {
    if (o.x < bmin.x || o.x > bmax.x) return CUDART_INF_F;
    txmin = -CUDART_INF_F;
    txmax = CUDART_INF_F;
  } else {
    float t1 = (bmin.x - o.x) / d.x;
    float t2 = (bmax.x - o.x) / d.x;
    txmin = fminf(t1, t2);
    txmax = fmaxf(t1, t2);
  }
  if (d.y == 0.0f) {
    if (o.y < bmin.y || o.y > bmax.y) return CUDART_INF_F;
    tymin = -CUDART_INF_F;
    tymax = CUDART_INF_F;
  } else {
    float t1 = (bmin.y - o.y) / d.y;
    float t2 = (bmax.y - o.y) / d.y;
    tymin = fminf(t1, t2);
    tymax = fmaxf(t1, t2);
  }
  if (d.z == 0.0f) {
    if (o.z < bmin.z || o.z > bmax.z) return CUDART_INF_F;
    tzmin = -CUDART_INF_F;
    tzmax = CUDART_INF_F;
  } else {
    float t1 = (bmin.z - o.z) / d.z;
    float t2 = (bmax.z - o.z) / d.z;
    tzmin = fminf(t1, t2);
    tzmax = fmaxf(t1, t2);
  }
  float tenter = fmaxf(fmaxf(txmin, tymin), tzmin);
  float texit = fminf(fminf(txmax, tymax), tzmax);
  if (tenter >= texit || texit <= after) return CUDART_INF_F;
  if (tenter > after) {
    if (NORMAL) {
      int ae = 0;
      float ev = txmin;
      if (tymin > ev) {
        ev = tymin;
        ae = 1;
      }
      if (tzmin > ev) ae = 2;
      float dc = ae == 0 ? d.x : (ae == 1 ? d.y : d.z);
      *axis_out = ae;
      *sign_out = dc > 0.0f ? -1.0f : 1.0f;
    }
    return tenter;
  }
  if (NORMAL) {
    int ax = 0;
    float xv = txmax;
    if (tymax < xv) {
      xv = tymax;
      ax = 1;
    }
    if (tzmax < xv) ax = 2;
    float dc = ax == 0 ? d.x : (ax == 1 ? d.y : d.z);
    *axis_out = ax;
    *sign_out = dc >= 0.0f ? 1.0f : -1.0f;
  }
  return texit;
}

__device__ __forceinline__ float3 axis_normal(int axis, float sign) {
  return axis == 0 ? v3(sign, 0.0f, 0.0f) : (axis == 1 ? v3(0.0f, sign, 0.0f) : v3(0.0f, 0.0f, sign));
}

template <bool NORMAL>
__device__ __forceinline__ float box_test(float4 lo, float4 hi, float3 o, float3 d, float3* n) {
  int axis = 0;
  float sign = 0.0f;
  float t = slab_test<NORMAL>(o, d, v3(lo.x, lo.y, lo.z), v3(hi.x, hi.y, hi.z), kEps, &axis, &sign);
  if (NORMAL && t != CUDART_INF_F) *n = axis_normal(axis, sign);
  return t;
}

// affineRayShift / applyAffineShiftedPoint / applyAffineVector, K:276-301.  Rows r0..r2
// hold the inverse linear map with the world centre in .w.
struct AffineRay {
  float shift;
  float3 lo, ld;
};
__device__ __forceinline__ AffineRay affine_ray(float4 r0, float4 r1, float4 r2, float3 o, float3 d,
                                                float dd) {
  AffineRay a;
  float3 c = v3(r0.w, r1.w, r2.w);
  a.shift = dd > 0.0f ? fmaxf(0.0f, dot(sub(c, o), d) / dd) : 0.0f;
  float3 rel = v3(fmaf(d.x, a.shift, o.x - r0.w), fmaf(d.y, a.shift, o.y - r1.w),
                  fmaf(d.z, a.shift, o.z - r2.w));
  a.lo = v3(r0.x * rel.x + r0.y * rel.y + r0.z * rel.z, r1.x * rel.x + r1.y * rel.y + r1.z * rel.z,
            r2.x * rel.x + r2.y * rel.y + r2.z * rel.z);
  a.ld = v3(r0.x * d.x + r0.y * d.y + r0.z * d.z, r1.x * d.x + r1.y * d.y + r1.z * d.z,
            r2.x * d.x + r2.y * d.y + r2.z * d.z);
  return a;
}

__device__ __forceinline__ float3 linear9(const float* m, float3 v) {  // K:303-309
  return v3(m[0] * v.x + m[1] * v.y + m[2] * v.z, m[3] * v.x + m[4] * v.y + m[5] * v.z,
            m[6] * v.x + m[7] * v.y + m[8] * v.z);
}

// traceAffineSphere, K:401-461 (normalizedDirection K:317-336 for degenerate local rays).
template <bool NORMAL>
__device__ __forceinline__ float affine_sphere_local(const AffineRay& ar, const float* nm, float3* n);

template <bool NORMAL>
__device__ __forceinline__ float affine_sphere_test(float4 r0, float4 r1, float4 r2, float3 o,
                                                    float3 d, float dd, const float* nm,
                                                    float3* n) {
  return affine_sphere_local<NORMAL>(affine_ray(r0, r1, r2, o, d, dd), nm, n);
}

// normalizedDirection (K:317-336) for a local direction whose squared length is not a
// positive finite float: the unit direction and the scale back to the mapped parameter.
// Out of line: rare, and kept out of the leaf test's code.  False when no direction exists.
static __device__ __noinline__ bool degenerate_local_direction(float3 dir, float3* sd, float* pscale) {
  float l2 = dot(dir, dir);
  if (isfinite(l2) && fabsf(l2 - 1.0f) <= 2.0e-6f) {
    *sd = dir;
    *pscale = 1.0f;
    return true;
  }
  float scale = fmaxf(fabsf(dir.x), fmaxf(fabsf(dir.y), fabsf(dir.z)));
  if (!(scale > 0.0f) || !isfinite(scale)) return false;
  float3 sc = v3(dir.x / scale, dir.y / scale, dir.z / scale);
  float sl = sqrtf(dot(sc, sc));
  float dl = scale * sl;
  float inv = 1.0f / dl;
  if (!(inv > 0.0f) || !isfinite(inv)) return false;
  *sd = mul(sc, 1.0f / sl);
  *pscale = inv;
  return true;
}

// The unit-sphere part of traceAffineSphere on the mapped ray.
template <bool NORMAL>
__device__ __forceinline__ float affine_sphere_local(const AffineRay& ar, const float* nm, float3* n) {
  float after_local = kEps - ar.shift;
  float solve_a = dot(ar.ld, ar.ld);
  float3 sd = ar.ld;
  float pscale = 1.0f;
  if (!(solve_a > 0.0f) || !isfinite(solve_a)) {
    if (!degenerate_local_direction(ar.ld, &sd, &pscale)) return CUDART_INF_F;
    solve_a = 1.0f;
  }
  float scaled_after = after_local / pscale;
  float center_t = -dot(ar.lo, sd) / solve_a;
  float3 cl = add(ar.lo, mul(sd, center_t));
  float radial_sq = fmaf(-cl.x, cl.x, fmaf(-cl.y, cl.y, fmaf(-cl.z, cl.z, 1.0f)));
  if (radial_sq <= 0.0f) return CUDART_INF_F;
  float half = sqrtf(radial_sq / solve_a);
  float t1 = center_t - half;
  float t2 = center_t + half;
  float sh;
  if (t1 > scaled_after)
    sh = t1;
  else if (t2 > scaled_after)
    sh = t2;
  else
    return CUDART_INF_F;
  float hit_t = sh * pscale;
  float world_t = ar.shift + hit_t;
  if (NORMAL) {
    float3 lh = add(ar.lo, mul(ar.ld, hit_t));
    *n = normalize_transformed(linear9(nm, lh));
  }
  return world_t;
}

// traceAffineBox, K:463-586.
template <bool NORMAL>
__device__ __forceinline__ float affine_box_local(const AffineRay& ar, const float* nm, float3* n);

template <bool NORMAL>
__device__ __forceinline__ float affine_box_test(float4 r0, float4 r1, float4 r2, float3 o, float3 d,
                                                 float dd, const float* nm, float3* n) {
  return affine_box_local<NORMAL>(affine_ray(r0, r1, r2, o, d, dd), nm, n);
}

// The unit-box part of traceAffineBox on the mapped ray.
template <bool NORMAL>
__device__ __forceinline__ float affine_box_local(const AffineRay& ar, const float* nm, float3* n) {
  float after_local = kEps - ar.shift;
  int axis = 0;
  float sign = 0.0f;
  float t = slab_test<NORMAL>(ar.lo, ar.ld, v3(-1.0f, -1.0f, -1.0f), v3(1.0f, 1.0f, 1.0f),
                              after_local, &axis, &sign);
  if (t == CUDART_INF_F) return t;
  float world_t = ar.shift + t;
  if (NORMAL) *n = normalize_transformed(linear9(nm, axis_normal(axis, sign)));
  return world_t;
}

// ---------------------------------------------------------------- closest hit
struct Best {
  float t;
  int order;
  int type;   // PrimType of the winner, -1 for none
  int index;  // storage index of the winner (plane index for planes)
};

__device__ __forceinline__ int order_of(const DevScene& S, int type, int index) {
  return S.order_base[type] + __ldg(S.orig[type] + index);
}

// Offers a candidate distance: the closest hit is the lexicographic minimum of
// (distance, global order), the contract of tracePrimitiveRef (K:772-806).
__device__ __forceinline__ void offer(const DevScene& S, Best& b, float t, int type, int index) {
  if (t < b.t) {
    b.t = t;
    b.type = type;
    b.index = index;
    b.order = order_of(S, type, index);
  } else if (t == b.t && t != CUDART_INF_F) {
    int o = order_of(S, type, index);
    if (o < b.order) {
      b.order = o;
      b.type = type;
      b.index = index;
    }
  }
}

struct TraceCounters {
  unsigned long long aabb, prim, type[5], internal, leaf, homo, mixed, maxstack, overflow;
};

template <bool METRICS>
__device__ __forceinline__ void test_ref(const DevScene& S, int type, int idx, float3 o, float3 d,
                                         float dd, Best& b, TraceCounters* c) {
  float t;
  float3 dummy;
  if (type == kSphere) {
    t = sphere_test<false>(__ldg(S.spheres + idx), o, d, dd, &dummy);
  } else {
    // boxes and affine boxes share one slab test, both affine types one ray mapping
    float3 so = o, sd = d, smin, smax;
    float after = kEps, shift = 0.0f;
    bool slab = true;
    if (type == kBox) {
      float4 lo = __ldg(S.boxes + 2 * idx), hi = __ldg(S.boxes + 2 * idx + 1);
      smin = v3(lo.x, lo.y, lo.z);
      smax = v3(hi.x, hi.y, hi.z);
    } else {
      const float4* r = (type == kAffineSphere ? S.aspheres : S.aboxes) + 3 * idx;
      AffineRay ar = affine_ray(__ldg(r), __ldg(r + 1), __ldg(r + 2), o, d, dd);
      if (type == kAffineSphere) {
        t = affine_sphere_local<false>(ar, nullptr, &dummy);
        slab = false;
      } else {
        so = ar.lo;
        sd = ar.ld;
        smin = v3(-1.0f, -1.0f, -1.0f);
        smax = v3(1.0f, 1.0f, 1.0f);
        after = kEps - ar.shift;
        shift = ar.shift;
      }
    }
    if (slab) {
      int axis = 0;
      float sign = 0.0f;
      float ts = slab_test<false>(so, sd, smin, smax, after, &axis, &sign);
      t = (type == kBox || ts == CUDART_INF_F) ? ts : shift + ts;
    }
  }
  if (METRICS) {
    c->prim++;
    c->type[type == kSphere ? 0 : type == kBox ? 1 : type == kAffineSphere ? 3 : 4]++;
  }
  offer(S, b, t, type, idx);
}

// Child-box entry distance for the node test.  (lo - o) * inv carries at most ~3 ulp
// relative error; far distances are widened by 2^-20 relative so that a box the exact
// ray touches is never culled (the reference widens by 1.00000072, K:764).
__device__ __forceinline__ float child_entry(float lox, float hix, float loy, float hiy, float loz,
                                             float hiz, float3 o, float3 inv, float limit) {
  float t0x = (lox - o.x) * inv.x, t1x = (hix - o.x) * inv.x;
  float t0y = (loy - o.y) * inv.y, t1y = (hiy - o.y) * inv.y;
  float t0z = (loz - o.z) * inv.z, t1z = (hiz - o.z) * inv.z;
  float tn = fmaxf(fmaxf(fminf(t0x, t1x), fminf(t0y, t1y)), fmaxf(fminf(t0z, t1z), kEps));
  float tf = fminf(fminf(fmaxf(t0x, t1x), fmaxf(t0y, t1y)), fmaxf(t0z, t1z));
  tf = tf * 1.00000095367431640625f;  // 1 + 2^-20
  tf = fminf(tf, limit);
  return tn <= tf ? tn : CUDART_INF_F;
}

// Conservative prune limit for the current best distance, K:746-748 / 889-891.
__device__ __forceinline__ float prune_limit(float t) {
  return isfinite(t) ? fmaf(t, 1.0000015f, 1.0e-6f) : t;
}

template <bool METRICS>
__device__ __noinline__ void test_all_refs(const DevScene& S, float3 o, float3 d, float dd, Best& b,
                                           TraceCounters* c) {
  for (int i = 0; i < S.ref_count; ++i) {
    int ref = __ldg(S.refs + i);
    test_ref<METRICS>(S, (int)((unsigned)ref >> kTypeShift), ref & kIndexMask, o, d, dd, b, c);
  }
}

template <bool METRICS>
__device__ __noinline__ void test_all_primitives(const DevScene& S, float3 o, float3 d, float dd,
                                                 Best& b, TraceCounters* c) {
  for (int t = 0; t < 4; ++t)
    for (int i = 0; i < S.count[t]; ++i) test_ref<METRICS>(S, t, i, o, d, dd, b, c);
}

// Closest hit of one ray against the resident scene (traceClosest, K:963-1020): the BVH
// (or every bounded primitive in linear mode), then the planes.  Returns true on a hit.
//
// Warp-cooperative: all 32 lanes of the warp call it together (lanes without a ray pass
// active = false).  The traversal loop is warp-uniform -- each iteration every lane that
// still walks processes one node: it tests both child boxes, records the leaf children it
// reached (a lane holds up to two recorded pairs, walking on after the first), then picks
// the next interior node; once at most kLeafPostponeLanes lanes can still walk, the
// recorded leaves of all lanes are tested together -- and the loop condition is a warp
// vote, so divergent lanes reconverge once per node.  Every lane
// takes part in the votes, also where lanes hold different scenes and only some of them
// have a tree (the batch kernel's lanes may belong to different jobs).
//
// SDEPTH > 0: the first SDEPTH stack entries live in shared memory, in the caller's column
// `ss` of an [SDEPTH][SSTRIDE] int2 array (node, entry distance bits), so that the entries
// a traversal uses most stay out of local memory; deeper entries spill to local memory.
template <bool METRICS, int SDEPTH = 0, int SSTRIDE = 1>
__device__ bool trace_closest(const DevScene& S, float3 o, float3 d, bool active, Best& b,
                              TraceCounters* c, int* overflow_flag, int2* ss = nullptr) {
  b.t = 1e30f;
  b.order = 0x7FFFFFFF;
  b.type = -1;
  b.index = -1;
  float dd = dot(d, d);
  const bool bvh = S.use_bvh && S.node_count > 0;
  {
    float3 inv = v3(d.x != 0.0f ? 1.0f / d.x : 1e30f, d.y != 0.0f ? 1.0f / d.y : 1e30f,
                    d.z != 0.0f ? 1.0f / d.z : 1e30f);
    int stack[kStackSize - SDEPTH];
    float estack[kStackSize - SDEPTH];
    int sp = 0;
    int node = (active && bvh) ? 0 : -1;
    bool overflow = false;
    // A tree visits each node at most once per ray; the cap only matters for malformed
    // (cyclic) caller-supplied trees, which then take the exhaustive path.
    int budget = S.node_count + 8;
    // Leaf postponing with speculative walking: a lane that reaches leaf children records
    // them and walks on to its next leaf children (two recorded pairs at most, then it
    // waits); the warp tests the recorded leaves together once at most kLeafPostponeLanes
    // lanes can still walk, so the expensive primitive tests run with many lanes at once.
    // The prune limits a lane uses while its leaves wait are from its older (farther) best
    // hit, which only visits more nodes, never fewer: the closest hit is unchanged.
    int pfirst0 = 0, pmeta0 = 0, pfirst1 = 0, pmeta1 = 0;
    int qfirst0 = 0, qmeta0 = 0, qfirst1 = 0, qmeta1 = 0;
    int npend = 0;
    bool pend = false;  // this lane cannot take another leaf pair
    while (true) {
      pend = npend >= 2;
      // lanes that can walk, lanes with recorded leaves (a lane that cannot walk has some)
      const unsigned walk = __ballot_sync(0xFFFFFFFFu, node >= 0 && !pend);
      const unsigned waiting = __ballot_sync(0xFFFFFFFFu, npend > 0);
      if ((walk | waiting) == 0u) break;
      if (__popc(walk) <= kLeafPostponeLanes && waiting != 0u) {
        int c0 = npend >= 1 ? (pmeta0 & 0xFFFFFF) : 0, c1 = npend >= 1 ? (pmeta1 & 0xFFFFFF) : 0;
        int c2 = npend >= 2 ? (qmeta0 & 0xFFFFFF) : 0, c3 = npend >= 2 ? (qmeta1 & 0xFFFFFF) : 0;
        int e1 = c0 + c1, e2 = e1 + c2, e3 = e2 + c3;
        for (int k = 0; k < e3; ++k) {
          int first, meta, off;
          if (k < c0) {
            first = pfirst0, meta = pmeta0, off = k;
          } else if (k < e1) {
            first = pfirst1, meta = pmeta1, off = k - c0;
          } else if (k < e2) {
            first = qfirst0, meta = qmeta0, off = k - e1;
          } else {
            first = qfirst1, meta = qmeta1, off = k - e2;
          }
          int code = meta >> 24;
          int ref = __ldg(S.refs + first + off);
          int type = code == 4 ? (int)((unsigned)ref >> kTypeShift) : code;
          test_ref<METRICS>(S, type, ref & kIndexMask, o, d, dd, b, c);
        }
        npend = 0;
        continue;
      }
      if (node >= 0 && !pend) {
        const float4* np = S.nodes + 4 * node;
        float4 n0 = __ldg(np), n1 = __ldg(np + 1), n2 = __ldg(np + 2);
        int4 n3 = __ldg(reinterpret_cast<const int4*>(np + 3));
        float lim = prune_limit(b.t);
        float e0 = child_entry(n0.x, n0.y, n0.z, n0.w, n2.x, n2.y, o, inv, lim);
        float e1 = child_entry(n1.x, n1.y, n1.z, n1.w, n2.z, n2.w, o, inv, lim);
        if (METRICS) {
          c->internal++;
          c->aabb += 2;
        }
        bool swap = e1 < e0;
        float en = swap ? e1 : e0, ef = swap ? e0 : e1;
        int ln = swap ? n3.y : n3.x, lf = swap ? n3.x : n3.y;
        int mn = swap ? n3.w : n3.z, mf = swap ? n3.z : n3.w;
        bool hn = en != CUDART_INF_F, hf = ef != CUDART_INF_F;
        // Leaf children: one loop over the near leaf's references then the far leaf's.
        // Testing the far leaf even if the near one already beats it is harmless: the
        // closest hit is a minimum over primitives.
        int first0 = (hn && ln < 0) ? ~ln : 0, count0 = (hn && ln < 0) ? (mn & 0xFFFFFF) : 0;
        int first1 = (hf && lf < 0) ? ~lf : 0, count1 = (hf && lf < 0) ? (mf & 0xFFFFFF) : 0;
        int code0 = mn >> 24, code1 = mf >> 24;
        if (METRICS) {
          if (count0 || (hn && ln < 0)) {
            c->leaf++;
            if (code0 == 4) c->mixed++; else c->homo++;
          }
          if (count1 || (hf && lf < 0)) {
            c->leaf++;
            if (code1 == 4) c->mixed++; else c->homo++;
          }
        }
        if (count0 + count1 > 0) {
          if (npend == 0) {
            pfirst0 = first0;
            pmeta0 = count0 | (code0 << 24);
            pfirst1 = first1;
            pmeta1 = count1 | (code1 << 24);
          } else {
            qfirst0 = first0;
            qmeta0 = count0 | (code0 << 24);
            qfirst1 = first1;
            qmeta1 = count1 | (code1 << 24);
          }
          npend++;
        }
        float plim = prune_limit(b.t);
        int next = (hn && ln >= 0) ? ln : -1;
        if (hf && lf >= 0 && ef <= plim) {
          if (next < 0) {
            next = lf;
          } else if (sp < kStackSize) {
            if (SDEPTH > 0 && sp < SDEPTH) {
              ss[sp * SSTRIDE] = make_int2(lf, __float_as_int(ef));
            } else {
              stack[sp - SDEPTH] = lf;
              estack[sp - SDEPTH] = ef;
            }
            sp++;
            if (METRICS && (unsigned long long)sp > c->maxstack) c->maxstack = sp;
          } else {
            overflow = true;
          }
        }
        // Pop the next subtree still closer than the current hit.
        while (next < 0 && sp > 0) {
          --sp;
          int sn;
          float se;
          if (SDEPTH > 0 && sp < SDEPTH) {
            int2 e = ss[sp * SSTRIDE];
            sn = e.x;
            se = __int_as_float(e.y);
          } else {
            sn = stack[sp - SDEPTH];
            se = estack[sp - SDEPTH];
          }
          if (se <= plim) next = sn;
        }
        if (--budget < 0) overflow = true;
        node = overflow ? -1 : next;
      }
    }
    if (overflow) {
      if (overflow_flag) atomicAdd(overflow_flag, 1);
      if (METRICS) c->overflow++;
      test_all_refs<METRICS>(S, o, d, dd, b, c);
    }
  }
  if (active && !bvh) test_all_primitives<METRICS>(S, o, d, dd, b, c);
  if (!active) return false;
  // tracePlane, K:708-734: a plane wins only when strictly closer.
  for (int i = 0; i < S.plane_count; ++i) {
    float4 p = __ldg(S.planes + i);
    float3 pn = v3(p.x, p.y, p.z);
    float den = dot(pn, d);
    if (den == 0.0f) continue;
    float t = -(dot(pn, o) + p.w) / den;
    if (t <= kEps || t >= b.t) continue;
    b.t = t;
    b.type = kPlane;
    b.index = i;
    b.order = S.order_base[kPlane] + i;
  }
  if (METRICS) {
    c->prim += S.plane_count;
    c->type[2] += S.plane_count;
  }
  return b.type >= 0;
}

__device__ __forceinline__ float positive_mod(float x, float y) { return x - y * floorf(x / y); }

// choosePlaneMaterialIndex, K:251-269.
__device__ __forceinline__ int plane_material(const float* p, float3 hp) {
  const float* g = p + 18;
  int surface = (int)g[5];
  if (g[0] == 0.0f) return surface;
  float3 rel = sub(hp, v3(p[4], p[5], p[6]));
  float be = dot(rel, v3(p[7], p[8], p[9])) / p[13];
  float bf = dot(rel, v3(p[10], p[11], p[12])) / p[14];
  float u = (be - bf * p[16]) / p[17];
  float v = (bf - be * p[15]) / p[17];
  float hx = g[3] * 0.5f;
  float hy = g[4] * 0.5f;
  float mx = positive_mod(u + hx, g[1]);
  float my = positive_mod(v + hy, g[2]);
  if (mx < g[3] || my < g[4]) return (int)g[7];
  return (int)g[6];
}

// The full hit record of the winner: position o + d t, the reference's normal for that
// primitive type, and its material index.
static __device__ __noinline__ void hit_record(const DevScene& S, const Best& b, float3 o, float3 d,
                                           float3* pos, float3* n, int* material) {
  float dd = dot(d, d);
  *pos = add(o, mul(d, b.t));
  float3 nn = v3(0.0f, 0.0f, 0.0f);
  int m = -1;
  int i = b.index;
  switch (b.type) {
    case kSphere:
      sphere_test<true>(__ldg(S.spheres + i), o, d, dd, &nn);
      m = __ldg(S.mat[kSphere] + i);
      break;
    case kBox:
      box_test<true>(__ldg(S.boxes + 2 * i), __ldg(S.boxes + 2 * i + 1), o, d, &nn);
      m = __ldg(S.mat[kBox] + i);
      break;
    case kAffineSphere: {
      const float4* r = S.aspheres + 3 * i;
      affine_sphere_test<true>(__ldg(r), __ldg(r + 1), __ldg(r + 2), o, d, dd, S.asphere_nm + 9 * i, &nn);
      m = __ldg(S.mat[kAffineSphere] + i);
      break;
    }
    case kAffineBox: {
      const float4* r = S.aboxes + 3 * i;
      affine_box_test<true>(__ldg(r), __ldg(r + 1), __ldg(r + 2), o, d, dd, S.abox_nm + 9 * i, &nn);
      m = __ldg(S.mat[kAffineBox] + i);
      break;
    }
    case kPlane: {
      float4 p = __ldg(S.planes + i);
      nn = v3(p.x, p.y, p.z);
      m = plane_material(S.plane_full + 26 * i, *pos);
      break;
    }
    default:
      break;
  }
  *n = nn;
  *material = m;
}

}  // namespace rtb
