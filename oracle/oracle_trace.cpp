// Oracle (test infrastructure only): a CPU restatement, in IEEE single precision, of the
// reference CUDA path tracer's closest-hit query and camera-sample loop.  Only tests/,
// __graft_entry__.smoke() and bench.py's cpu_baseline leg may load this code.
//
// Restated from gfxlab/gpu/GpuKernelSources.java (K below; gfxlab/ = src/xyz/marsavic/gfxlab/):
//   hash_u32 / rand01             K:165-179
//   normalizeSafe, normalizeTransformedNormal, normalizedDirection   K:96-110, 317-336
//   traceSphere                    K:338-399
//   traceAffineSphere              K:401-461   (affineRayShift / applyAffineShiftedPoint K:276-309)
//   traceAffineBox                 K:463-586
//   traceBox                       K:588-706
//   tracePlane                     K:708-734   (grid material K:214-269)
//   bvhEntryDistance               K:736-770
//   tracePrimitiveRef              K:772-806
//   traceBvhLeaf / traceBvh        K:808-961   (including the brute-force overflow fallback)
//   traceClosest                   K:963-1020
//   tracePath + BSDF helpers       K:1022-1165
//   renderKernel seed/jitter/camera/accumulation   K:1217-1293
//   traceReplayKernel outputs      K:1338-1376
// The arithmetic follows the source expression by expression with no contraction
// (compile with -ffp-contract=off); fmaf is used exactly where the source calls fmaf.
// This matches the reference kernel built with -fmad=false bit for bit on closest-hit
// queries.  Rendering calls the host libm cosf/sinf, which are not CUDA's, so rendered
// images agree with the device only statistically.
#include <cmath>
#include <cstdint>
#include <cstring>

namespace {

constexpr float EPS = 1e-4f;
constexpr int TYPE_MASK = (int)0xC0000000u;
constexpr int INDEX_MASK = 0x3FFFFFFF;
constexpr int T_SPHERE = 0;
constexpr int T_BOX = 0x40000000;
constexpr int T_ASPHERE = (int)0x80000000u;
constexpr int T_ABOX = (int)0xC0000000u;

struct f3 {
  float x, y, z;
};
inline f3 mk(float x, float y, float z) { return f3{x, y, z}; }
inline f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline f3 operator-(f3 v) { return mk(-v.x, -v.y, -v.z); }
inline f3 operator*(f3 v, float s) { return mk(v.x * s, v.y * s, v.z * s); }
inline f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline f3 operator/(f3 v, float s) {
  float inv = 1.0f / s;
  return mk(v.x * inv, v.y * inv, v.z * inv);
}
inline float dot(f3 a, f3 b) {
  float r = a.x * b.x;
  r = r + a.y * b.y;
  r = r + a.z * b.z;
  return r;
}
inline f3 normalize_safe(f3 v) {
  float len = std::sqrt(std::fmax(dot(v, v), 1e-20f));
  return v / len;
}
inline f3 normalize_transformed(f3 v) {
  float l2 = dot(v, v);
  if (l2 >= 1.0e-20f && std::isfinite(l2)) return v / std::sqrt(l2);
  float scale = std::fmax(std::fabs(v.x), std::fmax(std::fabs(v.y), std::fabs(v.z)));
  if (!(scale > 0.0f) || !std::isfinite(scale)) return mk(0, 0, 0);
  f3 s = mk(v.x / scale, v.y / scale, v.z / scale);
  return s / std::sqrt(dot(s, s));
}

struct DirFrame {
  bool valid;
  f3 unit;
  float inv_len;
};
inline DirFrame normalized_direction(f3 d) {
  float l2 = dot(d, d);
  if (std::isfinite(l2) && std::fabs(l2 - 1.0f) <= 2.0e-6f) return {true, d, 1.0f};
  float scale = std::fmax(std::fabs(d.x), std::fmax(std::fabs(d.y), std::fabs(d.z)));
  if (!(scale > 0.0f) || !std::isfinite(scale)) return {false, mk(0, 0, 0), 0.0f};
  f3 s = mk(d.x / scale, d.y / scale, d.z / scale);
  float sl = std::sqrt(dot(s, s));
  float dl = scale * sl;
  float inv = 1.0f / dl;
  if (!(inv > 0.0f) || !std::isfinite(inv)) return {false, mk(0, 0, 0), 0.0f};
  return {true, s * (1.0f / sl), inv};
}

inline uint32_t hash_u32(uint32_t x) {
  x ^= x >> 17;
  x *= 0xed5ad4bbU;
  x ^= x >> 11;
  x *= 0xac4c1b51U;
  x ^= x >> 15;
  x *= 0x31848babU;
  x ^= x >> 14;
  return x;
}
inline float rand01(uint32_t* s) {
  *s = hash_u32(*s + 0x9e3779b9U);
  return (float)(*s >> 8) * 0x1p-24f;
}

struct Hit {
  int hit = 0;
  float t = 0.0f;
  int order = 0;
  int material = -1;
  f3 pos{0, 0, 0};
  f3 normal{0, 0, 0};
};

struct Scene {
  const float* spheres;
  int ns;
  const float* boxes;
  int nb;
  const float* planes;
  int np;
  const float* aspheres;
  int nas;
  const float* aboxes;
  int nab;
  const float* materials;
  int nm;
  const float* node_bounds;
  const int* node_data;
  int node_count;
  const int* refs;
  int ref_count;
  const int* roots;
  int root_count;
  int use_bvh;
  int stack_size;
};

struct Stats {
  uint64_t v[14];
};

bool trace_sphere(const float* sp, int count, f3 o, f3 d, int base, Hit* h) {
  bool found = false;
  float closest_t = h->t;
  for (int i = 0; i < count; ++i) {
    const float* s = sp + 5 * i;
    f3 c = mk(s[0], s[1], s[2]);
    float radius = s[3];
    int mat = (int)s[4];
    f3 oc = o - c;
    float a = dot(d, d);
    float b = dot(oc, d);
    float center_t = -b / a;
    f3 cl = mk(std::fma(d.x, center_t, oc.x), std::fma(d.y, center_t, oc.y),
               std::fma(d.z, center_t, oc.z));
    float corr = -dot(cl, d) / a;
    center_t = center_t + corr;
    cl = mk(std::fma(d.x, corr, cl.x), std::fma(d.y, corr, cl.y), std::fma(d.z, corr, cl.z));
    float radial_sq = std::fma(radius, radius, -dot(cl, cl));
    if (radial_sq <= 0.0f) continue;
    float half = std::sqrt(radial_sq / a);
    float t1 = center_t - half;
    float t2 = center_t + half;
    float hit_t, roff;
    if (t1 > EPS) {
      hit_t = t1;
      roff = -half;
    } else if (t2 > EPS) {
      hit_t = t2;
      roff = half;
    } else {
      continue;
    }
    if (hit_t < closest_t) {
      closest_t = hit_t;
      h->hit = 1;
      h->t = hit_t;
      h->pos = o + d * hit_t;
      f3 radial = mk(std::fma(d.x, roff, cl.x), std::fma(d.y, roff, cl.y), std::fma(d.z, roff, cl.z));
      h->normal = normalize_safe(radial);
      h->material = mat;
      h->order = base + i;
      found = true;
    }
  }
  return found;
}

inline float affine_shift(const float* a, f3 o, f3 d) {
  f3 c = mk(a[3], a[7], a[11]);
  float den = dot(d, d);
  return den > 0.0f ? std::fmax(0.0f, dot(c - o, d) / den) : 0.0f;
}
inline f3 affine_point(const float* a, f3 o, f3 d, float shift) {
  f3 r = mk(std::fma(d.x, shift, o.x - a[3]), std::fma(d.y, shift, o.y - a[7]),
            std::fma(d.z, shift, o.z - a[11]));
  float x = a[0] * r.x;
  x = x + a[1] * r.y;
  x = x + a[2] * r.z;
  float y = a[4] * r.x;
  y = y + a[5] * r.y;
  y = y + a[6] * r.z;
  float z = a[8] * r.x;
  z = z + a[9] * r.y;
  z = z + a[10] * r.z;
  return mk(x, y, z);
}
inline f3 affine_vector(const float* a, f3 v) {
  float x = a[0] * v.x;
  x = x + a[1] * v.y;
  x = x + a[2] * v.z;
  float y = a[4] * v.x;
  y = y + a[5] * v.y;
  y = y + a[6] * v.z;
  float z = a[8] * v.x;
  z = z + a[9] * v.y;
  z = z + a[10] * v.z;
  return mk(x, y, z);
}
inline f3 linear9(const float* a, f3 v) {
  float x = a[0] * v.x;
  x = x + a[1] * v.y;
  x = x + a[2] * v.z;
  float y = a[3] * v.x;
  y = y + a[4] * v.y;
  y = y + a[5] * v.z;
  float z = a[6] * v.x;
  z = z + a[7] * v.y;
  z = z + a[8] * v.z;
  return mk(x, y, z);
}

bool trace_affine_sphere(const float* data, int count, f3 o, f3 d, int base, Hit* h) {
  bool found = false;
  float closest_t = h->t;
  for (int i = 0; i < count; ++i) {
    const float* a = data + 22 * i;
    float shift = affine_shift(a, o, d);
    f3 lo = affine_point(a, o, d, shift);
    f3 ld = affine_vector(a, d);
    float after_local = EPS - shift;
    float solve_a = dot(ld, ld);
    f3 sd = ld;
    float pscale = 1.0f;
    if (!(solve_a > 0.0f) || !std::isfinite(solve_a)) {
      DirFrame f = normalized_direction(ld);
      if (!f.valid) continue;
      sd = f.unit;
      solve_a = 1.0f;
      pscale = f.inv_len;
    }
    float scaled_after = after_local / pscale;
    float center_t = -dot(lo, sd) / solve_a;
    f3 cl = lo + sd * center_t;
    float radial_sq = std::fma(-cl.x, cl.x, std::fma(-cl.y, cl.y, std::fma(-cl.z, cl.z, 1.0f)));
    if (radial_sq <= 0.0f) continue;
    float half = std::sqrt(radial_sq / solve_a);
    float t1 = center_t - half;
    float t2 = center_t + half;
    float sh;
    if (t1 > scaled_after)
      sh = t1;
    else if (t2 > scaled_after)
      sh = t2;
    else
      continue;
    float hit_t = sh * pscale;
    float world_t = shift + hit_t;
    if (world_t >= closest_t) continue;
    f3 lh = lo + ld * hit_t;
    h->hit = 1;
    h->t = world_t;
    h->pos = o + d * world_t;
    h->normal = normalize_transformed(linear9(a + 12, lh));
    h->material = (int)a[21];
    h->order = base + i;
    closest_t = world_t;
    found = true;
  }
  return found;
}

// Shared slab logic of traceBox / traceAffineBox (K:588-706, 463-586).
inline bool slab_box(f3 o, f3 d, f3 bmin, f3 bmax, float after, float* t_out, int* axis_out,
                     float* sign_out) {
  float txmin, txmax, tymin, tymax, tzmin, tzmax;
  if (d.x == 0.0f) {
    if (o.x < bmin.x || o.x > bmax.x) return false;
    txmin = -INFINITY;
    txmax = INFINITY;
  } else {
    float t1 = (bmin.x - o.x) / d.x;
    float t2 = (bmax.x - o.x) / d.x;
    txmin = std::fmin(t1, t2);
    txmax = std::fmax(t1, t2);
  }
  if (d.y == 0.0f) {
    if (o.y < bmin.y || o.y > bmax.y) return false;
    tymin = -INFINITY;
    tymax = INFINITY;
  } else {
    float t1 = (bmin.y - o.y) / d.y;
    float t2 = (bmax.y - o.y) / d.y;
    tymin = std::fmin(t1, t2);
    tymax = std::fmax(t1, t2);
  }
  if (d.z == 0.0f) {
    if (o.z < bmin.z || o.z > bmax.z) return false;
    tzmin = -INFINITY;
    tzmax = INFINITY;
  } else {
    float t1 = (bmin.z - o.z) / d.z;
    float t2 = (bmax.z - o.z) / d.z;
    tzmin = std::fmin(t1, t2);
    tzmax = std::fmax(t1, t2);
  }
  float tenter = std::fmax(std::fmax(txmin, tymin), tzmin);
  float texit = std::fmin(std::fmin(txmax, tymax), tzmax);
  if (tenter >= texit || texit <= after) return false;
  int ae = 0;
  float ev = txmin;
  if (tymin > ev) {
    ev = tymin;
    ae = 1;
  }
  if (tzmin > ev) ae = 2;
  int ax = 0;
  float xv = txmax;
  if (tymax < xv) {
    xv = tymax;
    ax = 1;
  }
  if (tzmax < xv) ax = 2;
  if (tenter > after) {
    *t_out = tenter;
    *axis_out = ae;
    float dc = ae == 0 ? d.x : (ae == 1 ? d.y : d.z);
    *sign_out = dc > 0.0f ? -1.0f : 1.0f;
  } else {
    *t_out = texit;
    *axis_out = ax;
    float dc = ax == 0 ? d.x : (ax == 1 ? d.y : d.z);
    *sign_out = dc >= 0.0f ? 1.0f : -1.0f;
  }
  return true;
}

inline f3 axis_normal(int axis, float sign) {
  return axis == 0 ? mk(sign, 0, 0) : (axis == 1 ? mk(0, sign, 0) : mk(0, 0, sign));
}

bool trace_box(const float* data, int count, f3 o, f3 d, int base, Hit* h) {
  bool found = false;
  float closest_t = h->t;
  for (int i = 0; i < count; ++i) {
    const float* b = data + 7 * i;
    float t, sign;
    int axis;
    if (!slab_box(o, d, mk(b[0], b[1], b[2]), mk(b[3], b[4], b[5]), EPS, &t, &axis, &sign)) continue;
    if (t >= closest_t) continue;
    h->hit = 1;
    h->t = t;
    h->pos = o + d * t;
    h->normal = axis_normal(axis, sign);
    h->material = (int)b[6];
    h->order = base + i;
    closest_t = t;
    found = true;
  }
  return found;
}

bool trace_affine_box(const float* data, int count, f3 o, f3 d, int base, Hit* h) {
  bool found = false;
  float closest_t = h->t;
  for (int i = 0; i < count; ++i) {
    const float* a = data + 22 * i;
    float shift = affine_shift(a, o, d);
    f3 lo = affine_point(a, o, d, shift);
    f3 ld = affine_vector(a, d);
    float after_local = EPS - shift;
    float t, sign;
    int axis;
    if (!slab_box(lo, ld, mk(-1, -1, -1), mk(1, 1, 1), after_local, &t, &axis, &sign)) continue;
    float world_t = shift + t;
    if (world_t >= closest_t) continue;
    h->hit = 1;
    h->t = world_t;
    h->pos = o + d * world_t;
    h->normal = normalize_transformed(linear9(a + 12, axis_normal(axis, sign)));
    h->material = (int)a[21];
    h->order = base + i;
    closest_t = world_t;
    found = true;
  }
  return found;
}

inline float positive_mod(float x, float y) { return x - y * std::floor(x / y); }

int plane_material(const float* p, f3 hp) {
  const float* g = p + 18;
  int surface = (int)g[5];
  if (g[0] == 0.0f) return surface;
  f3 rel = hp - mk(p[4], p[5], p[6]);
  float be = dot(rel, mk(p[7], p[8], p[9])) / p[13];
  float bf = dot(rel, mk(p[10], p[11], p[12])) / p[14];
  float u = (be - bf * p[16]) / p[17];
  float v = (bf - be * p[15]) / p[17];
  float hx = g[3] * 0.5f;
  float hy = g[4] * 0.5f;
  float mx = positive_mod(u + hx, g[1]);
  float my = positive_mod(v + hy, g[2]);
  if (mx < g[3] || my < g[4]) return (int)g[7];
  return (int)g[6];
}

bool trace_plane(const float* planes, int count, f3 o, f3 d, int base, Hit* h) {
  bool found = false;
  float closest_t = h->t;
  for (int i = 0; i < count; ++i) {
    const float* p = planes + 26 * i;
    f3 n = mk(p[0], p[1], p[2]);
    float den = dot(n, d);
    if (den == 0.0f) continue;
    float t = -(dot(n, o) + p[3]) / den;
    if (t <= EPS || t >= closest_t) continue;
    f3 hp = o + d * t;
    h->hit = 1;
    h->t = t;
    h->pos = hp;
    h->normal = n;
    h->material = plane_material(p, hp);
    h->order = base + i;
    closest_t = t;
    found = true;
  }
  return found;
}

float entry_distance(const float* bounds, int node, f3 o, f3 d, float before_t) {
  const float* b = bounds + 6 * node;
  float tmin = EPS;
  float cb = std::isfinite(before_t) ? std::fma(before_t, 1.0000015f, 1.0e-6f) : before_t;
  float tmax = cb;
  for (int axis = 0; axis < 3; ++axis) {
    float oo = axis == 0 ? o.x : (axis == 1 ? o.y : o.z);
    float dd = axis == 0 ? d.x : (axis == 1 ? d.y : d.z);
    float lo = b[axis], hi = b[3 + axis];
    if (dd == 0.0f) {
      if (oo < lo || oo > hi) return INFINITY;
      continue;
    }
    float t0 = (lo - oo) / dd;
    float t1 = (hi - oo) / dd;
    if (t0 > t1) {
      float tmp = t0;
      t0 = t1;
      t1 = tmp;
    }
    if (t1 > 0.0f) t1 = t1 * 1.00000072f;
    tmin = std::fmax(tmin, t0);
    tmax = std::fmin(tmax, t1);
    if (tmax < tmin) return INFINITY;
  }
  return tmin <= cb ? tmin : INFINITY;
}

inline int type_index(int type) {
  return type == T_BOX ? 1 : type == T_ASPHERE ? 3 : type == T_ABOX ? 4 : 0;
}

bool trace_ref(const Scene& s, int ref, int type, f3 o, f3 d, Hit* h) {
  int index = ref & INDEX_MASK;
  Hit cand;
  cand.t = std::nextafter(h->t, INFINITY);
  bool ok;
  int order;
  if (type == T_BOX) {
    order = s.ns + index;
    ok = trace_box(s.boxes + 7 * index, 1, o, d, order, &cand);
  } else if (type == T_ASPHERE) {
    order = s.ns + s.nb + index;
    ok = trace_affine_sphere(s.aspheres + 22 * index, 1, o, d, order, &cand);
  } else if (type == T_ABOX) {
    order = s.ns + s.nb + s.nas + index;
    ok = trace_affine_box(s.aboxes + 22 * index, 1, o, d, order, &cand);
  } else {
    order = index;
    ok = trace_sphere(s.spheres + 5 * index, 1, o, d, order, &cand);
  }
  if (!ok || cand.t > h->t || (cand.t == h->t && order >= h->order)) return false;
  *h = cand;
  h->order = order;
  return true;
}

bool trace_leaf(const Scene& s, int kind, int first, int count, f3 o, f3 d, Hit* h, Stats* st) {
  if (st) st->v[2] += (uint64_t)count;
  bool found = false;
  int leaf_type = kind == -2 ? T_SPHERE : kind == -3 ? T_BOX : kind == -4 ? T_ASPHERE
                : kind == -5 ? T_ABOX : -1;
  for (int i = 0; i < count; ++i) {
    int ri = first + i;
    if (ri < 0 || ri >= s.ref_count) continue;
    int ref = s.refs[ri];
    int type = leaf_type == -1 ? (ref & TYPE_MASK) : leaf_type;
    if (st) st->v[3 + type_index(type)]++;
    found |= trace_ref(s, ref, type, o, d, h);
  }
  return found;
}

bool trace_bvh(const Scene& s, f3 o, f3 d, Hit* h, Stats* st) {
  if (s.node_count <= 0 || s.ref_count <= 0 || s.root_count <= 0 || s.root_count > 4) return false;
  int ss = s.stack_size;
  int nstack[256];
  float estack[256];
  int size = 0;
  bool found = false, overflow = false;
  for (int r = 0; r < s.root_count; ++r) {
    int ri = s.roots[r];
    if (ri < 0 || ri >= s.node_count) {
      overflow = true;
      break;
    }
    if (st) st->v[1]++;
    float e = entry_distance(s.node_bounds, ri, o, d, h->t);
    if (!std::isfinite(e)) continue;
    if (size >= ss) {
      overflow = true;
      break;
    }
    int pos = size;
    while (pos > 0 && e >= estack[pos - 1]) {
      nstack[pos] = nstack[pos - 1];
      estack[pos] = estack[pos - 1];
      pos--;
    }
    nstack[pos] = ri;
    estack[pos] = e;
    size++;
    if (st && (uint64_t)size > st->v[9]) st->v[9] = size;
  }
  while (!overflow && size > 0) {
    int node = nstack[--size];
    float entry = estack[size];
    float cht = std::isfinite(h->t) ? std::fma(h->t, 1.0000015f, 1.0e-6f) : h->t;
    if (entry > cht) continue;
    const int* nd = s.node_data + 4 * node;
    int left = nd[0], right = nd[1], first = nd[2], count = nd[3];
    if (left < 0) {
      if (st) {
        st->v[11]++;
        if (left == -1)
          st->v[13]++;
        else
          st->v[12]++;
      }
      found |= trace_leaf(s, left, first, count, o, d, h, st);
      continue;
    }
    if (st) st->v[10]++;
    float le = entry_distance(s.node_bounds, left, o, d, h->t);
    float re = entry_distance(s.node_bounds, right, o, d, h->t);
    if (st) st->v[1] += 2;
    int nn = left, fn = right;
    float ne = le, fe = re;
    if (re < le) {
      nn = right;
      fn = left;
      ne = re;
      fe = le;
    }
    if (std::isfinite(fe)) {
      if (size >= ss) {
        overflow = true;
        break;
      }
      nstack[size] = fn;
      estack[size++] = fe;
      if (st && (uint64_t)size > st->v[9]) st->v[9] = size;
    }
    if (std::isfinite(ne)) {
      if (size >= ss) {
        overflow = true;
        break;
      }
      nstack[size] = nn;
      estack[size++] = ne;
      if (st && (uint64_t)size > st->v[9]) st->v[9] = size;
    }
  }
  if (overflow) {
    if (st) st->v[8]++;
    for (int i = 0; i < s.ref_count; ++i) {
      int type = s.refs[i] & TYPE_MASK;
      if (st) {
        st->v[2]++;
        st->v[3 + type_index(type)]++;
      }
      found |= trace_ref(s, s.refs[i], type, o, d, h);
    }
  }
  return found;
}

bool trace_closest(const Scene& s, f3 o, f3 d, Hit* h, Stats* st) {
  h->hit = 0;
  h->t = 1e30f;
  h->order = 0x7FFFFFFF;
  bool found;
  if (s.use_bvh && s.node_count > 0) {
    found = trace_bvh(s, o, d, h, st);
  } else {
    if (st) {
      st->v[2] += (uint64_t)s.ns + s.nb + s.nas + s.nab;
      st->v[3] += s.ns;
      st->v[4] += s.nb;
      st->v[6] += s.nas;
      st->v[7] += s.nab;
    }
    found = trace_sphere(s.spheres, s.ns, o, d, 0, h);
    found |= trace_box(s.boxes, s.nb, o, d, s.ns, h);
    found |= trace_affine_sphere(s.aspheres, s.nas, o, d, s.ns + s.nb, h);
    found |= trace_affine_box(s.aboxes, s.nab, o, d, s.ns + s.nb + s.nas, h);
  }
  if (st) {
    st->v[2] += s.np;
    st->v[5] += s.np;
  }
  found |= trace_plane(s.planes, s.np, o, d, s.ns + s.nb + s.nas + s.nab, h);
  return found;
}

inline float luminance(f3 c) {
  float r = c.x * 0.212655f;
  r = r + c.y * 0.715158f;
  r = r + c.z * 0.072187f;
  return r;
}
inline f3 reflect_dir(f3 n, f3 i) { return n * (2.0f * dot(i, n)) - i; }
inline void refract_dir(f3 inc, f3 n, float eta, f3* out) {
  f3 i = normalize_safe(inc);
  float c1 = dot(i, n);
  float ri = (c1 >= 0.0f) ? eta : -1.0f / eta;
  float inv_ri2 = 1.0f / (ri * ri);
  float c2 = 1.0f - (1.0f - c1 * c1) * inv_ri2;
  if (c2 <= 0.0f) {
    *out = normalize_safe(reflect_dir(n, i));
    return;
  }
  float sq = std::sqrt(c2);
  *out = normalize_safe(n * (c1 - sq * ri) - i);
}

f3 trace_path(const Scene& s, f3 o, f3 d, f3 bg, int max_depth, uint32_t* rng) {
  f3 thr = mk(1, 1, 1);
  f3 rad = mk(0, 0, 0);
  const float* M = s.materials;
  for (int depth = 0; depth < max_depth; ++depth) {
    Hit h;
    if (!trace_closest(s, o, d, &h, nullptr)) {
      rad = rad + thr * bg;
      break;
    }
    const float* m = h.material >= 0 ? M + 13 * h.material : nullptr;
    f3 cd = m ? mk(m[0], m[1], m[2]) : mk(0, 0, 0);
    f3 cr = m ? mk(m[3], m[4], m[5]) : mk(0, 0, 0);
    f3 ct = m ? mk(m[6], m[7], m[8]) : mk(0, 0, 0);
    f3 ce = m ? mk(m[9], m[10], m[11]) : mk(0, 0, 0);
    float ior = m ? m[12] : 0.0f;
    rad = rad + thr * ce;
    f3 n = h.normal;
    f3 inc = -d;
    float wd = luminance(cd), wr = luminance(cr), wt = luminance(ct);
    float sum = (wd + wr) + wt;
    if (sum <= 0.0f) break;
    float xi = rand01(rng) * sum;
    f3 nd, wc;
    float p;
    if (xi < wd) {
      p = wd / sum;
      float z = rand01(rng) * 2.0f - 1.0f;
      float tt = rand01(rng) * 2.0f * 3.14159265358979323846f;
      float r = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
      nd = mk(r * std::cos(tt), r * std::sin(tt), z) + n;
      wc = cd / p;
    } else if (xi < wd + wr) {
      p = wr / sum;
      nd = reflect_dir(n, inc);
      wc = cr / p;
    } else {
      p = wt / sum;
      refract_dir(inc, n, ior, &nd);
      wc = ct / p;
    }
    o = h.pos + nd * EPS;
    thr = thr * wc;
    d = nd;
  }
  return rad;
}

Scene make_scene(const float* const* arrays, const int* counts, const int* bvh_ints,
                 const float* node_bounds, const int* node_data, const int* refs,
                 const int* roots) {
  Scene s{};
  s.spheres = arrays[0];
  s.ns = counts[0];
  s.boxes = arrays[1];
  s.nb = counts[1];
  s.planes = arrays[2];
  s.np = counts[2];
  s.aspheres = arrays[3];
  s.nas = counts[3];
  s.aboxes = arrays[4];
  s.nab = counts[4];
  s.materials = arrays[5];
  s.nm = counts[5];
  s.node_bounds = node_bounds;
  s.node_data = node_data;
  s.refs = refs;
  s.roots = roots;
  s.node_count = bvh_ints[0];
  s.ref_count = bvh_ints[1];
  s.root_count = bvh_ints[2];
  s.use_bvh = bvh_ints[3];
  s.stack_size = bvh_ints[4] > 0 && bvh_ints[4] <= 256 ? bvh_ints[4] : 32;
  return s;
}

}  // namespace

extern "C" {

// arrays: spheres, boxes, planes, affine spheres, affine boxes, materials (reference
// packed layouts, 5/7/26/22/22/13 floats per record); counts: the six record counts.
// bvh_ints: node_count, ref_count, root_count, use_bvh, stack_size.
// Outputs follow traceReplayKernel (K:1369-1376).  stats (14 u64, may be null)
// accumulates the reference's counter set.
void orc_trace(const float* const* arrays, const int* counts, const int* bvh_ints,
               const float* node_bounds, const int* node_data, const int* refs, const int* roots,
               const float* rays, int n, int* hit_flags, float* hit_t, int* hit_order,
               int* hit_material, float* hit_normal, unsigned long long* stats) {
  Scene s = make_scene(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots);
  Stats st;
  std::memset(&st, 0, sizeof(st));
  for (int r = 0; r < n; ++r) {
    f3 o = mk(rays[6 * r], rays[6 * r + 1], rays[6 * r + 2]);
    f3 d = mk(rays[6 * r + 3], rays[6 * r + 4], rays[6 * r + 5]);
    Hit h;
    Stats* sp = stats ? &st : nullptr;
    if (sp) sp->v[0]++;
    bool found = trace_closest(s, o, d, &h, sp);
    hit_flags[r] = found ? 1 : 0;
    hit_t[r] = found ? h.t : INFINITY;
    hit_order[r] = found ? h.order : -1;
    hit_material[r] = found ? h.material : -1;
    hit_normal[3 * r] = found ? h.normal.x : 0.0f;
    hit_normal[3 * r + 1] = found ? h.normal.y : 0.0f;
    hit_normal[3 * r + 2] = found ? h.normal.z : 0.0f;
  }
  if (stats) {
    for (int k = 0; k < 14; ++k) {
      if (k == 9)
        stats[k] = stats[k] > st.v[k] ? stats[k] : st.v[k];
      else
        stats[k] += st.v[k];
    }
  }
}

// Distance from each ray r to the one primitive with global order orders[r] (spheres,
// boxes, affine spheres, affine boxes, planes -- the kernel's tie-break order, K:1003-1017),
// in this file's uncontracted FP32 arithmetic, as that primitive's own test computes it
// with no earlier hit (INFINITY where the test misses).  Used to judge whether a hit that
// another build picked is a near tie of this arithmetic's winner.
void orc_primitive_distance(const float* const* arrays, const int* counts, const float* rays,
                            const int* orders, int n, float* out_t) {
  const int no_bvh[5] = {0, 0, 0, 0, 32};
  Scene s = make_scene(arrays, counts, no_bvh, nullptr, nullptr, nullptr, nullptr);
  const int b1 = s.ns, b2 = b1 + s.nb, b3 = b2 + s.nas, b4 = b3 + s.nab, b5 = b4 + s.np;
  for (int r = 0; r < n; ++r) {
    f3 o = mk(rays[6 * r], rays[6 * r + 1], rays[6 * r + 2]);
    f3 d = mk(rays[6 * r + 3], rays[6 * r + 4], rays[6 * r + 5]);
    int k = orders[r];
    Hit h;
    h.t = INFINITY;
    h.order = 0x7FFFFFFF;
    bool ok = false;
    if (k >= 0 && k < b1)
      ok = trace_sphere(s.spheres + 5 * k, 1, o, d, k, &h);
    else if (k >= b1 && k < b2)
      ok = trace_box(s.boxes + 7 * (k - b1), 1, o, d, k, &h);
    else if (k >= b2 && k < b3)
      ok = trace_affine_sphere(s.aspheres + 22 * (k - b2), 1, o, d, k, &h);
    else if (k >= b3 && k < b4)
      ok = trace_affine_box(s.aboxes + 22 * (k - b3), 1, o, d, k, &h);
    else if (k >= b4 && k < b5)
      ok = trace_plane(s.planes + 26 * (k - b4), 1, o, d, k, &h);
    out_t[r] = ok ? h.t : INFINITY;
  }
}

// Renders pixels [pixel_begin, pixel_end) of a width x height image with the
// renderKernel sample loop: samples 0..spp-1 in order, FP32 running sum, scaled by
// 1/spp after the last sample (K:1284-1293).  camera: pos, forward, right, up (12 floats);
// params: width, height, spp, max_depth, frame_index.  rgb receives 3 floats per pixel
// of the range.
void orc_render(const float* const* arrays, const int* counts, const int* bvh_ints,
                const float* node_bounds, const int* node_data, const int* refs, const int* roots,
                const float* camera, const float* background, const int* params,
                unsigned long long frame_seed, int pixel_begin, int pixel_end, float* rgb) {
  Scene s = make_scene(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots);
  int width = params[0], height = params[1], spp = params[2], max_depth = params[3];
  int frame_index = params[4];
  f3 cp = mk(camera[0], camera[1], camera[2]);
  f3 cf = mk(camera[3], camera[4], camera[5]);
  f3 cr = mk(camera[6], camera[7], camera[8]);
  f3 cu = mk(camera[9], camera[10], camera[11]);
  f3 bg = mk(background[0], background[1], background[2]);
  for (int p = pixel_begin; p < pixel_end; ++p) {
    int x = p % width, y = p / width;
    uint32_t base = hash_u32((uint32_t)(frame_seed & 0xFFFFFFFFULL));
    base ^= hash_u32((uint32_t)(frame_seed >> 32));
    base ^= hash_u32((uint32_t)frame_index);
    uint32_t pix = (uint32_t)y * (uint32_t)width + (uint32_t)x;
    base ^= hash_u32(pix);
    base = hash_u32(base);
    f3 acc = mk(0, 0, 0);
    for (int so = 0; so < spp; ++so) {
      uint32_t seed = base ^ hash_u32((uint32_t)so);
      seed ^= hash_u32((uint32_t)so * 0x9E3779B9u);
      seed = hash_u32(seed);
      uint32_t rng = seed;
      float jx = rand01(&rng) - 0.5f;
      float jy = rand01(&rng) - 0.5f;
      float aspect = (float)width / (float)height;
      float u = ((((float)x + 0.5f) + jx) * (2.0f / (float)width) - 1.0f) * aspect;
      float v = 1.0f - ((((float)y + 0.5f) + jy) * (2.0f / (float)height));
      f3 dir = (cf + cr * u) + cu * v;
      f3 c = trace_path(s, cp, dir, bg, max_depth, &rng);
      acc = so == 0 ? c : acc + c;
      if (so == spp - 1) acc = acc * (1.0f / (float)spp);
    }
    float* out = rgb + 3 * (p - pixel_begin);
    out[0] = acc.x;
    out[1] = acc.y;
    out[2] = acc.z;
  }
}

// FP64 adjoint of the sample loop for a pixel range (test infrastructure): the FP32 path of
// orc_render, with dLoss/d(albedo) and dLoss/d(emission) per material accumulated in double
// along the path backward (Li <- E + W Li), the lobe probability held fixed.  adjoint holds
// dLoss/dI (3 floats per pixel of the whole image); grads are 3 doubles per material each.
void orc_adjoint(const float* const* arrays, const int* counts, const int* bvh_ints,
                 const float* node_bounds, const int* node_data, const int* refs, const int* roots,
                 const float* camera, const float* background, const int* params,
                 unsigned long long frame_seed, int pixel_begin, int pixel_end, const float* adjoint,
                 double* grad_albedo, double* grad_emission) {
  Scene s = make_scene(arrays, counts, bvh_ints, node_bounds, node_data, refs, roots);
  int width = params[0], height = params[1], spp = params[2], max_depth = params[3];
  int frame_index = params[4];
  f3 cp = mk(camera[0], camera[1], camera[2]);
  f3 cf = mk(camera[3], camera[4], camera[5]);
  f3 cr = mk(camera[6], camera[7], camera[8]);
  f3 cu = mk(camera[9], camera[10], camera[11]);
  f3 bg = mk(background[0], background[1], background[2]);
  const float* M = s.materials;
  for (int p = pixel_begin; p < pixel_end; ++p) {
    int x = p % width, y = p / width;
    uint32_t base = hash_u32((uint32_t)(frame_seed & 0xFFFFFFFFULL));
    base ^= hash_u32((uint32_t)(frame_seed >> 32));
    base ^= hash_u32((uint32_t)frame_index);
    base ^= hash_u32((uint32_t)y * (uint32_t)width + (uint32_t)x);
    base = hash_u32(base);
    double adj[3] = {adjoint[3 * p] / (double)spp, adjoint[3 * p + 1] / (double)spp,
                     adjoint[3 * p + 2] / (double)spp};
    for (int so = 0; so < spp; ++so) {
      uint32_t seed = base ^ hash_u32((uint32_t)so);
      seed ^= hash_u32((uint32_t)so * 0x9E3779B9u);
      seed = hash_u32(seed);
      uint32_t rng = seed;
      float jx = rand01(&rng) - 0.5f;
      float jy = rand01(&rng) - 0.5f;
      float aspect = (float)width / (float)height;
      float u = ((((float)x + 0.5f) + jx) * (2.0f / (float)width) - 1.0f) * aspect;
      float v = 1.0f - ((((float)y + 0.5f) + jy) * (2.0f / (float)height));
      f3 o = cp, d = (cf + cr * u) + cu * v;
      f3 thr = mk(1, 1, 1);
      int vm[33];
      f3 vthr[33], vw[33];
      double vinvp[33];
      int nv = 0;
      bool escaped = false;
      for (int depth = 0; depth < max_depth; ++depth) {
        Hit h;
        if (!trace_closest(s, o, d, &h, nullptr)) {
          escaped = true;
          break;
        }
        const float* m = h.material >= 0 ? M + 13 * h.material : nullptr;
        f3 cd = m ? mk(m[0], m[1], m[2]) : mk(0, 0, 0);
        f3 crf = m ? mk(m[3], m[4], m[5]) : mk(0, 0, 0);
        f3 ct = m ? mk(m[6], m[7], m[8]) : mk(0, 0, 0);
        float ior = m ? m[12] : 0.0f;
        vm[nv] = h.material;
        vthr[nv] = thr;
        vw[nv] = mk(0, 0, 0);
        vinvp[nv] = 0.0;
        f3 n = h.normal, inc = -d;
        float wd = luminance(cd), wr = luminance(crf), wt = luminance(ct);
        float sum = (wd + wr) + wt;
        if (sum <= 0.0f) {
          nv++;
          break;
        }
        float xi = rand01(&rng) * sum;
        f3 nd, wc;
        if (xi < wd) {
          float pc = wd / sum;
          float z = rand01(&rng) * 2.0f - 1.0f;
          float tt = rand01(&rng) * 2.0f * 3.14159265358979323846f;
          float r = std::sqrt(std::fmax(0.0f, 1.0f - z * z));
          nd = mk(r * std::cos(tt), r * std::sin(tt), z) + n;
          wc = cd / pc;
          vinvp[nv] = 1.0 / (double)pc;
        } else if (xi < wd + wr) {
          float pc = wr / sum;
          nd = reflect_dir(n, inc);
          wc = crf / pc;
        } else {
          float pc = wt / sum;
          refract_dir(inc, n, ior, &nd);
          wc = ct / pc;
        }
        vw[nv] = wc;
        nv++;
        o = h.pos + nd * EPS;
        thr = thr * wc;
        d = nd;
      }
      double li[3] = {escaped ? (double)bg.x : 0.0, escaped ? (double)bg.y : 0.0,
                      escaped ? (double)bg.z : 0.0};
      for (int k = nv - 1; k >= 0; --k) {
        int mi = vm[k];
        double e[3] = {0, 0, 0};
        double t3[3] = {vthr[k].x, vthr[k].y, vthr[k].z};
        double w3[3] = {vw[k].x, vw[k].y, vw[k].z};
        if (mi >= 0) {
          const float* m = M + 13 * mi;
          for (int c = 0; c < 3; ++c) {
            e[c] = m[9 + c];
            double basev = adj[c] * t3[c];
            grad_emission[3 * mi + c] += basev;
            grad_albedo[3 * mi + c] += basev * li[c] * vinvp[k];
          }
        }
        for (int c = 0; c < 3; ++c) li[c] = e[c] + w3[c] * li[c];
      }
    }
  }
}

}  // extern "C"
