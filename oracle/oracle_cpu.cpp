// Oracle (test infrastructure only): a C++ restatement, in IEEE double precision, of the
// reference's host-CPU renderer for the same scenes -- the CPU baseline the GPU path is
// timed against and the FP64 image the GPU images are compared with (RMSE).
// Only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / --impl reference
// legs may load this code.
//
// Restated from (gfxlab/ = src/xyz/marsavic/gfxlab/):
//   CPU BVH build        gfxlab/graphics3d/bvh/BvhSolid.java:84-122, 336-451
//                        (unit-cost exact-sweep SAH, leaf size a hard maximum, default 4;
//                        outward bounds widened by two double ulps; split positions with
//                        equal neighbouring centroids skipped)
//   CPU BVH traversal    gfxlab/graphics3d/bvh/BvhSolid.java:157-246 and Aabb.entryDistance
//   sphere               gfxlab/graphics3d/solids/Ball.java:51-64
//   box                  gfxlab/graphics3d/solids/Box.java:83-131
//   half-space           gfxlab/graphics3d/solids/HalfSpace.java:87-96
//   affine instances     gfxlab/graphics3d/Solid.java:29-41 (ray into object space, normal
//                        through the inverse transpose)
//   path tracer          gfxlab/graphics3d/raytracers/PathTracer.java:30-71
//   material lobes       gfxlab/graphics3d/Material.java (BSDF.add of diffuse, reflective and
//                        refractive lobes weighted by luminance), gfxlab/graphics3d/BSDF.java:30-100
//   diffuse sampling     gfxlab/graphics3d/GeometryUtils.java:48-62 (rejection sampling in
//                        the unit ball, normalised, plus the normal)
//   row-parallel driver  gfxlab/playground/HeadlessCpuBvhRenderer.java:80, 118-146 (splitmix
//                        jitter per pixel and frame, one sample per pixel per frame)
// The reference draws its path random numbers from a closed library (mars-bits Sampler);
// this restatement draws them from the GPU kernel's counter hash instead, so images agree
// with the reference CPU renderer statistically, not sample for sample.
// Geometry is the float-packed scene promoted to double.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#include <omp.h>

namespace {

struct d3 {
  double x, y, z;
};
inline d3 mk(double x, double y, double z) { return d3{x, y, z}; }
inline d3 operator+(d3 a, d3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline d3 operator-(d3 a, d3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline d3 operator*(d3 a, double s) { return mk(a.x * s, a.y * s, a.z * s); }
inline d3 mul(d3 a, d3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline double dot(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double get(d3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline d3 normalized(d3 v) {
  double l = std::sqrt(dot(v, v));
  return mk(v.x / l, v.y / l, v.z / l);
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
struct Sampler {
  uint32_t s;
  double uniform() {
    s = hash_u32(s + 0x9e3779b9U);
    uint32_t hi = s >> 5;
    s = hash_u32(s + 0x9e3779b9U);
    uint32_t lo = s >> 6;
    return ((double)hi * 67108864.0 + (double)lo) * (1.0 / 9007199254740992.0);
  }
};

inline uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ULL;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

enum Kind { SPHERE = 0, BOX = 1, ASPHERE = 2, ABOX = 3 };

struct Prim {
  int kind;
  int index;
  int order;
  double bmin[3], bmax[3];
  double cen[3];
};

struct Material {
  d3 diffuse, reflective, refractive, emittance;
  double ior;
  double w[3];   // luminance weights of the non-zero lobes, normalised
  int lobe[3];   // lobe ids (0 diffuse, 1 reflective, 2 refractive)
  int m;
};

struct Hit {
  double t = INFINITY;
  int order = INT32_MAX;
  d3 n{0, 0, 0};
  int material = -1;
};

inline double next_up(double v) { return std::nextafter(v, INFINITY); }
inline double next_down(double v) { return std::nextafter(v, -INFINITY); }

struct CpuScene {
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
  std::vector<Material> materials;
  std::vector<Prim> prims;
  struct Node {
    double bmin[3], bmax[3];
    int left, right, first, count;
  };
  std::vector<Node> nodes;
  int leaf_size = 4;

  // --- primitive intersection (double) ---
  static bool ball(d3 c, double r, d3 p, d3 d, double after, double* t) {
    d3 e = c - p;
    double dsq = dot(d, d);
    double l = dot(e, d) / dsq;
    double msq = l * l - (dot(e, e) - r * r) / dsq;
    if (msq > 0) {
      double m = std::sqrt(msq);
      if (l - m > after) {
        *t = l - m;
        return true;
      }
      if (l + m > after) {
        *t = l + m;
        return true;
      }
    }
    return false;
  }
  static bool box(const double* lo, const double* hi, d3 p, d3 d, double after, double* t,
                  d3* n) {
    double te = -INFINITY, tx = INFINITY;
    int ea = -1, xa = -1;
    for (int a = 0; a < 3; ++a) {
      double o = get(p, a), dd = get(d, a);
      double mn = std::min(lo[a], hi[a]), mxv = std::max(lo[a], hi[a]);
      if (dd == 0.0) {
        if (o < mn || o > mxv) return false;
        continue;
      }
      double t0 = (mn - o) / dd, t1 = (mxv - o) / dd;
      if (t0 > t1) std::swap(t0, t1);
      if (t0 > te) {
        te = t0;
        ea = a;
      }
      if (t1 < tx) {
        tx = t1;
        xa = a;
      }
      if (te >= tx) return false;
    }
    if (ea >= 0 && te > after) {
      double s = get(d, ea) > 0 ? -1.0 : (get(d, ea) < 0 ? 1.0 : 0.0);
      *t = te;
      *n = mk(ea == 0 ? s : 0, ea == 1 ? s : 0, ea == 2 ? s : 0);
      return true;
    }
    if (xa >= 0 && tx > after) {
      double s = get(d, xa) > 0 ? 1.0 : (get(d, xa) < 0 ? -1.0 : 0.0);
      *t = tx;
      *n = mk(xa == 0 ? s : 0, xa == 1 ? s : 0, xa == 2 ? s : 0);
      return true;
    }
    return false;
  }

  bool prim_hit(const Prim& pr, d3 p, d3 d, double after, double* t, d3* n, int* mat) const {
    if (pr.kind == SPHERE) {
      const float* s = spheres + 5 * pr.index;
      d3 c = mk(s[0], s[1], s[2]);
      double r = s[3];
      if (!ball(c, r, p, d, after, t)) return false;
      d3 q = p + d * *t;
      *n = (q - c) * (1.0 / r);
      *mat = (int)s[4];
      return true;
    }
    if (pr.kind == BOX) {
      const float* b = boxes + 7 * pr.index;
      double lo[3] = {b[0], b[1], b[2]}, hi[3] = {b[3], b[4], b[5]};
      if (!box(lo, hi, p, d, after, t, n)) return false;
      *mat = (int)b[6];
      return true;
    }
    const float* a = (pr.kind == ASPHERE ? aspheres : aboxes) + 22 * pr.index;
    d3 rel = p - mk(a[3], a[7], a[11]);
    d3 lp = mk(a[0] * rel.x + a[1] * rel.y + a[2] * rel.z, a[4] * rel.x + a[5] * rel.y + a[6] * rel.z,
               a[8] * rel.x + a[9] * rel.y + a[10] * rel.z);
    d3 ld = mk(a[0] * d.x + a[1] * d.y + a[2] * d.z, a[4] * d.x + a[5] * d.y + a[6] * d.z,
               a[8] * d.x + a[9] * d.y + a[10] * d.z);
    d3 ln;
    if (pr.kind == ASPHERE) {
      if (!ball(mk(0, 0, 0), 1.0, lp, ld, after, t)) return false;
      ln = lp + ld * *t;
    } else {
      double lo[3] = {-1, -1, -1}, hi[3] = {1, 1, 1};
      if (!box(lo, hi, lp, ld, after, t, &ln)) return false;
    }
    const float* m = a + 12;
    *n = normalized(mk(m[0] * ln.x + m[1] * ln.y + m[2] * ln.z, m[3] * ln.x + m[4] * ln.y + m[5] * ln.z,
                       m[6] * ln.x + m[7] * ln.y + m[8] * ln.z));
    *mat = (int)a[21];
    return true;
  }

  // --- BVH (BvhSolid.BuildState) ---
  static double area(const double* mn, const double* mx) {
    double dx = mx[0] - mn[0], dy = mx[1] - mn[1], dz = mx[2] - mn[2];
    return 2.0 * (dx * dy + dx * dz + dy * dz);
  }
  void bounds_of(int s, int e, double* mn, double* mx) const {
    for (int k = 0; k < 3; ++k) {
      mn[k] = INFINITY;
      mx[k] = -INFINITY;
    }
    for (int i = s; i < e; ++i)
      for (int k = 0; k < 3; ++k) {
        mn[k] = std::min(mn[k], prims[i].bmin[k]);
        mx[k] = std::max(mx[k], prims[i].bmax[k]);
      }
  }
  int build(int s, int e) {
    int count = e - s;
    Node node;
    bounds_of(s, e, node.bmin, node.bmax);
    int idx = (int)nodes.size();
    nodes.push_back(node);
    auto make_leaf = [&]() {
      nodes[idx].left = nodes[idx].right = -1;
      nodes[idx].first = s;
      nodes[idx].count = count;
      return idx;
    };
    if (count <= leaf_size) return make_leaf();
    double node_area = area(node.bmin, node.bmax);
    double leaf_cost = node_area * count;
    int best_axis = -1, best_i = 0;
    double best_cost = INFINITY;
    std::vector<double> pmin(3 * count), pmax(3 * count), smin(3 * count), smax(3 * count);
    for (int axis = 0; axis < 3; ++axis) {
      std::stable_sort(prims.begin() + s, prims.begin() + e,
                       [axis](const Prim& a, const Prim& b) { return a.cen[axis] < b.cen[axis]; });
      double rmn[3] = {INFINITY, INFINITY, INFINITY}, rmx[3] = {-INFINITY, -INFINITY, -INFINITY};
      for (int i = 0; i < count; ++i) {
        for (int k = 0; k < 3; ++k) {
          rmn[k] = std::min(rmn[k], prims[s + i].bmin[k]);
          rmx[k] = std::max(rmx[k], prims[s + i].bmax[k]);
          pmin[3 * i + k] = rmn[k];
          pmax[3 * i + k] = rmx[k];
        }
      }
      for (int k = 0; k < 3; ++k) {
        rmn[k] = INFINITY;
        rmx[k] = -INFINITY;
      }
      for (int i = count - 1; i >= 0; --i) {
        for (int k = 0; k < 3; ++k) {
          rmn[k] = std::min(rmn[k], prims[s + i].bmin[k]);
          rmx[k] = std::max(rmx[k], prims[s + i].bmax[k]);
          smin[3 * i + k] = rmn[k];
          smax[3 * i + k] = rmx[k];
        }
      }
      for (int i = 1; i < count; ++i) {
        if (prims[s + i - 1].cen[axis] == prims[s + i].cen[axis]) continue;
        double cost = node_area + area(&pmin[3 * (i - 1)], &pmax[3 * (i - 1)]) * i +
                      area(&smin[3 * i], &smax[3 * i]) * (count - i);
        if (cost < best_cost) {
          best_cost = cost;
          best_axis = axis;
          best_i = i;
        }
      }
    }
    if (best_axis < 0 || best_cost >= leaf_cost) return make_leaf();
    std::stable_sort(prims.begin() + s, prims.begin() + e,
                     [best_axis](const Prim& a, const Prim& b) {
                       return a.cen[best_axis] < b.cen[best_axis];
                     });
    int mid = s + best_i;
    int l = build(s, mid);
    int r = build(mid, e);
    nodes[idx].left = l;
    nodes[idx].right = r;
    nodes[idx].first = -1;
    nodes[idx].count = 0;
    return idx;
  }

  double entry(const Node& n, d3 p, d3 d, double after, double before) const {
    double tmin = after, tmax = before;
    for (int a = 0; a < 3; ++a) {
      double o = get(p, a), dd = get(d, a);
      if (dd == 0.0) {
        if (o < n.bmin[a] || o > n.bmax[a]) return INFINITY;
        continue;
      }
      double t1 = (n.bmin[a] - o) / dd, t2 = (n.bmax[a] - o) / dd;
      if (t1 > t2) std::swap(t1, t2);
      if (t2 > 0.0 && std::isfinite(t2)) t2 = next_up(next_up(t2));
      tmin = std::max(tmin, t1);
      tmax = std::min(tmax, t2);
      if (tmax < tmin) return INFINITY;
    }
    return tmin <= before ? tmin : INFINITY;
  }

  Hit first_hit(d3 p, d3 d, double after) const {
    Hit best;
    for (int i = 0; i < np; ++i) {
      const float* pl = planes + 26 * i;
      d3 n = mk(pl[0], pl[1], pl[2]);
      double o = dot(n, d);
      double l = -(dot(n, p) + (double)pl[3]);
      if (o == 0) continue;
      double t = l / o;
      int order = ns + nb + nas + nab + i;
      if (t > after && (t < best.t || (t == best.t && order < best.order))) {
        best.t = t;
        best.order = order;
        best.n = n;
        best.material = (int)pl[18 + 5];
      }
    }
    if (nodes.empty()) return best;
    int stack[128];
    double estack[128];
    int size = 0;
    double re = entry(nodes[0], p, d, after, best.t);
    if (re == INFINITY) return best;
    stack[size] = 0;
    estack[size++] = re;
    while (size > 0) {
      int ni = stack[--size];
      double e = estack[size];
      if (e > best.t) continue;
      const Node& nd = nodes[ni];
      if (nd.left < 0) {
        for (int i = 0; i < nd.count; ++i) {
          const Prim& pr = prims[nd.first + i];
          double t;
          d3 n;
          int mat;
          if (prim_hit(pr, p, d, after, &t, &n, &mat) &&
              (t < best.t || (t == best.t && pr.order < best.order))) {
            best.t = t;
            best.order = pr.order;
            best.n = n;
            best.material = mat;
          }
        }
        continue;
      }
      double le = entry(nodes[nd.left], p, d, after, best.t);
      double ri = entry(nodes[nd.right], p, d, after, best.t);
      if (le == INFINITY && ri == INFINITY) continue;
      if (size + 2 > 128) continue;  // depth beyond 64 levels is not produced by the builder
      if (le <= ri) {
        if (ri != INFINITY) {
          stack[size] = nd.right;
          estack[size++] = ri;
        }
        if (le != INFINITY) {
          stack[size] = nd.left;
          estack[size++] = le;
        }
      } else {
        if (le != INFINITY) {
          stack[size] = nd.left;
          estack[size++] = le;
        }
        if (ri != INFINITY) {
          stack[size] = nd.right;
          estack[size++] = ri;
        }
      }
    }
    return best;
  }

  // --- path tracer (PathTracer.radiance, iterative form of the same recursion) ---
  d3 radiance(d3 p, d3 d, int depth, Sampler& sm, d3 bg) const {
    d3 result = mk(0, 0, 0);
    d3 weight = mk(1, 1, 1);
    for (; depth > 0; --depth) {
      Hit h = first_hit(p, d, 1e-9);
      if (h.t == INFINITY) {
        result = result + mul(weight, bg);
        break;
      }
      const Material& m = materials[h.material];
      result = result + mul(weight, m.emittance);
      if (m.m == 0) break;
      d3 i = mk(-d.x, -d.y, -d.z);
      d3 n = h.n;
      int lobe;
      double prob = 1.0;
      if (m.m == 1) {
        lobe = m.lobe[0];
      } else if (m.m == 2) {
        double u = sm.uniform();
        double k1 = 1.0 - m.w[0];
        lobe = u < k1 ? m.lobe[1] : m.lobe[0];
        prob = u < k1 ? k1 : 1.0 - k1;
      } else {
        double u = sm.uniform();
        double s = 0;
        int j = 0;
        while (s <= u && j < 3) s += m.w[j++];
        j--;
        lobe = m.lobe[j];
        prob = m.w[j];
      }
      d3 out, c;
      if (lobe == 0) {
        double x, y, z, l2;
        do {
          x = 2 * sm.uniform() - 1;
          y = 2 * sm.uniform() - 1;
          z = 2 * sm.uniform() - 1;
          l2 = x * x + y * y + z * z;
        } while (l2 > 1);
        double k = 1 / std::sqrt(l2);
        out = mk(x * k, y * k, z * k) + n;
        c = m.diffuse;
      } else if (lobe == 1) {
        out = n * (2 * dot(i, n)) - i;
        c = m.reflective;
      } else {
        d3 iu = normalized(i);
        double c1 = dot(iu, n);
        double ri = c1 >= 0 ? m.ior : -1.0 / m.ior;
        double c2 = 1 - (1 - c1 * c1) / (ri * ri);
        out = c2 > 0 ? n * (c1 - std::sqrt(c2) * ri) - iu : n * (2 * dot(iu, n)) - iu;
        c = m.refractive;
      }
      c = c * (1.0 / prob);
      if (c.x == 0 && c.y == 0 && c.z == 0) break;
      p = p + d * h.t;
      d = out;
      weight = mul(weight, c);
    }
    return result;
  }
};

inline double lum(d3 c) { return 0.212655 * c.x + 0.715158 * c.y + 0.072187 * c.z; }

void setup(CpuScene& sc, const float* const* arrays, const int* counts) {
  sc.spheres = arrays[0];
  sc.ns = counts[0];
  sc.boxes = arrays[1];
  sc.nb = counts[1];
  sc.planes = arrays[2];
  sc.np = counts[2];
  sc.aspheres = arrays[3];
  sc.nas = counts[3];
  sc.aboxes = arrays[4];
  sc.nab = counts[4];
  const float* M = arrays[5];
  sc.materials.resize(counts[5]);
  for (int i = 0; i < counts[5]; ++i) {
    const float* m = M + 13 * i;
    Material& mt = sc.materials[i];
    mt.diffuse = mk(m[0], m[1], m[2]);
    mt.reflective = mk(m[3], m[4], m[5]);
    mt.refractive = mk(m[6], m[7], m[8]);
    mt.emittance = mk(m[9], m[10], m[11]);
    mt.ior = m[12];
    double w[3] = {lum(mt.diffuse), lum(mt.reflective), lum(mt.refractive)};
    double sum = 0;
    mt.m = 0;
    for (int k = 0; k < 3; ++k)
      if (w[k] > 0) {
        sum += w[k];
        mt.m++;
      }
    int j = 0;
    for (int k = 0; k < 3; ++k)
      if (w[k] > 0) {
        mt.lobe[j] = k;
        mt.w[j] = w[k] / sum;
        j++;
      }
  }
  auto widen = [](Prim& p, double* mn, double* mx) {
    for (int k = 0; k < 3; ++k) {
      p.bmin[k] = next_down(next_down(mn[k]));
      p.bmax[k] = next_up(next_up(mx[k]));
      p.cen[k] = (p.bmin[k] + p.bmax[k]) * 0.5;
    }
  };
  int order = 0;
  for (int i = 0; i < sc.ns; ++i, ++order) {
    const float* s = sc.spheres + 5 * i;
    Prim p{SPHERE, i, order};
    double mn[3] = {s[0] - (double)s[3], s[1] - (double)s[3], s[2] - (double)s[3]};
    double mx[3] = {s[0] + (double)s[3], s[1] + (double)s[3], s[2] + (double)s[3]};
    widen(p, mn, mx);
    sc.prims.push_back(p);
  }
  for (int i = 0; i < sc.nb; ++i, ++order) {
    const float* b = sc.boxes + 7 * i;
    Prim p{BOX, i, order};
    double mn[3] = {b[0], b[1], b[2]}, mx[3] = {b[3], b[4], b[5]};
    widen(p, mn, mx);
    sc.prims.push_back(p);
  }
  for (int kind = ASPHERE; kind <= ABOX; ++kind) {
    int n = kind == ASPHERE ? sc.nas : sc.nab;
    const float* base = kind == ASPHERE ? sc.aspheres : sc.aboxes;
    for (int i = 0; i < n; ++i, ++order) {
      const float* a = base + 22 * i;
      // Forward linear map = inverse of the packed object-space map; bounds from its rows
      // (row lengths for the unit ball, row absolute sums for the unit box).
      double m[9] = {a[0], a[1], a[2], a[4], a[5], a[6], a[8], a[9], a[10]};
      double det = m[0] * (m[4] * m[8] - m[5] * m[7]) - m[1] * (m[3] * m[8] - m[5] * m[6]) +
                   m[2] * (m[3] * m[7] - m[4] * m[6]);
      double f[9] = {(m[4] * m[8] - m[5] * m[7]) / det, -(m[1] * m[8] - m[2] * m[7]) / det,
                     (m[1] * m[5] - m[2] * m[4]) / det, -(m[3] * m[8] - m[5] * m[6]) / det,
                     (m[0] * m[8] - m[2] * m[6]) / det, -(m[0] * m[5] - m[2] * m[3]) / det,
                     (m[3] * m[7] - m[4] * m[6]) / det, -(m[0] * m[7] - m[1] * m[6]) / det,
                     (m[0] * m[4] - m[1] * m[3]) / det};
      double c[3] = {a[3], a[7], a[11]};
      double mn[3], mx[3];
      for (int r = 0; r < 3; ++r) {
        double e = kind == ASPHERE
                       ? std::sqrt(f[3 * r] * f[3 * r] + f[3 * r + 1] * f[3 * r + 1] +
                                   f[3 * r + 2] * f[3 * r + 2])
                       : std::fabs(f[3 * r]) + std::fabs(f[3 * r + 1]) + std::fabs(f[3 * r + 2]);
        mn[r] = c[r] - e;
        mx[r] = c[r] + e;
      }
      Prim p{kind, i, order};
      widen(p, mn, mx);
      sc.prims.push_back(p);
    }
  }
  if (!sc.prims.empty()) sc.build(0, (int)sc.prims.size());
}

}  // namespace

extern "C" {

// Renders `frames` one-sample frames of rows [row_begin, row_end) of a width x height
// image and returns the per-pixel mean in rgb (3 doubles per pixel of the row range).
// camera: pos, forward, right, up (12 floats, the GPU camera of the same scene);
// params: width, height, frames, max_depth; threads: OpenMP threads (<= 0: all).
// Returns the number of BVH nodes built (for reporting).
int orc_cpu_render(const float* const* arrays, const int* counts, const float* camera,
                   const float* background, const int* params, unsigned long long seed,
                   int row_begin, int row_end, int threads, double* rgb) {
  CpuScene sc;
  setup(sc, arrays, counts);
  int width = params[0], height = params[1], frames = params[2], depth = params[3];
  d3 cp = mk(camera[0], camera[1], camera[2]);
  d3 cf = mk(camera[3], camera[4], camera[5]);
  d3 cr = mk(camera[6], camera[7], camera[8]);
  d3 cu = mk(camera[9], camera[10], camera[11]);
  d3 bg = mk(background[0], background[1], background[2]);
  double aspect = width / (double)height;
  int rows = row_end - row_begin;
  std::memset(rgb, 0, sizeof(double) * 3 * (size_t)rows * width);
  int nthreads = threads > 0 ? threads : omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) num_threads(nthreads)
  for (int yy = 0; yy < rows; ++yy) {
    int y = row_begin + yy;
    for (int frame = 0; frame < frames; ++frame) {
      for (int x = 0; x < width; ++x) {
        auto s01 = [&](int dim) {
          uint64_t key = seed ^ ((uint64_t)frame * 0x9E3779B97F4A7C15ULL) ^
                         ((uint64_t)x * 0xC2B2AE3D27D4EB4FULL) ^
                         ((uint64_t)y * 0x165667B19E3779F9ULL) ^
                         ((uint64_t)dim * 0xD6E8FEB86659FD93ULL);
          return (double)(mix64(key) >> 11) * 0x1.0p-53;
        };
        double sx = (-1.0 + 2.0 * (x + s01(0)) / width) * aspect;
        double sy = 1.0 - 2.0 * (y + s01(1)) / height;
        d3 dir = cf + cr * sx + cu * sy;
        Sampler sm{hash_u32((uint32_t)(y * width + x) ^ hash_u32((uint32_t)frame * 0x9E3779B9u) ^
                            (uint32_t)seed)};
        d3 c = sc.radiance(cp, dir, depth, sm, bg);
        double* o = rgb + 3 * ((size_t)yy * width + x);
        o[0] += c.x;
        o[1] += c.y;
        o[2] += c.z;
      }
    }
    for (int x = 0; x < width; ++x)
      for (int k = 0; k < 3; ++k) rgb[3 * ((size_t)yy * width + x) + k] /= frames;
  }
  return (int)sc.nodes.size();
}

}  // extern "C"
