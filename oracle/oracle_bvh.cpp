// Oracle (test infrastructure only): a CPU restatement of the reference's host-side
// BVH builder for the GPU path tracer.  Only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg may load this code; the product never does.
//
// Restated from the reference (paths relative to the reference project,
// gfxlab/ = src/xyz/marsavic/gfxlab/):
//   * primitive bounds      gfxlab/gpu/GpuScene.java:626-649, 840-903
//                           (spheres from float centre +/- float radius, boxes from the
//                           packed float corners, affines from the float-cast bounds; each
//                           widened by two float ulps: nextDown2 / nextUp2)
//   * centroid              gfxlab/gpu/GpuScene.java:78-80   ((min + max) * 0.5 in double)
//   * BvhBuildState.build   gfxlab/gpu/GpuScene.java:1424-1447
//   * bestSplit             gfxlab/gpu/GpuScene.java:1453-1488  (full sweep on every axis
//                           whose centroid extent exceeds 1e-12; sort key (centroid, order)
//                           with Double.compare; sequential prefix/suffix weight sums;
//                           strict '<' keeps the first minimum)
//   * weights               gfxlab/gpu/BvhBuildConfig.java:66-69  (q = 1 + lambda (c - 1))
//   * per-type forest       gfxlab/gpu/GpuScene.java:702-720
//   * flattenBvh / leafKind gfxlab/gpu/GpuScene.java:772-808   (preorder)
//   * SAH statistics        gfxlab/gpu/GpuScene.java:810-838
//   * BvhRotator            gfxlab/gpu/GpuScene.java:968-1057  (Kensler-style local
//                           rotations after the SAH build, for the *_ROTATIONS modes:
//                           bottom-up, four candidates per node, recursive areaCost,
//                           strict improvement by more than 1e-12, up to rotationPasses
//                           passes while any rotation happened)
//   * SpatialBuildState     gfxlab/gpu/GpuScene.java:1084-1412  (the SBVH modes: depth-first
//                           recursion comparing the object split with the best of
//                           spatialBins - 1 planes per axis, clipped duplicates under the
//                           global budget floor(N * maxReferenceMultiplier), the greedy
//                           unsplit pass over the split references in list order; leaves
//                           collect the (clipped) references in visit order)
// Arithmetic is IEEE double with no contraction (Java strictfp semantics); this file
// must be compiled with -ffp-contract=off.
//
// orc_build_bvh_binned restates this library's binned object-SAH mode (no reference
// counterpart; the reference builder is the full sweep above):
//   * per axis whose centroid extent exceeds 1e-12, B bins over the node's centroid bounds,
//     bin = min(B - 1, (int)((c - lo) * (B / extent)));
//   * per bin, integer counts per primitive type and the float box union;
//   * the weight of a set is ((n0 w0 + n1 w1) + n2 w2) + n3 w3 with the per-type
//     construction weights, so sums do not depend on the order of accumulation;
//   * plane j (1..B-1) puts bins [0, j) left; cost (A_P c_T + A_L W_L) + A_R W_R; first
//     minimum over (axis, j); both sides non-empty;
//   * leaf if count == 1, or count <= leafSize and !(cost < A_P W_P); a node whose
//     centroids coincide on every axis becomes a leaf when count <= leafSize and otherwise
//     splits at count / 2 in its current order;
//   * children are a stable partition of the node's primitives.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

constexpr int REF_TYPE_MASK = (int)0xC0000000u;
constexpr int REF_TYPE_SPHERE = 0x00000000;
constexpr int REF_TYPE_BOX = 0x40000000;
constexpr int REF_TYPE_AFFINE_SPHERE = (int)0x80000000u;
constexpr int REF_TYPE_AFFINE_BOX = (int)0xC0000000u;

struct Aabb {
  double mn[3], mx[3];
};

inline double surface_area(const Aabb& b) {
  double dx = b.mx[0] - b.mn[0];
  double dy = b.mx[1] - b.mn[1];
  double dz = b.mx[2] - b.mn[2];
  double a = dx * dy;
  double c = dx * dz;
  double s = a + c;
  double e = dy * dz;
  s = s + e;
  return 2.0 * s;
}

inline Aabb unite(const Aabb& a, const Aabb& b) {
  Aabb r;
  for (int k = 0; k < 3; ++k) {
    r.mn[k] = std::min(a.mn[k], b.mn[k]);
    r.mx[k] = std::max(a.mx[k], b.mx[k]);
  }
  return r;
}

struct Prim {
  int ref;
  int order;
  Aabb bounds;
  double cen[3];
  double measured;  // c_i, the raw per-type weight
};

// Double.compare semantics for finite values (-0.0 orders before +0.0).
inline int java_double_compare(double a, double b) {
  if (a < b) return -1;
  if (a > b) return 1;
  int64_t ia, ib;
  std::memcpy(&ia, &a, 8);
  std::memcpy(&ib, &b, 8);
  return ia == ib ? 0 : (ia < ib ? -1 : 1);
}

inline float next_down2(float v) { return std::nextafter(std::nextafter(v, -INFINITY), -INFINITY); }
inline float next_up2(float v) { return std::nextafter(std::nextafter(v, INFINITY), INFINITY); }

struct Node {
  Aabb bounds;
  int left = -1, right = -1;  // indices into the node pool, -1 for leaves
  int start = -1, end = -1;
};

struct Config {
  int weighted;
  int leaf_size;
  double traversal;
  double lambda;
  int bins = 0;               // 0: full sweep; 2..32: binned mode
  double type_weight[4] = {1.0, 1.0, 1.0, 1.0};
};

inline int type_of(int ref) { return (int)((unsigned)ref >> 30); }

inline int bin_of(double c, double lo, double scale, int bins) {
  double x = c - lo;
  x = x * scale;
  int b = (int)x;
  return b < bins ? b : bins - 1;
}

struct Builder {
  std::vector<Prim>& prims;
  const Config& cfg;
  std::vector<Node> pool;

  Builder(std::vector<Prim>& p, const Config& c) : prims(p), cfg(c) {}

  double objective(const Prim& p) const {
    if (!cfg.weighted) return 1.0;
    double t = p.measured - 1.0;
    t = cfg.lambda * t;
    return 1.0 + t;
  }

  int make_leaf(const Aabb& b, int s, int e) {
    Node n;
    n.bounds = b;
    n.start = s;
    n.end = e;
    pool.push_back(n);
    return (int)pool.size() - 1;
  }

  struct Split {
    bool valid = false;
    std::vector<Prim> sorted;
    int left_count = 0;
    double cost = 0.0;
  };

  Split best_split(int start, int end, const Aabb& bounds, const Aabb& cb) {
    int count = end - start;
    double node_area = surface_area(bounds);
    Split best;
    std::vector<Aabb> prefix(count), suffix(count);
    std::vector<double> pw(count), sw(count);
    for (int axis = 0; axis < 3; ++axis) {
      if (!(cb.mx[axis] - cb.mn[axis] > 1.0e-12)) continue;
      std::vector<Prim> sorted(prims.begin() + start, prims.begin() + end);
      std::stable_sort(sorted.begin(), sorted.end(), [axis](const Prim& a, const Prim& b) {
        int c = java_double_compare(a.cen[axis], b.cen[axis]);
        if (c != 0) return c < 0;
        return a.order < b.order;
      });
      prefix[0] = sorted[0].bounds;
      pw[0] = objective(sorted[0]);
      for (int i = 1; i < count; ++i) {
        prefix[i] = unite(prefix[i - 1], sorted[i].bounds);
        pw[i] = pw[i - 1] + objective(sorted[i]);
      }
      suffix[count - 1] = sorted[count - 1].bounds;
      sw[count - 1] = objective(sorted[count - 1]);
      for (int i = count - 2; i >= 0; --i) {
        suffix[i] = unite(suffix[i + 1], sorted[i].bounds);
        sw[i] = sw[i + 1] + objective(sorted[i]);
      }
      bool improved = false;
      int best_i = 0;
      double best_cost = best.valid ? best.cost : 0.0;
      bool have = best.valid;
      for (int i = 1; i < count; ++i) {
        double a = node_area * cfg.traversal;
        double b = surface_area(prefix[i - 1]) * pw[i - 1];
        double c = surface_area(suffix[i]) * sw[i];
        double cost = (a + b) + c;
        if (!have || cost < best_cost) {
          have = true;
          best_cost = cost;
          best_i = i;
          improved = true;
        }
      }
      if (improved) {
        best.valid = true;
        best.cost = best_cost;
        best.left_count = best_i;
        best.sorted = std::move(sorted);
      }
    }
    return best;
  }

  double set_weight(const long long* cnt) const {
    double w = (double)cnt[0] * cfg.type_weight[0];
    w = w + (double)cnt[1] * cfg.type_weight[1];
    w = w + (double)cnt[2] * cfg.type_weight[2];
    w = w + (double)cnt[3] * cfg.type_weight[3];
    return w;
  }

  struct BinnedSplit {
    bool valid = false;
    int axis = 0, plane = 0, left_count = 0;
    double lo = 0.0, scale = 0.0, cost = 0.0;
  };

  BinnedSplit binned_split(int start, int end, const Aabb& bounds, const Aabb& cb) {
    const int B = cfg.bins;
    double node_area = surface_area(bounds);
    BinnedSplit best;
    for (int axis = 0; axis < 3; ++axis) {
      double ext = cb.mx[axis] - cb.mn[axis];
      if (!(ext > 1.0e-12)) continue;
      double scale = (double)B / ext;
      std::vector<Aabb> box(B);
      std::vector<long long> cnt(4 * B, 0);
      std::vector<bool> used(B, false);
      for (int i = start; i < end; ++i) {
        const Prim& p = prims[i];
        int b = bin_of(p.cen[axis], cb.mn[axis], scale, B);
        box[b] = used[b] ? unite(box[b], p.bounds) : p.bounds;
        used[b] = true;
        cnt[4 * b + type_of(p.ref)]++;
      }
      // inclusive prefix (left) and suffix (right) over bins
      std::vector<Aabb> lbox(B), rbox(B);
      std::vector<long long> lc(4 * B), rc(4 * B);
      std::vector<bool> lu(B), ru(B);
      for (int b = 0; b < B; ++b) {
        for (int t = 0; t < 4; ++t) lc[4 * b + t] = cnt[4 * b + t] + (b ? lc[4 * (b - 1) + t] : 0);
        if (b && lu[b - 1]) {
          lbox[b] = used[b] ? unite(lbox[b - 1], box[b]) : lbox[b - 1];
          lu[b] = true;
        } else {
          lbox[b] = box[b];
          lu[b] = used[b];
        }
      }
      for (int b = B - 1; b >= 0; --b) {
        for (int t = 0; t < 4; ++t)
          rc[4 * b + t] = cnt[4 * b + t] + (b + 1 < B ? rc[4 * (b + 1) + t] : 0);
        if (b + 1 < B && ru[b + 1]) {
          rbox[b] = used[b] ? unite(rbox[b + 1], box[b]) : rbox[b + 1];
          ru[b] = true;
        } else {
          rbox[b] = box[b];
          ru[b] = used[b];
        }
      }
      for (int j = 1; j < B; ++j) {
        const long long* L = &lc[4 * (j - 1)];
        const long long* R = &rc[4 * j];
        long long nl = L[0] + L[1] + L[2] + L[3];
        long long nr = R[0] + R[1] + R[2] + R[3];
        if (nl == 0 || nr == 0) continue;
        double a = node_area * cfg.traversal;
        double bl = surface_area(lbox[j - 1]) * set_weight(L);
        double br = surface_area(rbox[j]) * set_weight(R);
        double cost = (a + bl) + br;
        if (!best.valid || cost < best.cost) {
          best.valid = true;
          best.cost = cost;
          best.axis = axis;
          best.plane = j;
          best.left_count = (int)nl;
          best.lo = cb.mn[axis];
          best.scale = scale;
        }
      }
    }
    return best;
  }

  int build_binned(int start, int end) {
    Aabb bounds = prims[start].bounds;
    Aabb cb;
    for (int k = 0; k < 3; ++k) cb.mn[k] = cb.mx[k] = prims[start].cen[k];
    long long cnt[4] = {0, 0, 0, 0};
    for (int i = start; i < end; ++i) {
      if (i > start) bounds = unite(bounds, prims[i].bounds);
      for (int k = 0; k < 3; ++k) {
        cb.mn[k] = std::min(cb.mn[k], prims[i].cen[k]);
        cb.mx[k] = std::max(cb.mx[k], prims[i].cen[k]);
      }
      cnt[type_of(prims[i].ref)]++;
    }
    int count = end - start;
    if (count == 1) return make_leaf(bounds, start, end);
    BinnedSplit split = binned_split(start, end, bounds, cb);
    int mid;
    if (!split.valid) {
      if (count <= cfg.leaf_size) return make_leaf(bounds, start, end);
      mid = start + count / 2;
    } else {
      double leaf_cost = surface_area(bounds) * set_weight(cnt);
      if (count <= cfg.leaf_size && !(split.cost < leaf_cost)) return make_leaf(bounds, start, end);
      std::vector<Prim> left, right;
      for (int i = start; i < end; ++i) {
        int b = bin_of(prims[i].cen[split.axis], split.lo, split.scale, cfg.bins);
        (b < split.plane ? left : right).push_back(prims[i]);
      }
      std::copy(left.begin(), left.end(), prims.begin() + start);
      std::copy(right.begin(), right.end(), prims.begin() + start + left.size());
      mid = start + (int)left.size();
    }
    int l = build_binned(start, mid);
    int r = build_binned(mid, end);
    Node n;
    n.bounds = bounds;
    n.left = l;
    n.right = r;
    pool.push_back(n);
    return (int)pool.size() - 1;
  }

  int build(int start, int end) {
    if (cfg.bins > 0) return build_binned(start, end);
    Aabb bounds = prims[start].bounds;
    Aabb cb;
    for (int k = 0; k < 3; ++k) cb.mn[k] = cb.mx[k] = prims[start].cen[k];
    for (int i = start + 1; i < end; ++i) {
      bounds = unite(bounds, prims[i].bounds);
      for (int k = 0; k < 3; ++k) {
        cb.mn[k] = std::min(cb.mn[k], prims[i].cen[k]);
        cb.mx[k] = std::max(cb.mx[k], prims[i].cen[k]);
      }
    }
    int count = end - start;
    if (count == 1) return make_leaf(bounds, start, end);
    Split split = best_split(start, end, bounds, cb);
    if (!split.valid) return make_leaf(bounds, start, end);
    double wsum = 0.0;
    for (int i = start; i < end; ++i) wsum += objective(prims[i]);
    double leaf_cost = surface_area(bounds) * wsum;
    if (count <= cfg.leaf_size && !(split.cost < leaf_cost)) return make_leaf(bounds, start, end);
    std::copy(split.sorted.begin(), split.sorted.end(), prims.begin() + start);
    int mid = start + split.left_count;
    int l = build(start, mid);
    int r = build(mid, end);
    Node n;
    n.bounds = bounds;
    n.left = l;
    n.right = r;
    pool.push_back(n);
    return (int)pool.size() - 1;
  }
};

// BvhRotator (GpuScene.java:968-1057) over a Builder's node pool.
struct Rotator {
  Builder& b;
  explicit Rotator(Builder& bb) : b(bb) {}

  int join(int l, int r) {
    Node n;
    n.bounds = unite(b.pool[l].bounds, b.pool[r].bounds);
    n.left = l;
    n.right = r;
    b.pool.push_back(n);
    return (int)b.pool.size() - 1;
  }

  // areaCost: recursive over the candidate's subtree
  double area_cost(int n) {
    const Node nd = b.pool[n];
    if (nd.left < 0) {
      double w = 0.0;
      for (int i = nd.start; i < nd.end; ++i) w += b.objective(b.prims[i]);
      return surface_area(nd.bounds) * w;
    }
    double x = surface_area(nd.bounds) * b.cfg.traversal;
    x = x + area_cost(nd.left);
    return x + area_cost(nd.right);
  }

  // optimizePass: returns the (possibly new) root of the subtree; counts rotations
  int pass(int n, int& rotations) {
    if (b.pool[n].left < 0) return n;
    int l = pass(b.pool[n].left, rotations);
    int r = pass(b.pool[n].right, rotations);
    int current = join(l, r);
    int best = current;
    double best_cost = area_cost(current);
    const double eps = 1.0e-12;
    if (b.pool[b.pool[current].left].left >= 0) {
      int L = b.pool[current].left;
      int a = b.pool[L].left, bb = b.pool[L].right, c = b.pool[current].right;
      int cand = join(a, join(bb, c));
      double cost = area_cost(cand);
      if (cost < best_cost - eps) {
        best = cand;
        best_cost = cost;
      }
      cand = join(bb, join(a, c));
      cost = area_cost(cand);
      if (cost < best_cost - eps) {
        best = cand;
        best_cost = cost;
      }
    }
    if (b.pool[b.pool[current].right].left >= 0) {
      int R = b.pool[current].right;
      int a = b.pool[current].left, bb = b.pool[R].left, c = b.pool[R].right;
      int cand = join(join(a, c), bb);
      double cost = area_cost(cand);
      if (cost < best_cost - eps) {
        best = cand;
        best_cost = cost;
      }
      cand = join(join(a, bb), c);
      cost = area_cost(cand);
      if (cost < best_cost - eps) best = cand;
    }
    if (best != current) rotations++;
    return best;
  }

  int optimize(int root, int passes, int& total) {
    total = 0;
    for (int p = 0; p < passes; ++p) {
      int rot = 0;
      root = pass(root, rot);
      total += rot;
      if (rot == 0) break;
    }
    return root;
  }
};

struct Summary {
  int nodes = 0, leaves = 0, max_depth = 0, min_leaf = INT32_MAX, max_leaf = 0;
};

void summarize(const std::vector<Node>& pool, int n, int depth, Summary& s) {
  s.nodes++;
  s.max_depth = std::max(s.max_depth, depth);
  const Node& nd = pool[n];
  if (nd.left < 0) {
    int occ = nd.end - nd.start;
    s.leaves++;
    s.min_leaf = std::min(s.min_leaf, occ);
    s.max_leaf = std::max(s.max_leaf, occ);
    return;
  }
  summarize(pool, nd.left, depth + 1, s);
  summarize(pool, nd.right, depth + 1, s);
}

int leaf_kind(const std::vector<Prim>& p, int s, int e) {
  int type = p[s].ref & REF_TYPE_MASK;
  for (int i = s + 1; i < e; ++i)
    if ((p[i].ref & REF_TYPE_MASK) != type) return -1;
  switch (type) {
    case REF_TYPE_SPHERE: return -2;
    case REF_TYPE_BOX: return -3;
    case REF_TYPE_AFFINE_SPHERE: return -4;
    default: return -5;
  }
}

struct Flat {
  float* bounds;
  int* data;
  int* refs;
  int next_node = 0;
  int next_ref = 0;
};

int flatten(const std::vector<Node>& pool, int n, const std::vector<Prim>& p, Flat& f) {
  int index = f.next_node++;
  const Node& nd = pool[n];
  for (int k = 0; k < 3; ++k) {
    f.bounds[index * 6 + k] = (float)nd.bounds.mn[k];
    f.bounds[index * 6 + 3 + k] = (float)nd.bounds.mx[k];
  }
  int* d = f.data + index * 4;
  if (nd.left < 0) {
    d[0] = leaf_kind(p, nd.start, nd.end);
    d[1] = -1;
    d[2] = f.next_ref;
    d[3] = nd.end - nd.start;
    for (int i = nd.start; i < nd.end; ++i) f.refs[f.next_ref++] = p[i].ref;
    return index;
  }
  int l = flatten(pool, nd.left, p, f);
  int r = flatten(pool, nd.right, p, f);
  d[0] = l;
  d[1] = r;
  d[2] = -1;
  d[3] = 0;
  return index;
}

// sahCost / constructionSahCost (GpuScene.java:810-838).  mode 0: unit weights,
// 1: measured weights, 2: construction weights.
double sah_cost(const std::vector<Node>& pool, int n, const std::vector<Prim>& p, int mode,
                const Builder& b) {
  const Node& nd = pool[n];
  if (nd.left < 0) {
    double c = 0.0;
    for (int i = nd.start; i < nd.end; ++i)
      c += mode == 0 ? 1.0 : (mode == 1 ? p[i].measured : b.objective(p[i]));
    return c;
  }
  double area = surface_area(nd.bounds);
  if (!(area > 0.0)) return sah_cost(pool, nd.left, p, mode, b) + sah_cost(pool, nd.right, p, mode, b);
  double l = surface_area(pool[nd.left].bounds) / area * sah_cost(pool, nd.left, p, mode, b);
  double r = surface_area(pool[nd.right].bounds) / area * sah_cost(pool, nd.right, p, mode, b);
  return (b.cfg.traversal + l) + r;
}

// ---- SpatialBuildState (GpuScene.java:1084-1412)
struct SRef {
  int ref;
  int order;
  Aabb bounds;
  double measured;
  int split_depth;
};

inline double sref_centroid(const SRef& r, int axis) { return (r.bounds.mn[axis] + r.bounds.mx[axis]) * 0.5; }

// Record equality of SpatialReference (List.remove(Object) removes the first equal element).
inline bool sref_equal(const SRef& a, const SRef& b) {
  if (a.ref != b.ref || a.order != b.order || a.split_depth != b.split_depth) return false;
  if (std::memcmp(&a.measured, &b.measured, 8) != 0) return false;
  return std::memcmp(&a.bounds, &b.bounds, sizeof(Aabb)) == 0;
}

struct SpatialOptions {
  int bins;
  double max_reference_multiplier;
  int max_splits_per_primitive;
  int min_spatial_references;
  double overlap_threshold;
};

struct ObjectSplit {
  std::vector<SRef> sorted;
  int left_count = 0;
  double cost = 0.0;
  Aabb left_bounds, right_bounds;
  bool valid = false;
};

struct SpatialBuilder {
  const Config& cfg;
  SpatialOptions opt;
  int max_refs;
  int current;
  int spatial_splits = 0;
  std::vector<Node> pool;
  std::vector<Prim> ordered;  // leaf references in visit order (clipped bounds)
  static constexpr double EPS = 1.0e-12;

  SpatialBuilder(const Config& c, const SpatialOptions& o, int n) : cfg(c), opt(o), current(n) {
    max_refs = std::max(n, (int)std::floor((double)n * o.max_reference_multiplier));
  }

  double objective(const SRef& r) const {
    if (!cfg.weighted) return 1.0;
    double t = r.measured - 1.0;
    t = cfg.lambda * t;
    return 1.0 + t;
  }

  double weight_sum(const std::vector<SRef>& v) const {
    double s = 0.0;
    for (const SRef& r : v) s += objective(r);
    return s;
  }

  static Aabb bounds_of(const std::vector<SRef>& v) {
    Aabb b = v[0].bounds;
    for (size_t i = 1; i < v.size(); ++i) b = unite(b, v[i].bounds);
    return b;
  }

  int leaf(const Aabb& b, const std::vector<SRef>& refs) {
    Node nd;
    nd.bounds = b;
    nd.start = (int)ordered.size();
    for (const SRef& r : refs) {
      Prim p{};
      p.ref = r.ref;
      p.order = r.order;
      p.bounds = r.bounds;
      p.measured = r.measured;
      ordered.push_back(p);
    }
    nd.end = (int)ordered.size();
    pool.push_back(nd);
    return (int)pool.size() - 1;
  }

  ObjectSplit best_object_split(const std::vector<SRef>& refs, const Aabb& node_bounds) {
    ObjectSplit best;
    const int count = (int)refs.size();
    for (int axis = 0; axis < 3; ++axis) {
      std::vector<SRef> sorted = refs;
      std::sort(sorted.begin(), sorted.end(), [axis](const SRef& a, const SRef& b) {
        int cmp = java_double_compare(sref_centroid(a, axis), sref_centroid(b, axis));
        return cmp != 0 ? cmp < 0 : a.order < b.order;
      });
      std::vector<Aabb> prefix(count), suffix(count);
      std::vector<double> pw(count), sw(count);
      prefix[0] = sorted[0].bounds;
      pw[0] = objective(sorted[0]);
      for (int i = 1; i < count; ++i) {
        prefix[i] = unite(prefix[i - 1], sorted[i].bounds);
        pw[i] = pw[i - 1] + objective(sorted[i]);
      }
      suffix[count - 1] = sorted[count - 1].bounds;
      sw[count - 1] = objective(sorted[count - 1]);
      for (int i = count - 2; i >= 0; --i) {
        suffix[i] = unite(suffix[i + 1], sorted[i].bounds);
        sw[i] = sw[i + 1] + objective(sorted[i]);
      }
      for (int i = 1; i < count; ++i) {
        double cost = surface_area(node_bounds) * cfg.traversal;
        cost = cost + surface_area(prefix[i - 1]) * pw[i - 1];
        cost = cost + surface_area(suffix[i]) * sw[i];
        if (!best.valid || cost < best.cost) {
          best.valid = true;
          best.sorted = sorted;
          best.left_count = i;
          best.cost = cost;
          best.left_bounds = prefix[i - 1];
          best.right_bounds = suffix[i];
        }
      }
    }
    return best;
  }

  bool should_attempt_spatial(const std::vector<SRef>& refs, const Aabb& node_bounds,
                              const ObjectSplit& os) const {
    if ((int)refs.size() < opt.min_spatial_references || current >= max_refs) return false;
    Aabb ov;
    bool empty = false;
    for (int k = 0; k < 3; ++k) {
      ov.mn[k] = std::max(os.left_bounds.mn[k], os.right_bounds.mn[k]);
      ov.mx[k] = std::min(os.left_bounds.mx[k], os.right_bounds.mx[k]);
    }
    for (int k = 0; k < 3; ++k)
      if (ov.mx[k] <= ov.mn[k]) empty = true;
    double overlap = empty ? 0.0 : surface_area(ov);
    return overlap / std::max(surface_area(node_bounds), 1.0e-30) > opt.overlap_threshold;
  }

  static Aabb clip_max(const Aabb& b, int axis, double v) {
    Aabb r = b;
    r.mx[axis] = std::min(b.mx[axis], v);
    return r;
  }
  static Aabb clip_min(const Aabb& b, int axis, double v) {
    Aabb r = b;
    r.mn[axis] = std::max(b.mn[axis], v);
    return r;
  }

  // best_plane: {axis, position}; false when no plane qualifies
  bool best_spatial_plane(const std::vector<SRef>& refs, const Aabb& node_bounds, int* best_axis,
                          double* best_pos) const {
    bool found = false;
    double best_cost = 0.0;
    for (int axis = 0; axis < 3; ++axis) {
      double lo = node_bounds.mn[axis], hi = node_bounds.mx[axis];
      double extent = hi - lo;
      if (!(extent > EPS)) continue;
      for (int bin = 1; bin < opt.bins; ++bin) {
        double plane = extent * (double)bin;
        plane = plane / (double)opt.bins;
        plane = lo + plane;
        Aabb lb{}, rb{};
        bool has_l = false, has_r = false;
        double lw = 0.0, rw = 0.0;
        int duplicates = 0;
        for (const SRef& r : refs) {
          if (r.bounds.mx[axis] <= plane + EPS) {
            lb = has_l ? unite(lb, r.bounds) : r.bounds;
            has_l = true;
            lw += objective(r);
          } else if (r.bounds.mn[axis] >= plane - EPS) {
            rb = has_r ? unite(rb, r.bounds) : r.bounds;
            has_r = true;
            rw += objective(r);
          } else if (r.split_depth < opt.max_splits_per_primitive) {
            Aabb cl = clip_max(r.bounds, axis, plane), cr = clip_min(r.bounds, axis, plane);
            lb = has_l ? unite(lb, cl) : cl;
            rb = has_r ? unite(rb, cr) : cr;
            has_l = has_r = true;
            double w = objective(r);
            lw += w;
            rw += w;
            duplicates++;
          } else if (sref_centroid(r, axis) <= plane) {
            lb = has_l ? unite(lb, r.bounds) : r.bounds;
            has_l = true;
            lw += objective(r);
          } else {
            rb = has_r ? unite(rb, r.bounds) : r.bounds;
            has_r = true;
            rw += objective(r);
          }
        }
        if (!has_l || !has_r || current + duplicates > max_refs) continue;
        double cost = surface_area(node_bounds) * cfg.traversal;
        cost = cost + surface_area(lb) * lw;
        cost = cost + surface_area(rb) * rw;
        if (!found || cost < best_cost) {
          found = true;
          best_cost = cost;
          *best_axis = axis;
          *best_pos = plane;
        }
      }
    }
    return found;
  }

  static void remove_first_equal(std::vector<SRef>& v, const SRef& x) {
    for (size_t i = 0; i < v.size(); ++i)
      if (sref_equal(v[i], x)) {
        v.erase(v.begin() + i);
        return;
      }
  }

  // partitionSpatial; false when a side would be empty
  bool partition_spatial(const std::vector<SRef>& refs, int axis, double pos, std::vector<SRef>& left,
                         std::vector<SRef>& right, int* duplicates) const {
    struct Choice {
      SRef original, l, r;
    };
    std::vector<Choice> choices;
    for (const SRef& r : refs) {
      double lo = r.bounds.mn[axis], hi = r.bounds.mx[axis];
      if (hi <= pos + EPS) {
        left.push_back(r);
      } else if (lo >= pos - EPS) {
        right.push_back(r);
      } else if (r.split_depth < opt.max_splits_per_primitive) {
        SRef lp = r, rp = r;
        lp.bounds = clip_max(r.bounds, axis, pos);
        lp.split_depth = r.split_depth + 1;
        rp.bounds = clip_min(r.bounds, axis, pos);
        rp.split_depth = r.split_depth + 1;
        left.push_back(lp);
        right.push_back(rp);
        choices.push_back({r, lp, rp});
      } else if (sref_centroid(r, axis) <= pos) {
        left.push_back(r);
      } else {
        right.push_back(r);
      }
    }
    if (left.empty() || right.empty()) return false;
    for (const Choice& ch : choices) {
      Aabb lb = bounds_of(left), rb = bounds_of(right);
      double lw = weight_sum(left), rw = weight_sum(right);
      double w = objective(ch.original);
      double split_cost = surface_area(lb) * lw;
      split_cost = split_cost + surface_area(rb) * rw;
      double left_only = surface_area(unite(lb, ch.original.bounds)) * lw;
      left_only = left_only + surface_area(rb) * std::max(0.0, rw - w);
      double right_only = surface_area(lb) * std::max(0.0, lw - w);
      right_only = right_only + surface_area(unite(rb, ch.original.bounds)) * rw;
      if (left_only < split_cost && left_only <= right_only && right.size() > 1) {
        remove_first_equal(left, ch.l);
        remove_first_equal(right, ch.r);
        left.push_back(ch.original);
      } else if (right_only < split_cost && left.size() > 1) {
        remove_first_equal(left, ch.l);
        remove_first_equal(right, ch.r);
        right.push_back(ch.original);
      }
    }
    *duplicates = (int)(left.size() + right.size()) - (int)refs.size();
    return true;
  }

  double split_cost(const std::vector<SRef>& left, const std::vector<SRef>& right,
                    const Aabb& node_bounds) const {
    double c = surface_area(node_bounds) * cfg.traversal;
    c = c + surface_area(bounds_of(left)) * weight_sum(left);
    c = c + surface_area(bounds_of(right)) * weight_sum(right);
    return c;
  }

  int build(const std::vector<SRef>& refs) {
    Aabb b = bounds_of(refs);
    if (refs.size() == 1) return leaf(b, refs);
    ObjectSplit os = best_object_split(refs, b);
    std::vector<SRef> sl, sr;
    bool have_spatial = false;
    int dup = 0;
    double spatial_cost = INFINITY;
    if (should_attempt_spatial(refs, b, os)) {
      int axis = 0;
      double pos = 0.0;
      if (best_spatial_plane(refs, b, &axis, &pos)) {
        std::vector<SRef> cl, cr;
        int d = 0;
        if (partition_spatial(refs, axis, pos, cl, cr, &d) && current + d <= max_refs) {
          spatial_cost = split_cost(cl, cr, b);
          sl.swap(cl);
          sr.swap(cr);
          dup = d;
          have_spatial = true;
        }
      }
    }
    double leaf_cost = surface_area(b) * weight_sum(refs);
    bool choose_spatial = have_spatial && spatial_cost < os.cost;
    double best_cost = choose_spatial ? spatial_cost : os.cost;
    if ((int)refs.size() <= cfg.leaf_size && !(best_cost < leaf_cost)) return leaf(b, refs);
    std::vector<SRef> left, right;
    if (choose_spatial) {
      left.swap(sl);
      right.swap(sr);
      current += dup;
      spatial_splits++;
    } else {
      left.assign(os.sorted.begin(), os.sorted.begin() + os.left_count);
      right.assign(os.sorted.begin() + os.left_count, os.sorted.end());
    }
    os.sorted.clear();
    os.sorted.shrink_to_fit();
    int l = build(left);
    int r = build(right);
    Node nd;
    nd.bounds = b;
    nd.left = l;
    nd.right = r;
    pool.push_back(nd);
    return (int)pool.size() - 1;
  }
};

Aabb float_box(float x0, float y0, float z0, float x1, float y1, float z1) {
  Aabb b;
  b.mn[0] = next_down2(x0);
  b.mn[1] = next_down2(y0);
  b.mn[2] = next_down2(z0);
  b.mx[0] = next_up2(x1);
  b.mx[1] = next_up2(y1);
  b.mx[2] = next_up2(z1);
  return b;
}

}  // namespace

extern "C" {

// Build configuration; mirrors gfxlab/gpu/BvhBuildConfig.java:6-15.  mode follows
// BvhBuildMode ordinals (0 UNIFORM_SAH, 1 WEIGHTED_SAH, 2 PER_TYPE_SAH,
// 3 PER_TYPE_WEIGHTED_SAH); the SBVH and rotation modes are not restated here.
typedef struct {
  int mode;
  int leaf_size;
  double traversal_weight;
  double sphere_weight, box_weight, affine_sphere_weight, affine_box_weight;
  double lambda;
} orc_build_config;

// The bounded primitives in global order (spheres, boxes, affine spheres, affine boxes)
// with their conservative bounds and centroids (GpuScene.java:626-649, 877-903).
static std::vector<Prim> make_prims(const float* spheres, int ns, const float* boxes, int nb,
                                    const float* affine_sphere_bounds, int nas,
                                    const float* affine_box_bounds, int nab,
                                    const orc_build_config* cfg) {
  int total = ns + nb + nas + nab;
  std::vector<Prim> all;
  all.reserve(total);
  int order = 0;
  for (int i = 0; i < ns; ++i, ++order) {
    const float* s = spheres + 5 * i;
    float cx = s[0], cy = s[1], cz = s[2], r = s[3];
    Prim p{};
    p.ref = REF_TYPE_SPHERE | i;
    p.order = order;
    p.bounds = float_box(cx - r, cy - r, cz - r, cx + r, cy + r, cz + r);
    p.measured = cfg->sphere_weight;
    all.push_back(p);
  }
  for (int i = 0; i < nb; ++i, ++order) {
    const float* b = boxes + 7 * i;
    Prim p{};
    p.ref = REF_TYPE_BOX | i;
    p.order = order;
    p.bounds = float_box(b[0], b[1], b[2], b[3], b[4], b[5]);
    p.measured = cfg->box_weight;
    all.push_back(p);
  }
  for (int i = 0; i < nas; ++i, ++order) {
    const float* b = affine_sphere_bounds + 6 * i;
    Prim p{};
    p.ref = REF_TYPE_AFFINE_SPHERE | i;
    p.order = order;
    p.bounds = float_box(b[0], b[1], b[2], b[3], b[4], b[5]);
    p.measured = cfg->affine_sphere_weight;
    all.push_back(p);
  }
  for (int i = 0; i < nab; ++i, ++order) {
    const float* b = affine_box_bounds + 6 * i;
    Prim p{};
    p.ref = REF_TYPE_AFFINE_BOX | i;
    p.order = order;
    p.bounds = float_box(b[0], b[1], b[2], b[3], b[4], b[5]);
    p.measured = cfg->affine_box_weight;
    all.push_back(p);
  }
  for (auto& p : all)
    for (int k = 0; k < 3; ++k) p.cen[k] = (p.bounds.mn[k] + p.bounds.mx[k]) * 0.5;
  return all;
}

// Outputs must hold 2*N nodes (6 floats / 4 ints each), N refs and 4 roots, with
// N = ns + nb + nas + nab.  counts: node_count, root_count, leaf_count, max_depth,
// ref_count, min_leaf, max_leaf.  sah: generalized, uniform, weighted.
// Returns 0 on success, negative on an unsupported configuration.
static int build_any(const float* spheres, int ns, const float* boxes, int nb,
                     const float* affine_sphere_bounds, int nas, const float* affine_box_bounds,
                     int nab, const orc_build_config* cfg, int bins, int rotation_passes,
                     float* node_bounds, int* node_data, int* refs, int* roots, int* counts,
                     double* sah, int* rotations_out) {
  bool rotations = cfg->mode == 6 || cfg->mode == 7;
  if (cfg->mode < 0 || (cfg->mode > 3 && !rotations) || cfg->leaf_size < 1) return -1;
  if (bins != 0 && (bins < 2 || bins > 32)) return -1;
  if (rotations && (bins != 0 || rotation_passes < 1)) return -1;
  bool weighted = cfg->mode == 1 || cfg->mode == 3 || cfg->mode == 7;
  bool per_type = cfg->mode == 2 || cfg->mode == 3;
  if (rotations_out) *rotations_out = 0;
  Config c{weighted ? 1 : 0, cfg->leaf_size, cfg->traversal_weight,
           weighted ? cfg->lambda : 0.0};
  c.bins = bins;
  {
    const double measured[4] = {cfg->sphere_weight, cfg->box_weight, cfg->affine_sphere_weight,
                                cfg->affine_box_weight};
    for (int t = 0; t < 4; ++t) {
      if (!weighted) continue;
      double x = measured[t] - 1.0;
      x = c.lambda * x;
      c.type_weight[t] = 1.0 + x;
    }
  }
  int total = ns + nb + nas + nab;
  std::memset(counts, 0, 7 * sizeof(int));
  sah[0] = sah[1] = sah[2] = 0.0;
  if (total == 0) return 0;
  std::vector<Prim> all = make_prims(spheres, ns, boxes, nb, affine_sphere_bounds, nas,
                                     affine_box_bounds, nab, cfg);

  std::vector<std::vector<Prim>> parts;
  if (per_type) {
    for (int type : {REF_TYPE_SPHERE, REF_TYPE_BOX, REF_TYPE_AFFINE_SPHERE, REF_TYPE_AFFINE_BOX}) {
      std::vector<Prim> part;
      for (auto& p : all)
        if ((p.ref & REF_TYPE_MASK) == type) part.push_back(p);
      if (!part.empty()) parts.push_back(std::move(part));
    }
  } else {
    parts.push_back(all);
  }
  Flat f{node_bounds, node_data, refs};
  Summary total_summary;
  int min_leaf = INT32_MAX, max_leaf = 0, max_depth = 0;
  for (size_t t = 0; t < parts.size(); ++t) {
    Builder b(parts[t], c);
    b.pool.reserve(2 * parts[t].size());
    int root = b.build(0, (int)parts[t].size());
    if (rotations) {
      Rotator rot(b);
      int n_rot = 0;
      root = rot.optimize(root, rotation_passes, n_rot);
      if (rotations_out) *rotations_out += n_rot;
    }
    Summary s;
    summarize(b.pool, root, 0, s);
    total_summary.nodes += s.nodes;
    total_summary.leaves += s.leaves;
    max_depth = std::max(max_depth, s.max_depth);
    min_leaf = std::min(min_leaf, s.min_leaf);
    max_leaf = std::max(max_leaf, s.max_leaf);
    roots[t] = flatten(b.pool, root, parts[t], f);
    sah[1] += sah_cost(b.pool, root, parts[t], 0, b);
    sah[2] += sah_cost(b.pool, root, parts[t], 1, b);
    sah[0] += sah_cost(b.pool, root, parts[t], 2, b);
  }
  counts[0] = total_summary.nodes;
  counts[1] = (int)parts.size();
  counts[2] = total_summary.leaves;
  counts[3] = max_depth;
  counts[4] = f.next_ref;
  counts[5] = min_leaf == INT32_MAX ? 0 : min_leaf;
  counts[6] = max_leaf;
  if (total_summary.nodes != 2 * total_summary.leaves - (int)parts.size()) return -2;
  return 0;
}

int orc_build_bvh(const float* spheres, int ns, const float* boxes, int nb,
                  const float* affine_sphere_bounds, int nas, const float* affine_box_bounds,
                  int nab, const orc_build_config* cfg, float* node_bounds, int* node_data,
                  int* refs, int* roots, int* counts, double* sah) {
  return build_any(spheres, ns, boxes, nb, affine_sphere_bounds, nas, affine_box_bounds, nab, cfg,
                   0, 4, node_bounds, node_data, refs, roots, counts, sah, nullptr);
}

// The rotation modes (6 SAH_ROTATIONS, 7 WEIGHTED_SAH_ROTATIONS) with an explicit
// BvhBuildOptions.rotationPasses; *rotations receives the rotation count.
int orc_build_bvh_rotations(const float* spheres, int ns, const float* boxes, int nb,
                            const float* affine_sphere_bounds, int nas,
                            const float* affine_box_bounds, int nab, const orc_build_config* cfg,
                            int rotation_passes, float* node_bounds, int* node_data, int* refs,
                            int* roots, int* counts, double* sah, int* rotations) {
  return build_any(spheres, ns, boxes, nb, affine_sphere_bounds, nas, affine_box_bounds, nab, cfg,
                   0, rotation_passes, node_bounds, node_data, refs, roots, counts, sah, rotations);
}

// Binned object-SAH mode with 2..32 bins per axis (see the header of this file).
int orc_build_bvh_binned(const float* spheres, int ns, const float* boxes, int nb,
                         const float* affine_sphere_bounds, int nas,
                         const float* affine_box_bounds, int nab, const orc_build_config* cfg,
                         int bins, float* node_bounds, int* node_data, int* refs, int* roots,
                         int* counts, double* sah) {
  if (bins < 2 || bins > 32) return -1;
  return build_any(spheres, ns, boxes, nb, affine_sphere_bounds, nas, affine_box_bounds, nab, cfg,
                   bins, 4, node_bounds, node_data, refs, roots, counts, sah, nullptr);
}

// The SBVH modes (4 UNIFORM_SBVH, 5 WEIGHTED_SBVH) with BvhBuildOptions (spatialBins,
// maxReferenceMultiplier, maxSplitsPerPrimitive, minSpatialReferences,
// spatialOverlapThreshold).  Outputs must hold 2*R nodes and R refs, with
// R = max(N, floor(N * maxReferenceMultiplier)); counts as orc_build_bvh's;
// *spatial_splits receives BvhStats.spatialSplitCount.
int orc_build_bvh_sbvh(const float* spheres, int ns, const float* boxes, int nb,
                       const float* affine_sphere_bounds, int nas, const float* affine_box_bounds,
                       int nab, const orc_build_config* cfg, int spatial_bins,
                       double max_reference_multiplier, int max_splits_per_primitive,
                       int min_spatial_references, double spatial_overlap_threshold,
                       float* node_bounds, int* node_data, int* refs, int* roots, int* counts,
                       double* sah, int* spatial_splits) {
  if ((cfg->mode != 4 && cfg->mode != 5) || cfg->leaf_size < 1) return -1;
  bool weighted = cfg->mode == 5;
  Config c{weighted ? 1 : 0, cfg->leaf_size, cfg->traversal_weight, weighted ? cfg->lambda : 0.0};
  std::memset(counts, 0, 7 * sizeof(int));
  sah[0] = sah[1] = sah[2] = 0.0;
  *spatial_splits = 0;
  int total = ns + nb + nas + nab;
  if (total == 0) return 0;
  std::vector<Prim> all = make_prims(spheres, ns, boxes, nb, affine_sphere_bounds, nas,
                                     affine_box_bounds, nab, cfg);
  SpatialOptions o{spatial_bins, max_reference_multiplier, max_splits_per_primitive,
                   min_spatial_references, spatial_overlap_threshold};
  SpatialBuilder sb(c, o, total);
  std::vector<SRef> initial(total);
  for (int i = 0; i < total; ++i)
    initial[i] = SRef{all[i].ref, all[i].order, all[i].bounds, all[i].measured, 0};
  int root = sb.build(initial);
  std::vector<Prim> dummy;
  Builder stats_builder(dummy, c);
  Summary s;
  summarize(sb.pool, root, 0, s);
  Flat f{node_bounds, node_data, refs};
  roots[0] = flatten(sb.pool, root, sb.ordered, f);
  sah[1] = sah_cost(sb.pool, root, sb.ordered, 0, stats_builder);
  sah[2] = sah_cost(sb.pool, root, sb.ordered, 1, stats_builder);
  sah[0] = sah_cost(sb.pool, root, sb.ordered, 2, stats_builder);
  counts[0] = s.nodes;
  counts[1] = 1;
  counts[2] = s.leaves;
  counts[3] = s.max_depth;
  counts[4] = f.next_ref;
  counts[5] = s.min_leaf == INT32_MAX ? 0 : s.min_leaf;
  counts[6] = s.max_leaf;
  *spatial_splits = sb.spatial_splits;
  if (s.nodes != 2 * s.leaves - 1) return -2;
  return 0;
}

}  // extern "C"
