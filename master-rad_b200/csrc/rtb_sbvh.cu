// SBVH builds: the reference's SpatialBuildState (gfxlab/gpu/GpuScene.java:1084-1412,
// modes UNIFORM_SBVH and WEIGHTED_SBVH), producing the same tree node for node.
//
// That builder walks the tree depth first against one global reference budget
// (currentReferenceCount <= floor(N * maxReferenceMultiplier)): whether a node may split
// spatially depends on every split made before it in depth-first order, so the build is a
// sequence, not a level-parallel pass.  It runs here on the host, in this library, with the
// reference's arithmetic (IEEE double, no contraction: the build uses -fmad=false and the
// host compiler emits no fused multiply-adds for x86-64 baseline code):
//   * references are kept in one structure-of-arrays pool (originals, then every clipped
//     part appended); a node is a list of pool indices in the reference's list order;
//   * the three object-split sorts run concurrently for large nodes;
//   * the spatial plane search -- (spatialBins - 1) planes per axis, each a pass over the
//     node's references in list order -- is spread over host threads for large nodes; every
//     plane keeps the reference's sequential weight sums, so the costs are its own;
//   * the depth-first walk is iterative (explicit stack, left child first), so deep trees
//     need no recursion;
//   * the greedy unsplit pass keeps List.remove / List.add semantics (a node holds at most
//     one part of any primitive, so removing the part by identity is removing the first
//     equal element).
// Primitive bounds come from the device pass every builder uses (k_prims: the float bounds
// widened by two ulps), so they are the bounds the object-SAH builders see.  The flattened
// arrays (preorder nodes with float-cast bounds, references in leaf order, leaf kinds) and
// BvhStats are those of GpuScene.buildBvhData (614-700, 772-838).
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <thread>

#include "rtb_build_common.cuh"

namespace rtb {
namespace {

constexpr double kSpatialEps = 1.0e-12;

struct HBox {
  double mn[3], mx[3];
};

inline HBox hunion(const HBox& a, const HBox& b) {
  HBox r;
  for (int k = 0; k < 3; ++k) {
    r.mn[k] = std::min(a.mn[k], b.mn[k]);
    r.mx[k] = std::max(a.mx[k], b.mx[k]);
  }
  return r;
}

// Aabb.surfaceArea (GpuScene.java:71-74): 2 (dx dy + dx dz + dy dz), left to right.
inline double harea(const HBox& b) {
  double dx = b.mx[0] - b.mn[0], dy = b.mx[1] - b.mn[1], dz = b.mx[2] - b.mn[2];
  double s = dx * dy;
  s = s + dx * dz;
  s = s + dy * dz;
  return 2.0 * s;
}

inline int java_compare(double a, double b) {
  if (a < b) return -1;
  if (a > b) return 1;
  long long ia, ib;
  std::memcpy(&ia, &a, 8);
  std::memcpy(&ib, &b, 8);
  return ia == ib ? 0 : (ia < ib ? -1 : 1);
}

// Every reference of the build: the N originals, then clipped parts as they are made.
struct RefPool {
  std::vector<HBox> box;
  std::vector<int> ref, order, type, depth;
  int add(const HBox& b, int r, int o, int t, int d) {
    box.push_back(b);
    ref.push_back(r);
    order.push_back(o);
    type.push_back(t);
    depth.push_back(d);
    return (int)ref.size() - 1;
  }
  double centroid(int i, int axis) const { return (box[i].mn[axis] + box[i].mx[axis]) * 0.5; }
};

struct SNode {
  HBox bounds;
  int left = -1, right = -1, start = 0, end = 0, depth = 0;
};

struct SbvhOptions {
  int bins, max_splits, min_refs;
  double overlap;
};

// Runs f(task) for task in [0, count) on up to `threads` host threads.
template <typename F>
void parallel_tasks(int count, int threads, F f) {
  if (threads <= 1 || count <= 1) {
    for (int t = 0; t < count; ++t) f(t);
    return;
  }
  std::vector<std::thread> pool;
  int per = (count + threads - 1) / threads;
  for (int w = 0; w < threads; ++w) {
    int a = w * per, b = std::min(count, a + per);
    if (a >= b) break;
    pool.emplace_back([=]() {
      for (int t = a; t < b; ++t) f(t);
    });
  }
  for (auto& th : pool) th.join();
}

struct SbvhBuild {
  RefPool R;
  const double* w;  // construction weight per primitive type
  double traversal;
  int leaf_size;
  SbvhOptions opt;
  int max_refs, current, spatial_splits = 0;
  int threads;
  std::vector<SNode> nodes;
  std::vector<int> leaf_refs;  // pool indices in leaf order (the reference's `ordered`)

  double weight_of(int i) const { return w[R.type[i]]; }
  double weight_sum(const std::vector<int>& v) const {
    double s = 0.0;
    for (int i : v) s += weight_of(i);
    return s;
  }
  HBox bounds_of(const std::vector<int>& v) const {
    HBox b = R.box[v[0]];
    for (size_t k = 1; k < v.size(); ++k) b = hunion(b, R.box[v[k]]);
    return b;
  }

  // bestObjectSplit (1167-1207): the first minimum over (axis, position) of the swept cost.
  struct ObjectChoice {
    int axis = -1, left_count = 0;
    double cost = 0.0;
    HBox lb, rb;
    std::vector<int> sorted;
  };
  ObjectChoice best_object(const std::vector<int>& v, const HBox& nb) const {
    const int n = (int)v.size();
    std::vector<int> order[3];
    auto sort_axis = [&](int a) {
      order[a] = v;
      std::sort(order[a].begin(), order[a].end(), [&](int x, int y) {
        int c = java_compare(R.centroid(x, a), R.centroid(y, a));
        return c != 0 ? c < 0 : R.order[x] < R.order[y];
      });
    };
    parallel_tasks(3, n >= 20000 ? 3 : 1, sort_axis);
    ObjectChoice best;
    std::vector<HBox> suf(n);
    std::vector<double> sw(n);
    const double node_term = harea(nb) * traversal;
    for (int a = 0; a < 3; ++a) {
      const std::vector<int>& s = order[a];
      suf[n - 1] = R.box[s[n - 1]];
      sw[n - 1] = weight_of(s[n - 1]);
      for (int i = n - 2; i >= 0; --i) {
        suf[i] = hunion(suf[i + 1], R.box[s[i]]);
        sw[i] = sw[i + 1] + weight_of(s[i]);
      }
      HBox pre = R.box[s[0]];
      double pw = weight_of(s[0]);
      for (int i = 1; i < n; ++i) {
        double cost = node_term + harea(pre) * pw;
        cost = cost + harea(suf[i]) * sw[i];
        if (best.axis < 0 || cost < best.cost) {
          best.axis = a;
          best.left_count = i;
          best.cost = cost;
          best.lb = pre;
          best.rb = suf[i];
        }
        pre = hunion(pre, R.box[s[i]]);
        pw = pw + weight_of(s[i]);
      }
    }
    best.sorted = std::move(order[best.axis]);
    return best;
  }

  // shouldAttemptSpatial (1209-1221)
  bool attempt_spatial(int n, const HBox& nb, const ObjectChoice& oc) const {
    if (n < opt.min_refs || current >= max_refs) return false;
    HBox ov;
    bool empty = false;
    for (int k = 0; k < 3; ++k) {
      ov.mn[k] = std::max(oc.lb.mn[k], oc.rb.mn[k]);
      ov.mx[k] = std::min(oc.lb.mx[k], oc.rb.mx[k]);
      if (ov.mx[k] <= ov.mn[k]) empty = true;
    }
    double overlap = empty ? 0.0 : harea(ov);
    return overlap / std::max(harea(nb), 1.0e-30) > opt.overlap;
  }

  static double plane_at(double lo, double extent, int bin, int bins) {
    double p = extent * (double)bin;
    p = p / (double)bins;
    return lo + p;
  }

  // bestSpatialPlane (1223-1276): every (axis, bin) plane evaluated on its own (each a pass
  // over the references in list order, the reference's sums), then the first minimum in
  // (axis, bin) order.
  bool best_plane(const std::vector<int>& v, const HBox& nb, int* out_axis, double* out_pos) const {
    const int B = opt.bins, tasks = 3 * (B - 1);
    std::vector<double> cost(tasks, 0.0);
    std::vector<char> ok(tasks, 0);
    const double node_term = harea(nb) * traversal;
    auto eval = [&](int t) {
      int axis = t / (B - 1), bin = 1 + t % (B - 1);
      double lo = nb.mn[axis], extent = nb.mx[axis] - lo;
      if (!(extent > kSpatialEps)) return;
      double plane = plane_at(lo, extent, bin, B);
      HBox lb{}, rb{};
      bool hl = false, hr = false;
      double lw = 0.0, rw = 0.0;
      int dup = 0;
      for (int i : v) {
        const HBox& b = R.box[i];
        int side;  // 0 left, 1 right, 2 both (clipped)
        if (b.mx[axis] <= plane + kSpatialEps) side = 0;
        else if (b.mn[axis] >= plane - kSpatialEps) side = 1;
        else if (R.depth[i] < opt.max_splits) side = 2;
        else side = R.centroid(i, axis) <= plane ? 0 : 1;
        double wi = weight_of(i);
        if (side == 2) {
          HBox cl = b, cr = b;
          cl.mx[axis] = std::min(b.mx[axis], plane);
          cr.mn[axis] = std::max(b.mn[axis], plane);
          lb = hl ? hunion(lb, cl) : cl;
          rb = hr ? hunion(rb, cr) : cr;
          hl = hr = true;
          lw += wi;
          rw += wi;
          dup++;
        } else if (side == 0) {
          lb = hl ? hunion(lb, b) : b;
          hl = true;
          lw += wi;
        } else {
          rb = hr ? hunion(rb, b) : b;
          hr = true;
          rw += wi;
        }
      }
      if (!hl || !hr || current + dup > max_refs) return;
      double c = node_term + harea(lb) * lw;
      cost[t] = c + harea(rb) * rw;
      ok[t] = 1;
    };
    parallel_tasks(tasks, (int)v.size() >= 2048 ? threads : 1, eval);
    int best = -1;
    for (int t = 0; t < tasks; ++t)
      if (ok[t] && (best < 0 || cost[t] < cost[best])) best = t;
    if (best < 0) return false;
    *out_axis = best / (B - 1);
    double lo = nb.mn[*out_axis];
    *out_pos = plane_at(lo, nb.mx[*out_axis] - lo, 1 + best % (B - 1), B);
    return true;
  }

  static void erase_value(std::vector<int>& v, int x) {
    for (size_t k = 0; k < v.size(); ++k)
      if (v[k] == x) {
        v.erase(v.begin() + k);
        return;
      }
  }

  // partitionSpatial (1278-1334) with the greedy unsplit pass; false if a side is empty.
  bool partition(const std::vector<int>& v, int axis, double pos, std::vector<int>& left,
                 std::vector<int>& right, int* dup) {
    struct Choice {
      int original, l, r;
    };
    std::vector<Choice> choices;
    for (int i : v) {
      HBox b = R.box[i];
      if (b.mx[axis] <= pos + kSpatialEps) {
        left.push_back(i);
      } else if (b.mn[axis] >= pos - kSpatialEps) {
        right.push_back(i);
      } else if (R.depth[i] < opt.max_splits) {
        HBox cl = b, cr = b;
        cl.mx[axis] = std::min(b.mx[axis], pos);
        cr.mn[axis] = std::max(b.mn[axis], pos);
        int l = R.add(cl, R.ref[i], R.order[i], R.type[i], R.depth[i] + 1);
        int r = R.add(cr, R.ref[i], R.order[i], R.type[i], R.depth[i] + 1);
        left.push_back(l);
        right.push_back(r);
        choices.push_back({i, l, r});
      } else if (R.centroid(i, axis) <= pos) {
        left.push_back(i);
      } else {
        right.push_back(i);
      }
    }
    if (left.empty() || right.empty()) return false;
    for (const Choice& ch : choices) {
      HBox lb = bounds_of(left), rb = bounds_of(right);
      double lw = weight_sum(left), rw = weight_sum(right);
      double wo = weight_of(ch.original);
      double split = harea(lb) * lw;
      split = split + harea(rb) * rw;
      double left_only = harea(hunion(lb, R.box[ch.original])) * lw;
      left_only = left_only + harea(rb) * std::max(0.0, rw - wo);
      double right_only = harea(lb) * std::max(0.0, lw - wo);
      right_only = right_only + harea(hunion(rb, R.box[ch.original])) * rw;
      if (left_only < split && left_only <= right_only && right.size() > 1) {
        erase_value(left, ch.l);
        erase_value(right, ch.r);
        left.push_back(ch.original);
      } else if (right_only < split && left.size() > 1) {
        erase_value(left, ch.l);
        erase_value(right, ch.r);
        right.push_back(ch.original);
      }
    }
    *dup = (int)(left.size() + right.size()) - (int)v.size();
    return true;
  }

  // SpatialBuildState.build (1120-1161), depth first with an explicit stack.
  void run(std::vector<int> all) {
    struct Item {
      int node;
      std::vector<int> refs;
    };
    std::vector<Item> stack;
    nodes.push_back(SNode{});
    stack.push_back(Item{0, std::move(all)});
    while (!stack.empty()) {
      Item it = std::move(stack.back());
      stack.pop_back();
      const std::vector<int>& v = it.refs;
      HBox nb = bounds_of(v);
      nodes[it.node].bounds = nb;
      auto make_leaf = [&]() {
        nodes[it.node].start = (int)leaf_refs.size();
        leaf_refs.insert(leaf_refs.end(), v.begin(), v.end());
        nodes[it.node].end = (int)leaf_refs.size();
      };
      const int n = (int)v.size();
      if (n == 1) {
        make_leaf();
        continue;
      }
      ObjectChoice oc = best_object(v, nb);
      std::vector<int> sl, sr;
      bool spatial = false;
      int dup = 0;
      double spatial_cost = std::numeric_limits<double>::infinity();
      if (attempt_spatial(n, nb, oc)) {
        int axis = 0;
        double pos = 0.0;
        if (best_plane(v, nb, &axis, &pos)) {
          std::vector<int> cl, cr;
          int d = 0;
          if (partition(v, axis, pos, cl, cr, &d) && current + d <= max_refs) {
            double c = harea(nb) * traversal;
            c = c + harea(bounds_of(cl)) * weight_sum(cl);
            spatial_cost = c + harea(bounds_of(cr)) * weight_sum(cr);
            sl.swap(cl);
            sr.swap(cr);
            dup = d;
            spatial = true;
          }
        }
      }
      double leaf_cost = harea(nb) * weight_sum(v);
      bool choose_spatial = spatial && spatial_cost < oc.cost;
      double best = choose_spatial ? spatial_cost : oc.cost;
      if (n <= leaf_size && !(best < leaf_cost)) {
        make_leaf();
        continue;
      }
      std::vector<int> left, right;
      if (choose_spatial) {
        left.swap(sl);
        right.swap(sr);
        current += dup;
        spatial_splits++;
      } else {
        left.assign(oc.sorted.begin(), oc.sorted.begin() + oc.left_count);
        right.assign(oc.sorted.begin() + oc.left_count, oc.sorted.end());
      }
      int l = (int)nodes.size(), r = l + 1;
      nodes.push_back(SNode{});
      nodes.push_back(SNode{});
      nodes[it.node].left = l;
      nodes[it.node].right = r;
      nodes[l].depth = nodes[r].depth = nodes[it.node].depth + 1;
      stack.push_back(Item{r, std::move(right)});
      stack.push_back(Item{l, std::move(left)});
    }
  }
};

// sahCost / constructionSahCost (GpuScene.java:810-838) over the pool tree, post order.
// mode 0: unit weights, 1: measured weights, 2: construction weights.
double sbvh_sah(const SbvhBuild& b, const double* measured, int node, int mode) {
  const SNode& nd = b.nodes[node];
  if (nd.left < 0) {
    double c = 0.0;
    for (int k = nd.start; k < nd.end; ++k) {
      int t = b.R.type[b.leaf_refs[k]];
      c += mode == 0 ? 1.0 : mode == 1 ? measured[t] : b.w[t];
    }
    return c;
  }
  double area = harea(nd.bounds);
  double cl = sbvh_sah(b, measured, nd.left, mode), cr = sbvh_sah(b, measured, nd.right, mode);
  if (!(area > 0.0)) return cl + cr;
  double x = b.traversal + harea(b.nodes[nd.left].bounds) / area * cl;
  return x + harea(b.nodes[nd.right].bounds) / area * cr;
}

}  // namespace

rtb_status build_bvh_sbvh(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                          const rtb_build_options* options, rtb_scene** out, rtb_bvh_stats* stats) {
  if (!desc || !cfg || !out) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  rtb_build_options o = options ? *options : rtb_build_options{128, 2.0, 8, 16, 1.0e-5, 4};
  if (o.spatial_bins < 2 || !(o.max_reference_multiplier >= 1.0) ||
      !std::isfinite(o.max_reference_multiplier) || o.max_splits_per_primitive < 1 ||
      o.min_spatial_references < 2 || !(o.spatial_overlap_threshold >= 0.0) ||
      !std::isfinite(o.spatial_overlap_threshold))
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "invalid BvhBuildOptions");
  rtb_build_config object_cfg = *cfg;
  object_cfg.mode = cfg->mode == 5 ? 1 : 0;  // bounds and weights as the object builders'
  BuildCfg c;
  bool per_type = false;
  rtb_status st = build_setup(ctx, desc, &object_cfg, c, per_type);
  if (st != RTB_OK) return st;
  if (stats) *stats = rtb_bvh_stats{};
  auto t0 = std::chrono::steady_clock::now();
  if (c.total == 0) {
    rtb_status s = scene_create(ctx, desc, nullptr, nullptr, nullptr, 0, nullptr, 0, nullptr, 0, out);
    if (stats) stats->leaf_size = cfg->leaf_size;
    return s;
  }
  const int n = c.total;
  cudaStream_t sm = ctx->stream;
  std::vector<float> lo[3], hi[3];
  std::vector<int> refs(n), types(n);
  {
    Workspace W;
    W.stream = sm;
    PrimInputs in = alloc_inputs(W, c);
    Prims P = alloc_prims(W, n);
    if (!W.ok) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "SBVH primitive bounds");
    upload_prims(desc, c, in, P, sm);
    for (int k = 0; k < 3; ++k) {
      lo[k].resize(n);
      hi[k].resize(n);
      cudaMemcpyAsync(lo[k].data(), P.lo[k], (size_t)n * 4, cudaMemcpyDeviceToHost, sm);
      cudaMemcpyAsync(hi[k].data(), P.hi[k], (size_t)n * 4, cudaMemcpyDeviceToHost, sm);
    }
    cudaMemcpyAsync(refs.data(), P.ref, (size_t)n * 4, cudaMemcpyDeviceToHost, sm);
    cudaMemcpyAsync(types.data(), P.type, (size_t)n * 4, cudaMemcpyDeviceToHost, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "SBVH primitive bounds");
  }
  double w[4], measured[4];
  for (int t = 0; t < 4; ++t) {
    measured[t] = c.measured[t];
    double x = c.measured[t] - 1.0;
    x = c.lambda * x;
    w[t] = c.weighted ? 1.0 + x : 1.0;
  }
  SbvhBuild b;
  b.w = w;
  b.traversal = c.traversal;
  b.leaf_size = c.leaf_size;
  b.opt = SbvhOptions{o.spatial_bins, o.max_splits_per_primitive, o.min_spatial_references,
                      o.spatial_overlap_threshold};
  b.current = n;
  b.max_refs = std::max(n, (int)std::floor((double)n * o.max_reference_multiplier));
  b.threads = std::max(1, std::min(32, (int)std::thread::hardware_concurrency()));
  std::vector<int> all(n);
  for (int i = 0; i < n; ++i) {
    HBox hb;
    for (int k = 0; k < 3; ++k) {
      hb.mn[k] = (double)lo[k][i];
      hb.mx[k] = (double)hi[k][i];
    }
    all[i] = b.R.add(hb, refs[i], i, types[i], 0);
  }
  b.run(std::move(all));

  // flattenBvh (772-808): preorder, float-cast bounds, references in leaf order
  const int count = (int)b.nodes.size();
  const int nrefs = (int)b.leaf_refs.size();
  std::vector<float> nb((size_t)count * 6);
  std::vector<int> nd((size_t)count * 4), orefs(nrefs);
  int leaves = 0, max_depth = 0, min_occ = INT32_MAX, max_occ = 0, next_node = 0, next_ref = 0;
  std::vector<std::pair<int, int>> walk;  // (pool node, parent slot to patch, or -1)
  std::vector<int> pre(count, -1);
  walk.push_back({0, -1});
  while (!walk.empty()) {
    auto [node, parent_slot] = walk.back();
    walk.pop_back();
    int at = next_node++;
    pre[node] = at;
    if (parent_slot >= 0) nd[parent_slot] = at;
    const SNode& s = b.nodes[node];
    for (int k = 0; k < 3; ++k) {
      nb[(size_t)at * 6 + k] = (float)s.bounds.mn[k];
      nb[(size_t)at * 6 + 3 + k] = (float)s.bounds.mx[k];
    }
    max_depth = std::max(max_depth, s.depth);
    if (s.left < 0) {
      int occ = s.end - s.start;
      leaves++;
      min_occ = std::min(min_occ, occ);
      max_occ = std::max(max_occ, occ);
      int t0 = b.R.type[b.leaf_refs[s.start]];
      bool mixed = false;
      for (int k = s.start; k < s.end; ++k) {
        orefs[next_ref + (k - s.start)] = b.R.ref[b.leaf_refs[k]];
        if (b.R.type[b.leaf_refs[k]] != t0) mixed = true;
      }
      nd[(size_t)at * 4] = mixed ? -1 : -2 - t0;
      nd[(size_t)at * 4 + 1] = -1;
      nd[(size_t)at * 4 + 2] = next_ref;
      nd[(size_t)at * 4 + 3] = occ;
      next_ref += occ;
      continue;
    }
    nd[(size_t)at * 4 + 2] = -1;
    nd[(size_t)at * 4 + 3] = 0;
    walk.push_back({s.right, at * 4 + 1});
    walk.push_back({s.left, at * 4});
  }
  if (next_node != count || next_ref != nrefs || count != 2 * leaves - 1)
    return fail(ctx, RTB_ERR_DEVICE_CHECK, "SBVH flattening is incomplete");
  int root = 0;
  rtb_bvh_desc hb{nb.data(), nd.data(), count, orefs.data(), nrefs, &root, 1};
  rtb_status s = scene_create(ctx, desc, &hb, nullptr, nullptr, 0, nullptr, 0, nullptr, 0, out);
  if (s != RTB_OK) return s;
  if (stats) {
    stats->node_count = count;
    stats->root_count = 1;
    stats->leaf_count = leaves;
    stats->max_depth = max_depth;
    stats->primitive_ref_count = nrefs;
    stats->leaf_size = cfg->leaf_size;
    stats->min_leaf_occupancy = min_occ == INT32_MAX ? 0 : min_occ;
    stats->max_leaf_occupancy = max_occ;
    stats->uniform_sah_cost = sbvh_sah(b, measured, 0, 0);
    stats->weighted_sah_cost = sbvh_sah(b, measured, 0, 1);
    stats->generalized_sah_cost = sbvh_sah(b, measured, 0, 2);
    stats->bytes = (long long)count * 24 + ((long long)count * 4 + nrefs + 1) * 4;
    stats->build_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    stats->sequential_nodes = 0;
    stats->rotation_count = 0;
    stats->spatial_split_count = b.spatial_splits;
    stats->duplicate_reference_count = nrefs - n;
  }
  return RTB_OK;
}

}  // namespace rtb
