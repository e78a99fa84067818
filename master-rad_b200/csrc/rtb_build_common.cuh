// Pieces shared by the device BVH builders (full sweep in rtb_build.cu, binned in
// rtb_binned.cu): primitive bounds and weights, the node arrays of a level-synchronous
// build, the stable partition of a level, and the bottom-up / preorder / flatten passes
// that turn the node arrays into the reference's flattened layout (GpuScene.java:772-838).
// Every symbol has internal linkage; each builder's translation unit gets its own copy.
// Compiled with -fmad=false: no double expression is contracted.
#pragma once

#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "rtb_internal.h"

namespace rtb {
namespace {

struct Box {
  float mn[3], mx[3];
};

struct BoxUnion {
  __device__ __forceinline__ Box operator()(const Box& a, const Box& b) const {
    Box r;
    for (int k = 0; k < 3; ++k) {
      r.mn[k] = fminf(a.mn[k], b.mn[k]);
      r.mx[k] = fmaxf(a.mx[k], b.mx[k]);
    }
    return r;
  }
};

// Aabb.surfaceArea (GpuScene.java:70-74) on float-valued bounds, in double.
__device__ __forceinline__ double surface_area(const Box& b) {
  double dx = (double)b.mx[0] - (double)b.mn[0];
  double dy = (double)b.mx[1] - (double)b.mn[1];
  double dz = (double)b.mx[2] - (double)b.mn[2];
  double s = dx * dy + dx * dz;
  s = s + dy * dz;
  return 2.0 * s;
}

__device__ __forceinline__ float down2(float v) {
  return nextafterf(nextafterf(v, -CUDART_INF_F), -CUDART_INF_F);
}
__device__ __forceinline__ float up2(float v) {
  return nextafterf(nextafterf(v, CUDART_INF_F), CUDART_INF_F);
}

// Double.compare order as an unsigned key (-0.0 before +0.0, finite values in order).
__device__ __forceinline__ unsigned long long order_key(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ULL);
}

struct Prims {
  float* lo[3];
  float* hi[3];
  Box* box;          // the same bounds, one 24-byte record per primitive (gathers)
  double* cen[3];
  double* w;         // construction weight q = 1 + lambda (c - 1), or 1
  double* measured;  // c
  int* ref;
  int* type;
};

struct BuildCfg {
  int n[4];
  int total;
  int leaf_size;
  int weighted;
  double traversal, lambda;
  double measured[4];
};

// Primitive bounds (GpuScene.java:626-649, 877-903) and weights.
__global__ void k_prims(const float* spheres, const float* boxes, const float* ab, const float* bb,
                        BuildCfg c, Prims P) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= c.total) return;
  int t = 0, i = p;
  while (t < 3 && i >= c.n[t]) {
    i -= c.n[t];
    ++t;
  }
  float lo[3], hi[3];
  if (t == 0) {
    const float* s = spheres + 5 * (size_t)i;
    float r = s[3];
    for (int k = 0; k < 3; ++k) {
      lo[k] = down2(s[k] - r);
      hi[k] = up2(s[k] + r);
    }
  } else if (t == 1) {
    const float* b = boxes + 7 * (size_t)i;
    for (int k = 0; k < 3; ++k) {
      lo[k] = down2(b[k]);
      hi[k] = up2(b[3 + k]);
    }
  } else {
    const float* b = (t == 2 ? ab : bb) + 6 * (size_t)i;
    for (int k = 0; k < 3; ++k) {
      lo[k] = down2(b[k]);
      hi[k] = up2(b[3 + k]);
    }
  }
  Box bx;
  for (int k = 0; k < 3; ++k) {
    P.lo[k][p] = lo[k];
    P.hi[k][p] = hi[k];
    P.cen[k][p] = ((double)lo[k] + (double)hi[k]) * 0.5;
    bx.mn[k] = lo[k];
    bx.mx[k] = hi[k];
  }
  P.box[p] = bx;
  double m = c.measured[t];
  P.measured[p] = m;
  P.w[p] = c.weighted ? 1.0 + c.lambda * (m - 1.0) : 1.0;
  P.ref[p] = (int)((unsigned)t << kTypeShift) | i;
  P.type[p] = t;
}


struct Nodes {
  int* start;
  int* end;
  int* order_axis;  // axis array holding the node's current order; -1: input order
  int* depth;
  int* left;
  int* right;
  int* leaf;        // 1 leaf, 0 interior
  int* split_axis;  // this level's decision (-1: none)
  int* split_pos;
  Box* bounds;
  int* size;
  int* pre;
  int* rsize;   // primitive references under the node
  int* rfirst;  // the node's first reference in preorder (leaf ranges after rotations)
  double* sah[3];   // generalized, uniform, weighted
};

// key[j] = the root whose range [start, end) holds position j (at most four roots).
__global__ void k_init_keys(int* key, const int* start, const int* end, int roots, int n) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  for (int r = 0; r < roots; ++r)
    if (j >= start[r] && j < end[r]) key[j] = r;
}

__device__ __forceinline__ int current_prim(const int* const* idx, int order_axis, int j) {
  return order_axis < 0 ? j : idx[order_axis][j];
}

struct IdxSet {
  int* a[3];
};


__global__ void k_left_flags(const int* idx, const Nodes N, const int* key, const int* level_of,
                             int level, int n, const unsigned char* side, int* flags) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  bool split = level_of[node] == level && N.split_axis[node] >= 0;
  flags[j] = split ? (side[idx[j]] == 0) : 0;
}

__global__ void k_scatter(const int* idx, const Nodes N, const int* key, const int* level_of, int level,
                          int n, const unsigned char* side, const int* lscan, int* out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  int p = idx[j];
  if (!(level_of[node] == level && N.split_axis[node] >= 0)) {
    out[j] = p;
    return;
  }
  int s = N.start[node];
  int lrank = lscan[j] - lscan[s];
  int dst = side[p] == 0 ? s + lrank : s + N.split_pos[node] + ((j - s) - lrank);
  out[dst] = p;
}

__global__ void k_update_keys(const Nodes N, const int* level_of, int level, int n, int* key) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  if (level_of[node] != level || N.split_axis[node] < 0) return;
  key[j] = j < N.start[node] + N.split_pos[node] ? N.left[node] : N.right[node];
}

// Bottom-up subtree sizes and SAH statistics (GpuScene.java:810-838) over one level.
__global__ void k_bottom_up(const Prims P, IdxSet I, Nodes N, const int* nodes, int k,
                            double traversal) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = nodes[g];
  if (N.leaf[node]) {
    N.size[node] = 1;
    N.rsize[node] = N.end[node] - N.start[node];
    double c0 = 0.0, c1 = 0.0, c2 = 0.0;
    for (int j = N.start[node]; j < N.end[node]; ++j) {
      int p = current_prim(I.a, N.order_axis[node], j);
      c0 = c0 + P.w[p];
      c1 = c1 + 1.0;
      c2 = c2 + P.measured[p];
    }
    N.sah[0][node] = c0;
    N.sah[1][node] = c1;
    N.sah[2][node] = c2;
    return;
  }
  int l = N.left[node], r = N.right[node];
  N.size[node] = 1 + N.size[l] + N.size[r];
  N.rsize[node] = N.rsize[l] + N.rsize[r];
  double area = surface_area(N.bounds[node]);
  double al = surface_area(N.bounds[l]), ar = surface_area(N.bounds[r]);
  for (int m = 0; m < 3; ++m) {
    double v;
    if (!(area > 0.0)) {
      v = N.sah[m][l] + N.sah[m][r];
    } else {
      double x = al / area * N.sah[m][l];
      double y = ar / area * N.sah[m][r];
      v = (traversal + x) + y;
    }
    N.sah[m][node] = v;
  }
}

__global__ void k_preorder(Nodes N, const int* nodes, int k) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = nodes[g];
  if (N.leaf[node]) return;
  int l = N.left[node];
  N.pre[l] = N.pre[node] + 1;
  N.rfirst[l] = N.rfirst[node];
  N.rfirst[N.right[node]] = N.rfirst[node] + N.rsize[l];
  N.pre[N.right[node]] = N.pre[node] + 1 + N.size[l];
}

// Flattened reference layout (flattenBvh / leafKind, GpuScene.java:772-808).
__global__ void k_flatten(const Prims P, IdxSet I, const Nodes N, int count, float* node_bounds,
                          int* node_data, int* refs) {
  int node = blockIdx.x * blockDim.x + threadIdx.x;
  if (node >= count) return;
  int at = N.pre[node];
  Box b = N.bounds[node];
  for (int k = 0; k < 3; ++k) {
    node_bounds[6 * (size_t)at + k] = b.mn[k];
    node_bounds[6 * (size_t)at + 3 + k] = b.mx[k];
  }
  int* d = node_data + 4 * (size_t)at;
  if (!N.leaf[node]) {
    d[0] = N.pre[N.left[node]];
    d[1] = N.pre[N.right[node]];
    d[2] = -1;
    d[3] = 0;
    return;
  }
  // references in preorder of the leaves (after rotations that differs from array order)
  int s = N.start[node], e = N.end[node], f = N.rfirst[node];
  int t0 = -1;
  bool mixed = false;
  for (int j = s; j < e; ++j) {
    int p = current_prim(I.a, N.order_axis[node], j);
    refs[f + (j - s)] = P.ref[p];
    int t = P.type[p];
    if (t0 < 0) t0 = t;
    else if (t != t0) mixed = true;
  }
  d[0] = mixed ? -1 : -2 - t0;
  d[1] = -1;
  d[2] = f;
  d[3] = e - s;
}

inline unsigned blocks(long long n, int b = 256) { return (unsigned)std::max<long long>(1, (n + b - 1) / b); }

// Build workspace from the device's stream-ordered pool: after the first build the pool
// holds the memory, so later builds allocate without a device-wide synchronisation.
struct Workspace {
  std::vector<void*> ptrs;
  cudaStream_t stream = nullptr;
  bool ok = true;
  template <typename T>
  T* alloc(size_t n) {
    void* p = nullptr;
    if (cudaMallocAsync(&p, std::max<size_t>(n, 1) * sizeof(T), stream) != cudaSuccess) {
      ok = false;
      return nullptr;
    }
    ptrs.push_back(p);
    return (T*)p;
  }
  ~Workspace() {
    for (void* p : ptrs) cudaFreeAsync(p, stream);
  }
};

// ---- host side shared by the builders

// Validates a build request and fills the per-build constants.
// allow_rotations: the full-sweep builder also takes the rotation modes (6, 7).
inline rtb_status build_setup(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                              BuildCfg& c, bool& per_type, bool allow_rotations = false) {
  if (!desc || !cfg) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (cfg->mode < 0 || cfg->mode > 7) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "unknown BVH build mode");
  if (cfg->mode == 4 || cfg->mode == 5)
    return fail(ctx, RTB_ERR_UNSUPPORTED, "the SBVH modes have their own builder (rtb_scene_build)");
  if (cfg->mode > 5 && !allow_rotations)
    return fail(ctx, RTB_ERR_UNSUPPORTED, "rotation modes apply to the full-sweep builder");
  if (cfg->leaf_size < 1) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "BVH leaf size must be positive.");
  bool weighted = cfg->mode == 1 || cfg->mode == 3 || cfg->mode == 7;
  per_type = cfg->mode == 2 || cfg->mode == 3;
  c.n[0] = desc->sphere_count;
  c.n[1] = desc->box_count;
  c.n[2] = desc->affine_sphere_count;
  c.n[3] = desc->affine_box_count;
  for (int t = 0; t < 4; ++t)
    if (c.n[t] < 0) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "negative primitive count");
  if ((c.n[2] > 0 && !desc->affine_sphere_bounds) || (c.n[3] > 0 && !desc->affine_box_bounds))
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "affine bounds are required to build a BVH");
  long long total = (long long)c.n[0] + c.n[1] + c.n[2] + c.n[3];
  if (total > (1LL << 30) - 1) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "too many primitives");
  c.total = (int)total;
  c.leaf_size = cfg->leaf_size;
  c.weighted = weighted ? 1 : 0;
  c.traversal = cfg->traversal_weight;
  c.lambda = weighted ? cfg->lambda : 0.0;
  c.measured[0] = cfg->sphere_weight;
  c.measured[1] = cfg->box_weight;
  c.measured[2] = cfg->affine_sphere_weight;
  c.measured[3] = cfg->affine_box_weight;
  return RTB_OK;
}

// Primitive arrays of one build, allocated from the workspace.
inline Prims alloc_prims(Workspace& W, int n) {
  Prims P;
  for (int k = 0; k < 3; ++k) {
    P.lo[k] = W.alloc<float>(n);
    P.hi[k] = W.alloc<float>(n);
    P.cen[k] = W.alloc<double>(n);
  }
  P.box = W.alloc<Box>(n);
  P.w = W.alloc<double>(n);
  P.measured = W.alloc<double>(n);
  P.ref = W.alloc<int>(n);
  P.type = W.alloc<int>(n);
  return P;
}

struct PrimInputs {
  float *sph, *box, *ab, *bb;
};

inline PrimInputs alloc_inputs(Workspace& W, const BuildCfg& c) {
  return PrimInputs{W.alloc<float>((size_t)c.n[0] * 5), W.alloc<float>((size_t)c.n[1] * 7),
                    W.alloc<float>((size_t)c.n[2] * 6), W.alloc<float>((size_t)c.n[3] * 6)};
}

// Copies the packed host arrays in and computes bounds, centroids and weights.
inline void upload_prims(const rtb_scene_desc* desc, const BuildCfg& c, const PrimInputs& in,
                         const Prims& P, cudaStream_t sm) {
  if (c.n[0]) cudaMemcpyAsync(in.sph, desc->spheres, (size_t)c.n[0] * 20, cudaMemcpyHostToDevice, sm);
  if (c.n[1]) cudaMemcpyAsync(in.box, desc->boxes, (size_t)c.n[1] * 28, cudaMemcpyHostToDevice, sm);
  if (c.n[2])
    cudaMemcpyAsync(in.ab, desc->affine_sphere_bounds, (size_t)c.n[2] * 24, cudaMemcpyHostToDevice, sm);
  if (c.n[3])
    cudaMemcpyAsync(in.bb, desc->affine_box_bounds, (size_t)c.n[3] * 24, cudaMemcpyHostToDevice, sm);
  k_prims<<<blocks(c.total), 256, 0, sm>>>(in.sph, in.box, in.ab, in.bb, c, P);
}

inline Nodes alloc_nodes(Workspace& W, int cap) {
  Nodes N;
  N.start = W.alloc<int>(cap);
  N.end = W.alloc<int>(cap);
  N.order_axis = W.alloc<int>(cap);
  N.depth = W.alloc<int>(cap);
  N.left = W.alloc<int>(cap);
  N.right = W.alloc<int>(cap);
  N.leaf = W.alloc<int>(cap);
  N.split_axis = W.alloc<int>(cap);
  N.split_pos = W.alloc<int>(cap);
  N.bounds = W.alloc<Box>(cap);
  N.size = W.alloc<int>(cap);
  N.pre = W.alloc<int>(cap);
  N.rsize = W.alloc<int>(cap);
  N.rfirst = W.alloc<int>(cap);
  for (int m = 0; m < 3; ++m) N.sah[m] = W.alloc<double>(cap);
  return N;
}

// Root ranges: one tree over all primitives, or one per non-empty type (per-type forests,
// GpuScene.java:702-720); primitives are laid out type by type.
inline int root_ranges(const BuildCfg& c, bool per_type, int* rs, int* re) {
  if (!per_type) {
    rs[0] = 0;
    re[0] = c.total;
    return 1;
  }
  int roots = 0, off = 0;
  for (int t = 0; t < 4; ++t) {
    if (c.n[t] > 0) {
      rs[roots] = off;
      re[roots] = off + c.n[t];
      roots++;
    }
    off += c.n[t];
  }
  return roots;
}

// Bottom-up sizes and SAH statistics, preorder indices, the flattened arrays and the
// resident scene.  all_nodes lists the nodes level by level (level_begin offsets);
// counters + 2 holds {leaves, min occupancy, max occupancy, max depth}.
inline rtb_status finish_build(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                               Workspace& W, const BuildCfg& c, const Prims& P, const IdxSet& I,
                               const Nodes& N, const int* all_nodes, const std::vector<int>& level_begin,
                               int roots, int total_nodes, const int* counters, rtb_scene** out,
                               rtb_bvh_stats* stats) {
  cudaStream_t sm = ctx->stream;
  const int n = c.total;
  for (int L = (int)level_begin.size() - 2; L >= 0; --L) {
    int b = level_begin[L], cnt = level_begin[L + 1] - b;
    k_bottom_up<<<blocks(cnt, 128), 128, 0, sm>>>(P, I, N, all_nodes + b, cnt, c.traversal);
  }
  // Tree roots in order: preorder index = sizes of the previous trees.
  std::vector<int> h_size(roots), h_rsize(roots);
  for (int r = 0; r < roots; ++r) cudaMemcpyAsync(&h_size[r], N.size + r, 4, cudaMemcpyDeviceToHost, sm);
  for (int r = 0; r < roots; ++r) cudaMemcpyAsync(&h_rsize[r], N.rsize + r, 4, cudaMemcpyDeviceToHost, sm);
  double h_sah[4][3];
  for (int r = 0; r < roots; ++r)
    for (int m = 0; m < 3; ++m) cudaMemcpyAsync(&h_sah[r][m], N.sah[m] + r, 8, cudaMemcpyDeviceToHost, sm);
  cudaError_t e = cudaStreamSynchronize(sm);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH sizes");
  std::vector<int> h_pre(roots), h_rfirst(roots);
  int acc = 0;
  for (int r = 0; r < roots; ++r) {
    h_pre[r] = acc;
    acc += h_size[r];
    h_rfirst[r] = r ? h_rfirst[r - 1] + h_rsize[r - 1] : 0;
  }
  cudaMemcpyAsync(N.pre, h_pre.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(N.rfirst, h_rfirst.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  for (int L = 0; L + 1 < (int)level_begin.size(); ++L) {
    int b = level_begin[L], cnt = level_begin[L + 1] - b;
    k_preorder<<<blocks(cnt, 128), 128, 0, sm>>>(N, all_nodes + b, cnt);
  }
  float* o_nb = W.alloc<float>((size_t)total_nodes * 6);
  int* o_nd = W.alloc<int>((size_t)total_nodes * 4);
  int* o_refs = W.alloc<int>(n);
  int* o_roots = W.alloc<int>(4);
  if (!W.ok) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "BVH output");
  k_flatten<<<blocks(total_nodes, 128), 128, 0, sm>>>(P, I, N, total_nodes, o_nb, o_nd, o_refs);
  cudaMemcpyAsync(o_roots, h_pre.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  cudaEventRecord(ctx->ev1, sm);
  int h_stats[4];
  cudaMemcpyAsync(h_stats, counters + 2, sizeof(h_stats), cudaMemcpyDeviceToHost, sm);
  e = cudaStreamSynchronize(sm);
  if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH flatten");
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1);
  if (total_nodes != 2 * h_stats[0] - roots)
    return fail(ctx, RTB_ERR_DEVICE_CHECK, "A binary BVH forest must contain 2 * leafCount - rootCount nodes.");
  rtb_status s = scene_create(ctx, desc, nullptr, o_nb, o_nd, total_nodes, o_refs, n, o_roots, roots, out);
  if (s != RTB_OK) return s;
  if (stats) {
    stats->node_count = total_nodes;
    stats->root_count = roots;
    stats->leaf_count = h_stats[0];
    stats->max_depth = h_stats[3];
    stats->primitive_ref_count = n;
    stats->leaf_size = cfg->leaf_size;
    stats->min_leaf_occupancy = h_stats[1];
    stats->max_leaf_occupancy = h_stats[2];
    double g = 0.0, u = 0.0, w = 0.0;
    for (int r = 0; r < roots; ++r) {
      u = u + h_sah[r][1];
      w = w + h_sah[r][2];
      g = g + h_sah[r][0];
    }
    stats->generalized_sah_cost = g;
    stats->uniform_sah_cost = u;
    stats->weighted_sah_cost = w;
    stats->bytes = (long long)total_nodes * 24 + ((long long)total_nodes * 4 + n + roots) * 4;
    stats->build_ms = ms;
    stats->sequential_nodes = 0;
    stats->rotation_count = 0;
  }
  return RTB_OK;
}

}  // namespace
}  // namespace rtb
