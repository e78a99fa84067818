// Scene residency: packs the reference's float records into the device layout described in
// rtb_device.cuh and converts a flattened reference BVH into 64-byte child-pair nodes.
// Everything after the host-to-device copy of the caller's arrays runs on the GPU.
//
// Reference counterparts: GpuRayTracer.uploadScene / ensureSceneResident
// (gfxlab/gpu/GpuRayTracer.java:873-948) and the array layouts of
// gfxlab/gpu/GpuScene.java:23-31, 507-601, 772-808.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>

#include "rtb_internal.h"

namespace rtb {
namespace {

constexpr int kMaxRoots = 4;

struct Arena {
  size_t off = 0;
  template <typename T>
  size_t take(size_t count) {
    size_t o = (off + 255) & ~size_t(255);
    off = o + std::max<size_t>(count, 1) * sizeof(T);
    return o;
  }
};

__device__ __forceinline__ int checked_material(float v, int nmat, int* err) {
  int m = (int)v;
  if (m < -1 || m >= nmat) {
    atomicOr(err, 16);
    return -1;
  }
  return m;
}

__global__ void k_pack_spheres(const float* raw, int n, const int* orig_of_new, float4* out,
                               int* mat, int* orig, int nmat, int* err) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int o = orig_of_new ? orig_of_new[s] : s;
  const float* r = raw + 5 * (size_t)o;
  out[s] = make_float4(r[0], r[1], r[2], r[3]);
  mat[s] = checked_material(r[4], nmat, err);
  orig[s] = o;
}

__global__ void k_pack_boxes(const float* raw, int n, const int* orig_of_new, float4* out, int* mat,
                             int* orig, int nmat, int* err) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int o = orig_of_new ? orig_of_new[s] : s;
  const float* r = raw + 7 * (size_t)o;
  out[2 * s] = make_float4(r[0], r[1], r[2], 0.0f);
  out[2 * s + 1] = make_float4(r[3], r[4], r[5], 0.0f);
  mat[s] = checked_material(r[6], nmat, err);
  orig[s] = o;
}

__global__ void k_pack_affine(const float* raw, int n, const int* orig_of_new, float4* rows,
                              float* nm, int* mat, int* orig, int nmat, int* err) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  int o = orig_of_new ? orig_of_new[s] : s;
  const float* r = raw + 22 * (size_t)o;
  rows[3 * s] = make_float4(r[0], r[1], r[2], r[3]);
  rows[3 * s + 1] = make_float4(r[4], r[5], r[6], r[7]);
  rows[3 * s + 2] = make_float4(r[8], r[9], r[10], r[11]);
  for (int k = 0; k < 9; ++k) nm[9 * (size_t)s + k] = r[12 + k];
  mat[s] = checked_material(r[21], nmat, err);
  orig[s] = o;
}

__global__ void k_pack_planes(const float* raw, int n, float4* out, float* full, int nmat, int* err) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float* r = raw + 26 * (size_t)s;
  checked_material(r[18 + 5], nmat, err);
  if (r[18] != 0.0f) {
    checked_material(r[18 + 6], nmat, err);
    checked_material(r[18 + 7], nmat, err);
  }
  out[s] = make_float4(r[0], r[1], r[2], r[3]);
  for (int k = 0; k < 26; ++k) full[26 * (size_t)s + k] = r[k];
}

__global__ void k_pack_materials(const float* raw, int n, float4* out) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  const float* r = raw + 13 * (size_t)s;
  out[4 * s] = make_float4(r[0], r[1], r[2], r[12]);
  out[4 * s + 1] = make_float4(r[3], r[4], r[5], 0.0f);
  out[4 * s + 2] = make_float4(r[6], r[7], r[8], 0.0f);
  out[4 * s + 3] = make_float4(r[9], r[10], r[11], 0.0f);
}

// Per-type reference flags: flag[t * n + j] = (type of ref j == t).  Also validates the
// indices and records first sightings, so duplicate or out-of-range references are seen.
__global__ void k_ref_flags(const int* refs, int n, const int* counts, int* flags, int* seen,
                            const int* seen_base, int* err) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int ref = refs[j];
  int t = (int)((unsigned)ref >> kTypeShift);
  int idx = ref & kIndexMask;
  for (int k = 0; k < 4; ++k) flags[k * (size_t)n + j] = (k == t);
  if (idx >= counts[t]) {
    atomicOr(err, 1);
    return;
  }
  if (atomicAdd(seen + seen_base[t] + idx, 1) != 0) atomicOr(err, 2);  // duplicate reference
}

// New storage index for every reference, inverse maps, and the rewritten reference words.
__global__ void k_ref_remap(const int* refs, int n, const int* ranks, int* refs_out,
                            int* orig_of_new, const int* base) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int ref = refs[j];
  int t = (int)((unsigned)ref >> kTypeShift);
  int idx = ref & kIndexMask;
  int s = ranks[t * (size_t)n + j];
  orig_of_new[base[t] + s] = idx;
  refs_out[j] = (int)((unsigned)t << kTypeShift) | s;
}

__global__ void k_identity_refs(const int* refs, int n, int* refs_out) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) refs_out[j] = refs[j];
}

__global__ void k_interior_flags(const int* node_data, int n, int* flags) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) flags[i] = node_data[4 * (size_t)i] >= 0;
}

__device__ int leaf_code(int kind) {
  switch (kind) {
    case -2: return 0;
    case -3: return 1;
    case -4: return 2;
    case -5: return 3;
    default: return 4;
  }
}

// Child slot c of a converted node from reference node `child` (or an empty slot).
__device__ void write_child(float4* node, int c, int child, const float* bounds, const int* data,
                            const int* rank, int synth, int node_count, int ref_count, int* err) {
  float lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int link = ~0, meta = 0;
  if (child >= 0) {
    if (child >= node_count) {
      atomicOr(err, 4);
    } else {
      for (int k = 0; k < 3; ++k) {
        lo[k] = bounds[6 * (size_t)child + k];
        hi[k] = bounds[6 * (size_t)child + 3 + k];
      }
      int kind = data[4 * (size_t)child];
      if (kind >= 0) {
        link = synth + rank[child];
      } else {
        int first = data[4 * (size_t)child + 2];
        int count = data[4 * (size_t)child + 3];
        if (kind < -5 || first < 0 || count < 0 || count > 0xFFFFFF ||
            (long long)first + count > ref_count) {
          atomicOr(err, 8);
        } else {
          link = ~first;
          meta = count | (leaf_code(kind) << 24);
        }
      }
    }
  }
  float* f = reinterpret_cast<float*>(node);
  int* iv = reinterpret_cast<int*>(node + 3);
  if (c == 0) {
    f[0] = lo[0];
    f[1] = hi[0];
    f[2] = lo[1];
    f[3] = hi[1];
    f[8] = lo[2];
    f[9] = hi[2];
    iv[0] = link;
    iv[2] = meta;
  } else {
    f[4] = lo[0];
    f[5] = hi[0];
    f[6] = lo[1];
    f[7] = hi[1];
    f[10] = lo[2];
    f[11] = hi[2];
    iv[1] = link;
    iv[3] = meta;
  }
}

__global__ void k_convert_nodes(const float* bounds, const int* data, int n, int ref_count,
                                const int* rank, int synth, float4* nodes, int* err) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int l = data[4 * (size_t)i];
  if (l < 0) return;
  int r = data[4 * (size_t)i + 1];
  float4* node = nodes + 4 * (size_t)(synth + rank[i]);
  write_child(node, 0, l, bounds, data, rank, synth, n, ref_count, err);
  write_child(node, 1, r, bounds, data, rank, synth, n, ref_count, err);
}

// Synthetic top: node 0 holds the first two roots; with 3-4 roots node 0 points at two
// more synthetic nodes holding roots (0,1) and (2,3).
__global__ void k_top_nodes(const float* bounds, const int* data, int n, int ref_count,
                            const int* rank, const int* roots, int root_count, int synth,
                            float4* nodes, int* err) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int r[4] = {-1, -1, -1, -1};
  for (int k = 0; k < root_count && k < 4; ++k) r[k] = roots[k];
  if (root_count <= 2) {
    write_child(nodes, 0, r[0], bounds, data, rank, synth, n, ref_count, err);
    write_child(nodes, 1, r[1], bounds, data, rank, synth, n, ref_count, err);
    return;
  }
  write_child(nodes + 4, 0, r[0], bounds, data, rank, synth, n, ref_count, err);
  write_child(nodes + 4, 1, r[1], bounds, data, rank, synth, n, ref_count, err);
  write_child(nodes + 8, 0, r[2], bounds, data, rank, synth, n, ref_count, err);
  write_child(nodes + 8, 1, r[3], bounds, data, rank, synth, n, ref_count, err);
  // Node 0: children are synthetic nodes 1 and 2 with the union bounds of their roots.
  float* f = reinterpret_cast<float*>(nodes);
  int* iv = reinterpret_cast<int*>(nodes + 3);
  for (int c = 0; c < 2; ++c) {
    const float* a = reinterpret_cast<const float*>(nodes + 4 * (1 + c));
    float lox = fminf(a[0], a[4]), hix = fmaxf(a[1], a[5]);
    float loy = fminf(a[2], a[6]), hiy = fmaxf(a[3], a[7]);
    float loz = fminf(a[8], a[10]), hiz = fmaxf(a[9], a[11]);
    if (c == 1 && r[3] < 0) {  // the empty slot's zero box must not widen the union
      lox = a[0];
      hix = a[1];
      loy = a[2];
      hiy = a[3];
      loz = a[8];
      hiz = a[9];
    }
    int base = c == 0 ? 0 : 4;
    f[base + 0] = lox;
    f[base + 1] = hix;
    f[base + 2] = loy;
    f[base + 3] = hiy;
    f[8 + 2 * c] = loz;
    f[9 + 2 * c] = hiz;
    iv[c] = 1 + c;
    iv[2 + c] = 0;
  }
}

inline unsigned blocks(long long n, int b = 256) { return (unsigned)((n + b - 1) / b); }

}  // namespace

void scene_free(rtb_scene* s, cudaStream_t stream) {
  if (!s) return;
  cudaFreeAsync(s->arena, stream);
  for (void* p : s->extra) cudaFreeAsync(p, stream);
  delete s;
}

rtb_status scene_create(rtb_context* ctx, const rtb_scene_desc* d, const rtb_bvh_desc* hb,
                        const float* d_nb, const int* d_nd, int node_count, const int* d_refs,
                        int ref_count, const int* d_roots, int root_count, rtb_scene** out) {
  if (!d || !out) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "scene description is required");
  const int cnt[6] = {d->sphere_count, d->box_count, d->plane_count, d->affine_sphere_count,
                      d->affine_box_count, d->material_count};
  const float* src[6] = {d->spheres, d->boxes, d->planes, d->affine_spheres, d->affine_boxes,
                         d->materials};
  const int fpr[6] = {5, 7, 26, 22, 22, 13};
  for (int k = 0; k < 6; ++k) {
    if (cnt[k] < 0 || (cnt[k] > 0 && !src[k]))
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "scene array missing or negative count");
    if (k < 5 && cnt[k] > kIndexMask)
      return fail(ctx, RTB_ERR_LIMIT, "primitive count exceeds the 30-bit reference index");
  }
  if (hb) {
    if (hb->node_count < 0 || hb->primitive_ref_count < 0 || hb->root_count < 0 ||
        hb->root_count > kMaxRoots || (hb->node_count > 0 && (!hb->node_bounds || !hb->node_data)) ||
        (hb->primitive_ref_count > 0 && !hb->primitive_refs) ||
        (hb->root_count > 0 && !hb->root_indices))
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "invalid BVH description");
    node_count = hb->node_count;
    ref_count = hb->primitive_ref_count;
    root_count = hb->root_count;
  }
  bool has_bvh = node_count > 0 && ref_count > 0 && root_count > 0;
  if (has_bvh && (long long)node_count > 2LL * ref_count + 8)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "BVH has more nodes than a binary tree over its references");
  int nprim[4] = {cnt[0], cnt[1], cnt[3], cnt[4]};
  int nbounded = nprim[0] + nprim[1] + nprim[2] + nprim[3];

  // ---- staging: raw packed arrays (+ host BVH) in one device buffer
  Arena st;
  size_t raw_off[6];
  for (int k = 0; k < 6; ++k) raw_off[k] = st.take<float>((size_t)cnt[k] * fpr[k]);
  size_t hb_off[4] = {0, 0, 0, 0};
  if (hb && has_bvh) {
    hb_off[0] = st.take<float>((size_t)node_count * 6);
    hb_off[1] = st.take<int>((size_t)node_count * 4);
    hb_off[2] = st.take<int>((size_t)ref_count);
    hb_off[3] = st.take<int>((size_t)root_count);
  }
  size_t flags_off = st.take<int>((size_t)4 * std::max(ref_count, 1));
  size_t ranks_off = st.take<int>((size_t)4 * std::max(ref_count, 1));
  size_t seen_off = st.take<int>((size_t)std::max(nbounded, 1));
  size_t iflag_off = st.take<int>((size_t)std::max(node_count, 1));
  size_t meta_off = st.take<int>(16);  // err word, counts[4], seen_base[4], base[4]
  size_t scan_tmp_bytes = 0;
  {
    int* dummy = nullptr;
    cub::DeviceScan::ExclusiveSum(nullptr, scan_tmp_bytes, dummy, dummy,
                                  4 * std::max(ref_count, std::max(node_count, 1)));
  }
  size_t tmp_off = st.take<char>(scan_tmp_bytes);
  char* sb = (char*)stage(ctx, st.off);
  if (!sb) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "staging allocation failed");
  cudaStream_t sm = ctx->stream;
  for (int k = 0; k < 6; ++k)
    if (cnt[k] > 0)
      cudaMemcpyAsync(sb + raw_off[k], src[k], (size_t)cnt[k] * fpr[k] * 4, cudaMemcpyHostToDevice, sm);
  if (hb && has_bvh) {
    cudaMemcpyAsync(sb + hb_off[0], hb->node_bounds, (size_t)node_count * 24, cudaMemcpyHostToDevice, sm);
    cudaMemcpyAsync(sb + hb_off[1], hb->node_data, (size_t)node_count * 16, cudaMemcpyHostToDevice, sm);
    cudaMemcpyAsync(sb + hb_off[2], hb->primitive_refs, (size_t)ref_count * 4, cudaMemcpyHostToDevice, sm);
    cudaMemcpyAsync(sb + hb_off[3], hb->root_indices, (size_t)root_count * 4, cudaMemcpyHostToDevice, sm);
    d_nb = (const float*)(sb + hb_off[0]);
    d_nd = (const int*)(sb + hb_off[1]);
    d_refs = (const int*)(sb + hb_off[2]);
    d_roots = (const int*)(sb + hb_off[3]);
  }

  // ---- arena layout
  int interior = 0;
  int synth = root_count > 2 ? 3 : 1;
  Arena ar;
  size_t o_sph = ar.take<float4>(nprim[0]);
  size_t o_box = ar.take<float4>(2 * (size_t)nprim[1]);
  size_t o_asp = ar.take<float4>(3 * (size_t)nprim[2]);
  size_t o_abx = ar.take<float4>(3 * (size_t)nprim[3]);
  size_t o_asn = ar.take<float>(9 * (size_t)nprim[2]);
  size_t o_abn = ar.take<float>(9 * (size_t)nprim[3]);
  size_t o_mat = ar.take<int>(nbounded);
  size_t o_orig = ar.take<int>(nbounded);
  size_t o_oon = ar.take<int>(nbounded);  // orig_of_new, concatenated by type
  size_t o_pl = ar.take<float4>(cnt[2]);
  size_t o_plf = ar.take<float>(26 * (size_t)cnt[2]);
  size_t o_mt = ar.take<float4>(4 * (size_t)cnt[5]);
  size_t o_refs = ar.take<int>(ref_count);
  size_t o_rnb = ar.take<float>(6 * (size_t)node_count);
  size_t o_rnd = ar.take<int>(4 * (size_t)node_count);
  size_t o_rrf = ar.take<int>(ref_count);
  size_t o_rrt = ar.take<int>(root_count);

  int* err = (int*)(sb + meta_off);
  int* d_counts = err + 1;
  int* d_seen_base = err + 5;
  int* d_base = err + 9;
  int h_meta[16] = {0};
  for (int t = 0; t < 4; ++t) {
    h_meta[1 + t] = nprim[t];
    int b = 0;
    for (int u = 0; u < t; ++u) b += nprim[u];
    h_meta[5 + t] = b;
    h_meta[9 + t] = b;
  }
  // Interior-node count is needed for the node array size; compute it on the device.
  int* iflag = (int*)(sb + iflag_off);
  int* irank = (int*)(sb + ranks_off);  // reused below only after the node conversion
  cudaMemcpyAsync(err, h_meta, sizeof(h_meta), cudaMemcpyHostToDevice, sm);
  if (has_bvh) {
    k_interior_flags<<<blocks(node_count), 256, 0, sm>>>(d_nd, node_count, iflag);
    size_t tb = scan_tmp_bytes;
    cub::DeviceScan::ExclusiveSum(sb + tmp_off, tb, iflag, irank, node_count, sm);
    int last_flag = 0, last_rank = 0;
    cudaMemcpyAsync(&last_flag, iflag + node_count - 1, 4, cudaMemcpyDeviceToHost, sm);
    cudaMemcpyAsync(&last_rank, irank + node_count - 1, 4, cudaMemcpyDeviceToHost, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH interior scan");
    interior = last_flag + last_rank;
  }
  size_t o_nodes = ar.take<float4>(4 * (size_t)(synth + interior));

  rtb_scene* s = new rtb_scene();
  cudaError_t e = cudaMallocAsync(&s->arena, ar.off, sm);
  if (e != cudaSuccess) {
    delete s;
    return cuda_fail(ctx, e, "scene arena");
  }
  s->arena_bytes = ar.off;
  char* A = (char*)s->arena;
  cudaMemsetAsync(A, 0, ar.off, sm);

  // ---- node conversion (uses irank before the reference ranks overwrite the buffer)
  float4* nodes = (float4*)(A + o_nodes);
  if (has_bvh) {
    k_convert_nodes<<<blocks(node_count), 256, 0, sm>>>(d_nb, d_nd, node_count, ref_count, irank,
                                                         synth, nodes, err);
    k_top_nodes<<<1, 32, 0, sm>>>(d_nb, d_nd, node_count, ref_count, irank, d_roots, root_count,
                                  synth, nodes, err);
    cudaMemcpyAsync(A + o_rnb, d_nb, (size_t)node_count * 24, cudaMemcpyDeviceToDevice, sm);
    cudaMemcpyAsync(A + o_rnd, d_nd, (size_t)node_count * 16, cudaMemcpyDeviceToDevice, sm);
    cudaMemcpyAsync(A + o_rrf, d_refs, (size_t)ref_count * 4, cudaMemcpyDeviceToDevice, sm);
    cudaMemcpyAsync(A + o_rrt, d_roots, (size_t)root_count * 4, cudaMemcpyDeviceToDevice, sm);
  }

  // ---- reference permutation: records in first-appearance order of the leaf references
  int* oon = (int*)(A + o_oon);
  bool permute = false;
  if (has_bvh) {
    int* flags = (int*)(sb + flags_off);
    int* ranks = (int*)(sb + ranks_off);
    int* seen = (int*)(sb + seen_off);
    cudaMemsetAsync(seen, 0, (size_t)std::max(nbounded, 1) * 4, sm);
    k_ref_flags<<<blocks(ref_count), 256, 0, sm>>>(d_refs, ref_count, d_counts, flags, seen,
                                                    d_seen_base, err);
    int herr = 0;
    cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, sm);
    e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) {
      scene_free(s, sm);
      return cuda_fail(ctx, e, "BVH reference check");
    }
    if (herr & 1) {
      scene_free(s, sm);
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "BVH reference index out of range");
    }
    if (herr & (4 | 8)) {
      scene_free(s, sm);
      return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "BVH node child or leaf range out of range");
    }
    // A permutation needs every primitive referenced exactly once (no duplicates).
    permute = !(herr & 2) && ref_count == nbounded;
    if (permute) {
      for (int t = 0; t < 4; ++t) {
        size_t tb = scan_tmp_bytes;
        cub::DeviceScan::ExclusiveSum(sb + tmp_off, tb, flags + (size_t)t * ref_count,
                                      ranks + (size_t)t * ref_count, ref_count, sm);
      }
      k_ref_remap<<<blocks(ref_count), 256, 0, sm>>>(d_refs, ref_count, ranks, (int*)(A + o_refs),
                                                      oon, d_base);
    } else {
      k_identity_refs<<<blocks(ref_count), 256, 0, sm>>>(d_refs, ref_count, (int*)(A + o_refs));
    }
  }

  // ---- primitive packing
  int* mat = (int*)(A + o_mat);
  int* orig = (int*)(A + o_orig);
  int base[4] = {h_meta[9], h_meta[10], h_meta[11], h_meta[12]};
  if (nprim[0])
    k_pack_spheres<<<blocks(nprim[0]), 256, 0, sm>>>((const float*)(sb + raw_off[0]), nprim[0],
                                                      permute ? oon + base[0] : nullptr,
                                                      (float4*)(A + o_sph), mat + base[0], orig + base[0],
                                                      cnt[5], err);
  if (nprim[1])
    k_pack_boxes<<<blocks(nprim[1]), 256, 0, sm>>>((const float*)(sb + raw_off[1]), nprim[1],
                                                    permute ? oon + base[1] : nullptr,
                                                    (float4*)(A + o_box), mat + base[1], orig + base[1],
                                                    cnt[5], err);
  if (nprim[2])
    k_pack_affine<<<blocks(nprim[2]), 256, 0, sm>>>((const float*)(sb + raw_off[3]), nprim[2],
                                                     permute ? oon + base[2] : nullptr,
                                                     (float4*)(A + o_asp), (float*)(A + o_asn),
                                                     mat + base[2], orig + base[2], cnt[5], err);
  if (nprim[3])
    k_pack_affine<<<blocks(nprim[3]), 256, 0, sm>>>((const float*)(sb + raw_off[4]), nprim[3],
                                                     permute ? oon + base[3] : nullptr,
                                                     (float4*)(A + o_abx), (float*)(A + o_abn),
                                                     mat + base[3], orig + base[3], cnt[5], err);
  if (cnt[2])
    k_pack_planes<<<blocks(cnt[2]), 256, 0, sm>>>((const float*)(sb + raw_off[2]), cnt[2],
                                                   (float4*)(A + o_pl), (float*)(A + o_plf),
                                                   cnt[5], err);
  if (cnt[5])
    k_pack_materials<<<blocks(cnt[5]), 256, 0, sm>>>((const float*)(sb + raw_off[5]), cnt[5],
                                                      (float4*)(A + o_mt));
  int herr = 0;
  cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, sm);
  e = cudaStreamSynchronize(sm);
  if (e == cudaSuccess) e = cudaGetLastError();
  if (e != cudaSuccess) {
    scene_free(s, sm);
    return cuda_fail(ctx, e, "scene packing");
  }
  if (herr & (1 | 4 | 8)) {
    scene_free(s, sm);
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "BVH arrays failed the device range checks");
  }
  if (herr & 16) {
    scene_free(s, sm);
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "material index outside the material table");
  }

  DevScene& D = s->dev;
  D.nodes = has_bvh ? nodes : nullptr;
  D.node_count = has_bvh ? synth + interior : 0;
  D.refs = (const int*)(A + o_refs);
  D.ref_count = has_bvh ? ref_count : 0;
  D.spheres = (const float4*)(A + o_sph);
  D.boxes = (const float4*)(A + o_box);
  D.aspheres = (const float4*)(A + o_asp);
  D.aboxes = (const float4*)(A + o_abx);
  D.asphere_nm = (const float*)(A + o_asn);
  D.abox_nm = (const float*)(A + o_abn);
  for (int t = 0; t < 4; ++t) {
    D.mat[t] = mat + base[t];
    D.orig[t] = orig + base[t];
    D.count[t] = nprim[t];
    D.order_base[t] = base[t];
  }
  D.order_base[4] = nbounded;
  D.planes = (const float4*)(A + o_pl);
  D.plane_full = (const float*)(A + o_plf);
  D.plane_count = cnt[2];
  D.materials = (const float4*)(A + o_mt);
  D.material_count = cnt[5];
  D.background = make_float3(d->background[0], d->background[1], d->background[2]);
  D.use_bvh = has_bvh ? 1 : 0;
  s->has_bvh = has_bvh;
  s->device = ctx->device;
  s->ref_node_bounds = (float*)(A + o_rnb);
  s->ref_node_data = (int*)(A + o_rnd);
  s->ref_refs = (int*)(A + o_rrf);
  s->ref_roots = (int*)(A + o_rrt);
  s->ref_node_count = has_bvh ? node_count : 0;
  s->ref_ref_count = has_bvh ? ref_count : 0;
  s->ref_root_count = has_bvh ? root_count : 0;
  *out = s;
  return RTB_OK;
}

}  // namespace rtb
