// Device BVH builder, binned mode: object SAH over B = 2..32 centroid bins per axis with the
// per-type construction weights.  This mode has no counterpart in the reference (its builder
// is the full sweep of GpuScene.java:1453-1488, restated in rtb_build.cu); it trades the
// node-for-node identity with the Java tree for a build that touches every primitive a
// constant number of times per level.
//
// Definition (restated on the CPU by the oracle, which the tests compare node for node):
//  * a node's centroid bounds, box and per-type counts are exact reductions;
//  * on every axis whose centroid extent exceeds 1e-12, bin(c) = min(B - 1,
//    (int)((c - lo) * (B / extent))); each bin keeps integer counts per primitive type and
//    the union of its primitives' float boxes;
//  * the weight of a set is ((n0 w0 + n1 w1) + n2 w2) + n3 w3 in double, w_t the per-type
//    construction weights 1 + lambda (c_t - 1): it depends only on integer counts, so the
//    result does not depend on the order in which atomics land;
//  * plane j = 1..B-1 puts bins [0, j) left; cost (A_P c_T + A_L W_L) + A_R W_R; the first
//    minimum over (axis, j) with both sides non-empty wins;
//  * leaf if count == 1, or count <= leafSize and !(cost < A_P W_P); a node whose centroids
//    coincide on every axis is a leaf when count <= leafSize and otherwise splits at
//    count / 2 in its current order;
//  * children are a stable partition of the node's primitives (left first).
//
// Per level, nodes above kSmall primitives are "large": their bounds and bins are
// accumulated over all primitives of the level by warp-aggregated atomics (counts per bin
// from __match_any_sync groups and ballots, box bounds by group reductions), privatised in
// shared memory for the node that owns a block's chunk; one warp per node then scans the
// 32 bins (prefix / suffix in registers, one bin per lane) and picks the split.  Smaller
// nodes are handled entirely by one warp each (primitives in registers, bins in shared
// memory).  The level's stable partition and the bottom-up / preorder / flatten passes are
// shared with the full-sweep builder.
#include "rtb_build_common.cuh"

namespace rtb {
namespace {

constexpr int kSmall = 128;           // nodes up to this size are split by one warp alone
constexpr int kPerLane = kSmall / 32;
constexpr int kChunk = 4096;          // positions per block in the large-node passes
constexpr double kMinExtent = 1.0e-12;
constexpr unsigned kFull = 0xFFFFFFFFu;

// float <-> order-preserving unsigned, so atomicMin / atomicMax order float values.
__device__ __forceinline__ unsigned f2o(float f) {
  unsigned b = __float_as_uint(f);
  return (b >> 31) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float o2f(unsigned o) {
  return __uint_as_float((o >> 31) ? (o & 0x7FFFFFFFu) : ~o);
}
// Inverse of order_key (double -> order-preserving 64-bit).
__device__ __forceinline__ double k2d(unsigned long long k) {
  return __longlong_as_double((long long)((k >> 63) ? (k & 0x7FFFFFFFFFFFFFFFULL) : ~k));
}

__device__ __forceinline__ int bin_of(double c, double lo, double scale, int bins) {
  double x = c - lo;
  x = x * scale;
  int b = (int)x;
  return b < bins ? b : bins - 1;
}

// Accumulators of a large node (one slot per large node of the level).
struct NodeAcc {
  unsigned long long cmin[3], cmax[3];  // order keys of the centroid bounds
  unsigned bmin[3], bmax[3];            // order bits of the box
  int cnt[4];
};

struct BinAcc {
  int cnt[4];
  unsigned bmin[3], bmax[3];
};

// Per-node results of the split decision that the partition pass reads.
struct BinX {
  int* slot_of;     // large-node slot of a node of the current level, -1 for small nodes
  int* split_bin;   // plane j: bins [0, j) go left
  double* bin_lo;   // centroid lower bound on the split axis
  double* bin_scale;
};

struct SplitCfg {
  int bins, leaf_size, weighted;
  double traversal, lambda;
  double measured[4];
};

__device__ __forceinline__ void bin_clear(BinAcc& b) {
  for (int t = 0; t < 4; ++t) b.cnt[t] = 0;
  for (int k = 0; k < 3; ++k) {
    b.bmin[k] = 0xFFFFFFFFu;
    b.bmax[k] = 0u;
  }
}

__device__ __forceinline__ void bin_merge(BinAcc& a, const BinAcc& b) {
  for (int t = 0; t < 4; ++t) a.cnt[t] += b.cnt[t];
  for (int k = 0; k < 3; ++k) {
    a.bmin[k] = min(a.bmin[k], b.bmin[k]);
    a.bmax[k] = max(a.bmax[k], b.bmax[k]);
  }
}

__device__ __forceinline__ BinAcc bin_shfl_up(const BinAcc& v, int off) {
  BinAcc r;
  for (int t = 0; t < 4; ++t) r.cnt[t] = __shfl_up_sync(kFull, v.cnt[t], off);
  for (int k = 0; k < 3; ++k) {
    r.bmin[k] = __shfl_up_sync(kFull, v.bmin[k], off);
    r.bmax[k] = __shfl_up_sync(kFull, v.bmax[k], off);
  }
  return r;
}

__device__ __forceinline__ BinAcc bin_shfl_down(const BinAcc& v, int off) {
  BinAcc r;
  for (int t = 0; t < 4; ++t) r.cnt[t] = __shfl_down_sync(kFull, v.cnt[t], off);
  for (int k = 0; k < 3; ++k) {
    r.bmin[k] = __shfl_down_sync(kFull, v.bmin[k], off);
    r.bmax[k] = __shfl_down_sync(kFull, v.bmax[k], off);
  }
  return r;
}

__device__ __forceinline__ double set_weight(const int* cnt, const double* wt) {
  double w = (double)cnt[0] * wt[0];
  w = w + (double)cnt[1] * wt[1];
  w = w + (double)cnt[2] * wt[2];
  w = w + (double)cnt[3] * wt[3];
  return w;
}

__device__ __forceinline__ Box box_of(const unsigned* bmin, const unsigned* bmax) {
  Box b;
  for (int k = 0; k < 3; ++k) {
    b.mn[k] = o2f(bmin[k]);
    b.mx[k] = o2f(bmax[k]);
  }
  return b;
}

__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int off = 16; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(kFull, v, off);
    v = o < v ? o : v;
  }
  return v;
}
__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
  for (int off = 16; off > 0; off >>= 1) {
    unsigned long long o = __shfl_xor_sync(kFull, v, off);
    v = o > v ? o : v;
  }
  return v;
}

__global__ void k_iota(int* idx, int n) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) idx[j] = j;
}

__global__ void k_init_acc(NodeAcc* acc, BinAcc* bins, int slots) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < slots) {
    NodeAcc a;
    for (int k = 0; k < 3; ++k) {
      a.cmin[k] = ~0ULL;
      a.cmax[k] = 0ULL;
      a.bmin[k] = 0xFFFFFFFFu;
      a.bmax[k] = 0u;
    }
    for (int t = 0; t < 4; ++t) a.cnt[t] = 0;
    acc[i] = a;
  }
  if (i < slots * 96) {
    BinAcc b;
    bin_clear(b);
    bins[i] = b;
  }
}

// Bounds and type counts of every large node: positions of one node are contiguous, so a
// warp reduces each run of equal slots with shuffles and the run's first lane commits it.
__global__ void k_node_acc(const Prims P, const int* idx, const int* key, const int* level_of, int level,
                           const int* slot_of, int n, NodeAcc* acc) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int lane = threadIdx.x & 31;
  int slot = -1;
  if (j < n) {
    int node = key[j];
    if (level_of[node] == level) slot = slot_of[node];
  }
  unsigned long long cmn[3], cmx[3];
  unsigned bmn[3], bmx[3];
  int t = -1;
  if (slot >= 0) {
    int p = idx[j];
    t = P.type[p];
    for (int k = 0; k < 3; ++k) {
      cmn[k] = cmx[k] = order_key(P.cen[k][p]);
      bmn[k] = f2o(P.lo[k][p]);
      bmx[k] = f2o(P.hi[k][p]);
    }
  } else {
    for (int k = 0; k < 3; ++k) {
      cmn[k] = ~0ULL;
      cmx[k] = 0ULL;
      bmn[k] = 0xFFFFFFFFu;
      bmx[k] = 0u;
    }
  }
  for (int off = 1; off < 32; off <<= 1) {
    int os = __shfl_down_sync(kFull, slot, off);
    bool take = lane + off < 32 && os == slot;
    for (int k = 0; k < 3; ++k) {
      unsigned long long a = __shfl_down_sync(kFull, cmn[k], off);
      unsigned long long b = __shfl_down_sync(kFull, cmx[k], off);
      unsigned c = __shfl_down_sync(kFull, bmn[k], off);
      unsigned d = __shfl_down_sync(kFull, bmx[k], off);
      if (take) {
        cmn[k] = a < cmn[k] ? a : cmn[k];
        cmx[k] = b > cmx[k] ? b : cmx[k];
        bmn[k] = min(bmn[k], c);
        bmx[k] = max(bmx[k], d);
      }
    }
  }
  unsigned run = __match_any_sync(kFull, slot);
  unsigned tmask[4];
  for (int q = 0; q < 4; ++q) tmask[q] = __ballot_sync(kFull, t == q);
  int prev = __shfl_up_sync(kFull, slot, 1);
  bool head = slot >= 0 && (lane == 0 || prev != slot);
  if (head) {
    NodeAcc& A = acc[slot];
    for (int k = 0; k < 3; ++k) {
      atomicMin(&A.cmin[k], cmn[k]);
      atomicMax(&A.cmax[k], cmx[k]);
      atomicMin(&A.bmin[k], bmn[k]);
      atomicMax(&A.bmax[k], bmx[k]);
    }
    for (int q = 0; q < 4; ++q) {
      int c = __popc(run & tmask[q]);
      if (c) atomicAdd(&A.cnt[q], c);
    }
  }
}

// Bin accumulation of the large nodes.  Each block takes kChunk positions; the node that
// owns the chunk's first position accumulates in shared memory (flushed once), any other
// large node of the chunk directly in global memory.  Within a warp, lanes that hit the
// same (node, axis, bin) form a __match_any_sync group whose leader commits the group's
// per-type counts (popcounts of type ballots) and box bounds (group reductions).
__global__ void __launch_bounds__(256) k_bin_large(const Prims P, const int* idx, const int* key,
                                                   const int* level_of, int level, const int* slot_of,
                                                   const NodeAcc* acc, int n, int bins, BinAcc* gbins) {
  __shared__ BinAcc sb[96];
  int c0 = blockIdx.x * kChunk;
  int c1 = min(n, c0 + kChunk);
  for (int i = threadIdx.x; i < 96; i += blockDim.x) bin_clear(sb[i]);
  int pnode = key[c0];
  int pslot = level_of[pnode] == level ? slot_of[pnode] : -1;
  __syncthreads();
  int lane = threadIdx.x & 31;
  for (int base = c0; base < c1; base += blockDim.x) {
    int j = base + threadIdx.x;
    int slot = -1;
    if (j < c1) {
      int node = key[j];
      if (level_of[node] == level) slot = slot_of[node];
    }
    int p = slot >= 0 ? idx[j] : 0;
    int t = slot >= 0 ? P.type[p] : -1;
    unsigned tmask[4];
    for (int q = 0; q < 4; ++q) tmask[q] = __ballot_sync(kFull, t == q);
    unsigned lo[3], hi[3];
    if (slot >= 0)
      for (int k = 0; k < 3; ++k) {
        lo[k] = f2o(P.lo[k][p]);
        hi[k] = f2o(P.hi[k][p]);
      }
    for (int a = 0; a < 3; ++a) {
      int b = -1;
      if (slot >= 0) {
        double clo = k2d(acc[slot].cmin[a]);
        double ext = k2d(acc[slot].cmax[a]) - clo;
        if (ext > kMinExtent) b = bin_of(P.cen[a][p], clo, (double)bins / ext, bins);
      }
      unsigned act = __ballot_sync(kFull, b >= 0);
      if (b < 0) continue;
      unsigned grp = __match_any_sync(act, slot * 96 + a * 32 + b);
      unsigned gmn[3], gmx[3];
      for (int k = 0; k < 3; ++k) {
        gmn[k] = __reduce_min_sync(grp, lo[k]);
        gmx[k] = __reduce_max_sync(grp, hi[k]);
      }
      if (lane == __ffs(grp) - 1) {
        BinAcc* dst = slot == pslot ? &sb[a * 32 + b] : &gbins[((size_t)slot * 3 + a) * 32 + b];
        for (int q = 0; q < 4; ++q) {
          int c = __popc(grp & tmask[q]);
          if (c) atomicAdd(&dst->cnt[q], c);
        }
        for (int k = 0; k < 3; ++k) {
          atomicMin(&dst->bmin[k], gmn[k]);
          atomicMax(&dst->bmax[k], gmx[k]);
        }
      }
    }
  }
  __syncthreads();
  if (pslot < 0) return;
  for (int i = threadIdx.x; i < 96; i += blockDim.x) {
    const BinAcc& s = sb[i];
    if ((s.cnt[0] | s.cnt[1] | s.cnt[2] | s.cnt[3]) == 0) continue;
    BinAcc* g = &gbins[(size_t)pslot * 96 + i];
    for (int q = 0; q < 4; ++q)
      if (s.cnt[q]) atomicAdd(&g->cnt[q], s.cnt[q]);
    for (int k = 0; k < 3; ++k) {
      atomicMin(&g->bmin[k], s.bmin[k]);
      atomicMax(&g->bmax[k], s.bmax[k]);
    }
  }
}

// Split decision of every active node, one warp per node.
__global__ void __launch_bounds__(256) k_split_binned(const Prims P, const int* idx, Nodes N, BinX X,
                                                      const int* active, int k, SplitCfg S,
                                                      const NodeAcc* acc, const BinAcc* gbins,
                                                      int* counters, int* next_active, int* level_of,
                                                      int level) {
  __shared__ BinAcc sb[8][32];
  int warp = threadIdx.x >> 5;
  int lane = threadIdx.x & 31;
  int g = blockIdx.x * 8 + warp;
  if (g >= k) return;
  int node = active[g];
  int s = N.start[node], e = N.end[node];
  int n = e - s;
  int slot = X.slot_of[node];
  double wt[4];
  for (int q = 0; q < 4; ++q) wt[q] = S.weighted ? 1.0 + S.lambda * (S.measured[q] - 1.0) : 1.0;

  unsigned long long cmn[3], cmx[3];
  unsigned bmn[3], bmx[3];
  int cnt[4];
  int hp[kPerLane];
  if (slot >= 0) {
    const NodeAcc& A = acc[slot];
    for (int q = 0; q < 3; ++q) {
      cmn[q] = A.cmin[q];
      cmx[q] = A.cmax[q];
      bmn[q] = A.bmin[q];
      bmx[q] = A.bmax[q];
    }
    for (int q = 0; q < 4; ++q) cnt[q] = A.cnt[q];
  } else {
    for (int q = 0; q < 3; ++q) {
      cmn[q] = ~0ULL;
      cmx[q] = 0ULL;
      bmn[q] = 0xFFFFFFFFu;
      bmx[q] = 0u;
    }
    for (int q = 0; q < 4; ++q) cnt[q] = 0;
    for (int i = 0; i < kPerLane; ++i) {
      int j = s + lane + 32 * i;
      int p = j < e ? idx[j] : -1;
      hp[i] = p;
      int t = p >= 0 ? P.type[p] : -1;
      for (int q = 0; q < 4; ++q) cnt[q] += __popc(__ballot_sync(kFull, t == q));
      if (p < 0) continue;
      for (int q = 0; q < 3; ++q) {
        unsigned long long c = order_key(P.cen[q][p]);
        cmn[q] = c < cmn[q] ? c : cmn[q];
        cmx[q] = c > cmx[q] ? c : cmx[q];
        bmn[q] = min(bmn[q], f2o(P.lo[q][p]));
        bmx[q] = max(bmx[q], f2o(P.hi[q][p]));
      }
    }
    for (int q = 0; q < 3; ++q) {
      cmn[q] = warp_min_u64(cmn[q]);
      cmx[q] = warp_max_u64(cmx[q]);
      bmn[q] = __reduce_min_sync(kFull, bmn[q]);
      bmx[q] = __reduce_max_sync(kFull, bmx[q]);
    }
  }
  Box nb = box_of(bmn, bmx);
  double area = surface_area(nb);
  double wnode = set_weight(cnt, wt);

  bool have = false;
  double best_cost = 0.0, best_lo = 0.0, best_scale = 0.0;
  int best_axis = -1, best_plane = 0, best_left = 0;
  for (int a = 0; a < 3 && n > 1; ++a) {
    double clo = k2d(cmn[a]);
    double ext = k2d(cmx[a]) - clo;
    if (!(ext > kMinExtent)) continue;
    double scale = (double)S.bins / ext;
    BinAcc v;
    if (slot >= 0) {
      if (lane < S.bins) v = gbins[((size_t)slot * 3 + a) * 32 + lane];
      else bin_clear(v);
    } else {
      bin_clear(sb[warp][lane]);
      __syncwarp();
      for (int i = 0; i < kPerLane; ++i) {
        int p = hp[i];
        if (p < 0) continue;
        int b = bin_of(P.cen[a][p], clo, scale, S.bins);
        BinAcc& d = sb[warp][b];
        atomicAdd(&d.cnt[P.type[p]], 1);
        for (int q = 0; q < 3; ++q) {
          atomicMin(&d.bmin[q], f2o(P.lo[q][p]));
          atomicMax(&d.bmax[q], f2o(P.hi[q][p]));
        }
      }
      __syncwarp();
      v = sb[warp][lane];
      __syncwarp();
    }
    // Inclusive prefix (bins 0..lane) and suffix (bins lane..31) in registers.
    BinAcc L = v, R = v;
    for (int off = 1; off < 32; off <<= 1) {
      BinAcc u = bin_shfl_up(L, off);
      BinAcc d = bin_shfl_down(R, off);
      if (lane >= off) bin_merge(L, u);
      if (lane + off < 32) bin_merge(R, d);
    }
    BinAcc left = bin_shfl_up(L, 1);  // bins [0, lane)
    int nl = left.cnt[0] + left.cnt[1] + left.cnt[2] + left.cnt[3];
    int nr = R.cnt[0] + R.cnt[1] + R.cnt[2] + R.cnt[3];
    double cost = CUDART_INF;
    if (lane >= 1 && lane < S.bins && nl > 0 && nr > 0) {
      double x = area * S.traversal;
      double y = surface_area(box_of(left.bmin, left.bmax)) * set_weight(left.cnt, wt);
      double z = surface_area(box_of(R.bmin, R.bmax)) * set_weight(R.cnt, wt);
      cost = (x + y) + z;
    }
    // first minimum over the planes of this axis
    double mc = cost;
    int mj = lane;
    for (int off = 16; off > 0; off >>= 1) {
      double oc = __shfl_xor_sync(kFull, mc, off);
      int oj = __shfl_xor_sync(kFull, mj, off);
      if (oc < mc || (oc == mc && oj < mj)) {
        mc = oc;
        mj = oj;
      }
    }
    int mleft = __shfl_sync(kFull, nl, mj);
    if (mc != CUDART_INF && (!have || mc < best_cost)) {
      have = true;
      best_cost = mc;
      best_axis = a;
      best_plane = mj;
      best_left = mleft;
      best_lo = clo;
      best_scale = scale;
    }
  }

  bool leaf = n == 1;
  bool median = false;
  if (!leaf) {
    if (!have) {
      if (n <= S.leaf_size) leaf = true;
      else median = true;
    } else if (n <= S.leaf_size && !(best_cost < area * wnode)) {
      leaf = true;
    }
  }
  if (lane != 0) return;
  N.bounds[node] = nb;
  int* stats = counters + 2;
  if (leaf) {
    N.leaf[node] = 1;
    N.split_axis[node] = -1;
    atomicAdd(stats + 0, 1);
    atomicMin(stats + 1, n);
    atomicMax(stats + 2, n);
    atomicMax(stats + 3, N.depth[node]);
    return;
  }
  int lc = median ? n / 2 : best_left;
  int c = atomicAdd(counters + 0, 2);
  int l = c, r = c + 1;
  N.leaf[node] = 0;
  N.left[node] = l;
  N.right[node] = r;
  N.split_axis[node] = median ? 3 : best_axis;
  N.split_pos[node] = lc;
  X.split_bin[node] = best_plane;
  X.bin_lo[node] = best_lo;
  X.bin_scale[node] = best_scale;
  N.start[l] = s;
  N.end[l] = s + lc;
  N.start[r] = s + lc;
  N.end[r] = e;
  N.order_axis[l] = N.order_axis[r] = 0;
  N.depth[l] = N.depth[r] = N.depth[node] + 1;
  N.leaf[l] = N.leaf[r] = 0;
  level_of[l] = level_of[r] = level + 1;
  X.slot_of[l] = lc > kSmall ? atomicAdd(counters + 6, 1) : -1;
  X.slot_of[r] = n - lc > kSmall ? atomicAdd(counters + 6, 1) : -1;
  atomicMax(stats + 3, N.depth[node] + 1);
  int q = atomicAdd(counters + 1, 2);
  next_active[q] = l;
  next_active[q + 1] = r;
}

__global__ void k_sides_binned(const Prims P, const int* idx, const Nodes N, BinX X, const int* key,
                               const int* level_of, int level, int n, int bins, unsigned char* side) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  if (level_of[node] != level) return;
  int axis = N.split_axis[node];
  if (axis < 0) return;
  int p = idx[j];
  if (axis == 3)
    side[p] = (j - N.start[node]) >= N.split_pos[node] ? 1 : 0;
  else
    side[p] = bin_of(P.cen[axis][p], X.bin_lo[node], X.bin_scale[node], bins) >= X.split_bin[node] ? 1 : 0;
}

// Stable partition scatter that checks every destination against the node's range (the
// left count comes from the bins and must equal the flags' count); a mismatch is counted
// in *error and the write is skipped.
__global__ void k_scatter_checked(const int* idx, const Nodes N, const int* key, const int* level_of,
                                  int level, int n, const unsigned char* side, const int* lscan, int* out,
                                  int* error) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  int p = idx[j];
  if (!(level_of[node] == level && N.split_axis[node] >= 0)) {
    out[j] = p;
    return;
  }
  int s = N.start[node], e = N.end[node];
  int lc = N.split_pos[node];
  int lrank = lscan[j] - lscan[s];
  int rrank = (j - s) - lrank;
  int dst = side[p] == 0 ? s + lrank : s + lc + rrank;
  bool ok = side[p] == 0 ? lrank < lc : lc + rrank < e - s;
  if (!ok) {
    atomicAdd(error, 1);
    return;
  }
  out[dst] = p;
}

}  // namespace

rtb_status build_bvh_binned(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                            int bins, rtb_scene** out, rtb_bvh_stats* stats) {
  if (!out) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (bins < 2 || bins > 32) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "binned BVH build needs 2..32 bins");
  BuildCfg c;
  bool per_type = false;
  rtb_status st = build_setup(ctx, desc, cfg, c, per_type);
  if (st != RTB_OK) return st;
  if (stats) *stats = rtb_bvh_stats{};
  if (c.total == 0) {
    rtb_status s = scene_create(ctx, desc, nullptr, nullptr, nullptr, 0, nullptr, 0, nullptr, 0, out);
    if (stats) stats->leaf_size = cfg->leaf_size;
    return s;
  }
  const int n = c.total;
  cudaStream_t sm = ctx->stream;
  Workspace W;
  W.stream = sm;
  PrimInputs in = alloc_inputs(W, c);
  Prims P = alloc_prims(W, n);
  int* idx = W.alloc<int>(n);
  int* tmp_idx = W.alloc<int>(n);
  int cap = 2 * n + 8;
  Nodes N = alloc_nodes(W, cap);
  BinX X;
  X.slot_of = W.alloc<int>(cap);
  X.split_bin = W.alloc<int>(cap);
  X.bin_lo = W.alloc<double>(cap);
  X.bin_scale = W.alloc<double>(cap);
  int max_slots = n / (kSmall + 1) + 4;
  NodeAcc* acc = W.alloc<NodeAcc>(max_slots);
  BinAcc* gbins = W.alloc<BinAcc>((size_t)max_slots * 96);
  int* level_of = W.alloc<int>(cap);
  int* key = W.alloc<int>(n);
  unsigned char* side = W.alloc<unsigned char>(n);
  int* flags = W.alloc<int>(n);
  int* lscan = W.alloc<int>(n);
  int* active = W.alloc<int>(cap);
  int* next_active = W.alloc<int>(cap);
  int* all_nodes = W.alloc<int>(cap);
  // node counter, next count, stats {leaves, min occupancy, max occupancy, max depth},
  // next large count, partition errors
  int* counters = W.alloc<int>(8);
  int* root_start = W.alloc<int>(4);
  int* root_end = W.alloc<int>(4);
  size_t tmp_bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, flags, lscan, n);
  void* tmp = W.alloc<char>(tmp_bytes);
  if (!W.ok) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "BVH build workspace");

  cudaEventRecord(ctx->ev0, sm);
  upload_prims(desc, c, in, P, sm);
  k_iota<<<blocks(n), 256, 0, sm>>>(idx, n);

  int h_rs[4], h_re[4];
  int roots = root_ranges(c, per_type, h_rs, h_re);
  std::vector<int> h_init(roots), h_slot(roots);
  int large = 0;
  for (int r = 0; r < roots; ++r) {
    h_init[r] = r;
    h_slot[r] = h_re[r] - h_rs[r] > kSmall ? large++ : -1;
  }
  int h_counters[8] = {roots, 0, 0, 0x7FFFFFFF, 0, 0, 0, 0};
  cudaMemcpyAsync(root_start, h_rs, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(root_end, h_re, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(N.start, h_rs, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(N.end, h_re, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(X.slot_of, h_slot.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(active, h_init.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(all_nodes, h_init.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(counters, h_counters, sizeof(h_counters), cudaMemcpyHostToDevice, sm);
  cudaMemsetAsync(N.order_axis, 0, (size_t)roots * 4, sm);
  cudaMemsetAsync(N.depth, 0, (size_t)roots * 4, sm);
  cudaMemsetAsync(level_of, 0, (size_t)roots * 4, sm);
  k_init_keys<<<blocks(n), 256, 0, sm>>>(key, root_start, root_end, roots, n);

  SplitCfg S;
  S.bins = bins;
  S.leaf_size = c.leaf_size;
  S.weighted = c.weighted;
  S.traversal = c.traversal;
  S.lambda = c.lambda;
  for (int q = 0; q < 4; ++q) S.measured[q] = c.measured[q];

  std::vector<int> level_begin = {0};
  int k = roots, level = 0, total_nodes = roots;
  while (k > 0) {
    level_begin.push_back(level_begin.back() + k);
    if (large > 0) {
      k_init_acc<<<blocks((long long)large * 96), 256, 0, sm>>>(acc, gbins, large);
      k_node_acc<<<blocks(n), 256, 0, sm>>>(P, idx, key, level_of, level, X.slot_of, n, acc);
      k_bin_large<<<blocks(n, kChunk), 256, 0, sm>>>(P, idx, key, level_of, level, X.slot_of, acc, n,
                                                      bins, gbins);
    }
    cudaMemsetAsync(counters + 1, 0, 4, sm);
    cudaMemsetAsync(counters + 6, 0, 4, sm);
    k_split_binned<<<blocks(k, 8), 256, 0, sm>>>(P, idx, N, X, active, k, S, acc, gbins, counters,
                                                 next_active, level_of, level);
    k_sides_binned<<<blocks(n), 256, 0, sm>>>(P, idx, N, X, key, level_of, level, n, bins, side);
    k_left_flags<<<blocks(n), 256, 0, sm>>>(idx, N, key, level_of, level, n, side, flags);
    size_t tb = tmp_bytes;
    cub::DeviceScan::ExclusiveSum(tmp, tb, flags, lscan, n, sm);
    k_scatter_checked<<<blocks(n), 256, 0, sm>>>(idx, N, key, level_of, level, n, side, lscan, tmp_idx,
                                                 counters + 7);
    std::swap(idx, tmp_idx);
    k_update_keys<<<blocks(n), 256, 0, sm>>>(N, level_of, level, n, key);
    int h[8];
    cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "binned BVH build level");
    if (h[7] != 0) return fail(ctx, RTB_ERR_DEVICE_CHECK, "binned BVH partition disagrees with its bins");
    int next = h[1];
    if (next > 0) {
      cudaMemcpyAsync(all_nodes + total_nodes, next_active, (size_t)next * 4, cudaMemcpyDeviceToDevice, sm);
      std::swap(active, next_active);
    }
    total_nodes += next;
    large = h[6];
    k = next;
    level++;
  }
  IdxSet I;
  for (int a = 0; a < 3; ++a) I.a[a] = idx;
  return finish_build(ctx, desc, cfg, W, c, P, I, N, all_nodes, level_begin, roots, total_nodes,
                      counters, out, stats);
}

}  // namespace rtb
