// Device BVH builder: the reference's full-sweep, primitive-cost-weighted object SAH
// (gfxlab/gpu/GpuScene.java BvhBuildState, 1414-1499) executed level by level on the GPU,
// producing the same tree node for node and the same flattened arrays
// (flattenBvh / leafKind, GpuScene.java:772-808).
//
// How the Java recursion maps onto data-parallel passes:
//  * bestSplit sorts a node's primitives on each axis by (centroid, order) with
//    Double.compare.  That order restricted to any subset is the global order restricted
//    to it, so the three axis orders are sorted ONCE (radix sort on an order-preserving
//    64-bit image of the double centroid, stable for the order tie-break) and every split
//    stable-partitions each axis array inside the node's range.
//  * Prefix and suffix bounds are exact min/max unions: segmented scans.
//  * Prefix and suffix weights are SEQUENTIAL double sums in the reference; with
//    non-dyadic weights (1.3, 2.1) their rounding depends on the order.  With unit weights
//    the sums are exact integers and are written directly.  Otherwise a node of more than
//    kSeqNodeSize primitives takes its weights from per-type counts (a segmented integer
//    scan), summed exactly and rounded once, and its costs carry a rigorous bound on how far
//    the reference's sequentially rounded costs can be from them; its argmin is the
//    reference's whenever every other candidate's cost minus its bound exceeds the winner's
//    cost plus its bound.  Smaller nodes, and the few large ones whose winner is not that
//    clear, sum their weights sequentially per (node, axis, direction), the reference's own
//    additions in its own order.
//  * Costs are evaluated in double with the reference's expression order
//    (nodeArea*cT + A_L*W_L) + A_R*W_R; the argmin keeps the first minimum in
//    (axis, position) order, as the strict '<' does.
//  * The leaf test (count <= leafSize and !(cost < area * sequential weight sum in the
//    node's current order)) uses the parent's split-axis order, which is the order the
//    Java primitives array holds when build() reaches the node.
// The file is compiled with -fmad=false: no double expression is contracted.
#include "rtb_build_common.cuh"

namespace rtb {
namespace {

__global__ void k_keys(const Prims P, int axis, int n, unsigned long long* keys, int* vals) {
  int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  keys[p] = order_key(P.cen[axis][p]);
  vals[p] = p;
}

__global__ void k_type_keys(const Prims P, const int* idx, int n, int* keys) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) keys[j] = P.type[idx[j]];
}


__global__ void k_gather_weights(const Prims P, const int* idx, int n, double* wpos) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j < n) wpos[j] = P.w[idx[j]];
}

// Unit construction weights: prefix / suffix sums are exact integers, one thread per position.
__global__ void k_weights_unit(const Nodes N, const int* key, const int* level_of, int level, int n,
                               double* pw, double* sw) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  if (level_of[node] != level) return;
  int s = N.start[node], e = N.end[node];
  pw[j] = (double)(j - s + 1);
  sw[j] = (double)(e - j);
}

// Weighted prefix / suffix sums in the reference's sequential order, one warp per
// (node, axis, direction), all three axes in one launch: the warp loads 32 weights at a
// time (coalesced, the next chunk prefetched), broadcasts them to every lane with all 32
// shuffles issued ahead, and every lane then runs the same strictly sequential chain of 32
// additions, lane j keeping the running sum after element j.  The additions happen in
// exactly the Java loop's order (0 + w0 = w0 exactly, then one add per element), so every
// partial sum is bit-identical to it; only the loads and shuffles are parallel.
struct WeightChains {
  const double* w[3];  // weights in each axis order
  double* pw[3];
  double* sw[3];
};

// `nodes` lists the nodes to sum; their number is *count when count is given (a list built
// on the device; k is then only the grid's bound), else k.
__global__ void __launch_bounds__(128) k_weights_seq(const WeightChains C, const Nodes N, const int* nodes,
                                                     int k, const int* count) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (count) k = min(k, *count);
  if (warp >= 6 * k) return;
  const int* active = nodes;
  int node = active[warp / 6];
  int axis = (warp >> 1) % 3;
  bool suffix = warp & 1;
  int s = N.start[node], e = N.end[node];
  int n = e - s;
  if (n < 2) return;
  const double* wp = C.w[axis];
  double* out = suffix ? C.sw[axis] : C.pw[axis];
  double acc = 0.0;
  double w = lane < n ? wp[suffix ? e - 1 - lane : s + lane] : 0.0;
  for (int base = 0; base < n; base += 32) {
    int j = base + lane;
    int pos = suffix ? e - 1 - j : s + j;
    int jn = j + 32;
    double wn = jn < n ? wp[suffix ? e - 1 - jn : s + jn] : 0.0;  // next chunk
    double mine = 0.0;
    if (n - base >= 32) {
      double v[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) v[q] = __shfl_sync(0xFFFFFFFFu, w, q);
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        acc = acc + v[q];
        mine = q == lane ? acc : mine;
      }
    } else {
      int m = n - base;
      for (int q = 0; q < m; ++q) {
        double v = __shfl_sync(0xFFFFFFFFu, w, q);
        acc = acc + v;
        if (q == lane) mine = acc;
      }
    }
    if (j < n) out[pos] = mine;
    w = wn;
  }
}

// ---- certified weights for large nodes
//
// Nodes above kSeqNodeSize primitives: prefix weight of positions [s, j] = sum over the four
// primitive types of (count of that type in [s, j]) x (its construction weight), from a
// segmented inclusive scan of per-type counts, summed in double-double (each product split
// exactly with fma) and rounded once.  The reference's sequential sum of the same k weights
// (all positive) is within (k - 1) u of the exact sum relatively (u = 2^-53, the standard
// bound for recursive summation), so each cost gets a bound on its distance from the
// reference's: the weight errors times the areas, plus the cost expression's own roundings
// in both evaluations, doubled for margin.
constexpr int kSeqNodeSize = 256;

struct TypeCounts {
  unsigned long long a, b;  // (sphere | box << 32), (affine sphere | affine box << 32)
};
// sum_t c_t w_t, exact in double-double, rounded once: within one rounding of the true sum.
__device__ __forceinline__ double counts_weight(TypeCounts c, const double* wt) {
  double cnt[4] = {(double)(c.a & 0xFFFFFFFFULL), (double)(c.a >> 32), (double)(c.b & 0xFFFFFFFFULL),
                   (double)(c.b >> 32)};
  double hi = 0.0, lo = 0.0;
  for (int t = 0; t < 4; ++t) {
    double p = cnt[t] * wt[t];
    double pe = fma(cnt[t], wt[t], -p);  // exact: cnt < 2^32 is an integer
    double s = hi + p;                    // two-sum of hi and p
    double bp = s - hi;
    double se = (hi - (s - bp)) + (p - bp);
    hi = s;
    lo = lo + (se + pe);
  }
  return hi + lo;
}

struct TypeWeights {
  double w[4];
};

// ---- segmented scans over node-sorted positions
//
// The positions are sorted by node (key[j]), every node one contiguous segment.  For every
// position j of a node at the current level, the forward scan gives the combination of the
// values over [start of j's node, j] and the backward scan over [j, end of j's node].  Three
// launches cover all three axes: every chunk of kSegChunk positions reduces to its partial
// aggregates in both directions (k_seg_chunks); one block per (axis, direction) carries
// them across the chunks (k_seg_carries); every chunk then scans again with its carries and
// hands each position's results to a consumer (k_seg_apply) that evaluates the split costs
// or the count-based weights in place, so no scanned array is written.  Chunks holding no
// position of a node at the current level do no work (a node at the level never spans
// such a chunk).  Box unions (min / max) and integer sums are exact, so any association of
// them gives the sequential result bit for bit.
#ifndef RTB_SEG_ITEMS
#define RTB_SEG_ITEMS 4
#endif
constexpr int kSegThreads = 256, kSegItems = RTB_SEG_ITEMS, kSegChunk = kSegThreads * kSegItems;
constexpr int kSegWarps = kSegThreads / 32, kCarryThreads = 1024;

template <class V>
struct Seg {
  int flag;  // a segment starts inside the span (in scan order): v starts there
  V v;
};

template <bool DOWN, class V>
__device__ __forceinline__ V shfl_v(V x, int d) {
  static_assert(sizeof(V) % 4 == 0, "values of whole words");
  constexpr int kWords = sizeof(V) / 4;
  int w[kWords];
  memcpy(w, &x, sizeof(V));
#pragma unroll
  for (int q = 0; q < kWords; ++q)
    w[q] = DOWN ? __shfl_down_sync(0xFFFFFFFFu, w[q], d) : __shfl_up_sync(0xFFFFFFFFu, w[q], d);
  memcpy(&x, w, sizeof(V));
  return x;
}

// Segmented scan of a block's items in scan order: thread by thread, ITEMS consecutive
// positions each; REV runs from the block's last position down.  flag[i] marks the first
// position of a segment in scan order.  before[i] / incl[i] combine the segment's values up
// to item i, excluding / including it, with `carry` standing for all positions ahead of
// the block.  Returns the block's own aggregate (carry left out).
template <class O, bool REV, int ITEMS, int WARPS>
__device__ __forceinline__ Seg<typename O::V> seg_scan_block(const int (&flag)[ITEMS],
                                                             const typename O::V (&v)[ITEMS],
                                                             typename O::V carry,
                                                             typename O::V (&before)[ITEMS],
                                                             typename O::V (&incl)[ITEMS],
                                                             Seg<typename O::V>* s_warp) {
  using V = typename O::V;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  int tf = 0;
  V tv = O::identity();
#pragma unroll
  for (int q = 0; q < ITEMS; ++q) {
    const int i = REV ? ITEMS - 1 - q : q;
    tv = flag[i] ? v[i] : O::combine(tv, v[i]);
    tf |= flag[i];
  }
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int of = REV ? __shfl_down_sync(0xFFFFFFFFu, tf, d) : __shfl_up_sync(0xFFFFFFFFu, tf, d);
    V ov = shfl_v<REV>(tv, d);
    if (REV ? lane + d < 32 : lane >= d) {
      if (!tf) tv = O::combine(ov, tv);
      tf |= of;
    }
  }
  int ef = REV ? __shfl_down_sync(0xFFFFFFFFu, tf, 1) : __shfl_up_sync(0xFFFFFFFFu, tf, 1);
  V ev = shfl_v<REV>(tv, 1);
  if (REV ? lane == 31 : lane == 0) {
    ef = 0;
    ev = O::identity();
  }
  if (REV ? lane == 0 : lane == 31) s_warp[w] = Seg<V>{tf, tv};
  __syncthreads();
  V acc = carry;
  Seg<V> agg{0, O::identity()};
  for (int q = 0; q < WARPS; ++q) {
    const int u = REV ? WARPS - 1 - q : q;
    const Seg<V> s = s_warp[u];
    if (REV ? u > w : u < w) acc = s.flag ? s.v : O::combine(acc, s.v);
    agg.v = s.flag ? s.v : O::combine(agg.v, s.v);
    agg.flag |= s.flag;
  }
  V run = ef ? ev : O::combine(acc, ev);
#pragma unroll
  for (int q = 0; q < ITEMS; ++q) {
    const int i = REV ? ITEMS - 1 - q : q;
    before[i] = run;
    run = flag[i] ? v[i] : O::combine(run, v[i]);
    incl[i] = run;
  }
  __syncthreads();  // s_warp is free again
  return agg;
}

// One thread's kSegItems positions from j0: segment starts (head) and ends (tail), node
// ids, and values (the identity outside the loader's active nodes); bit i of the result is
// set when position j0 + i is active.  Positions past n are segments of their own.
template <class L>
__device__ __forceinline__ int seg_load(const L& load, const int* key, int n, int a, int j0,
                                        int (&head)[kSegItems], int (&tail)[kSegItems],
                                        int (&node)[kSegItems], typename L::V (&v)[kSegItems]) {
  int act = 0;
  int kp = j0 > 0 && j0 <= n ? key[j0 - 1] : -1;
#pragma unroll
  for (int i = 0; i < kSegItems; ++i) {
    const int j = j0 + i;
    const int kj = j < n ? key[j] : -1;
    const int kn = j + 1 < n ? key[j + 1] : -1;
    node[i] = kj;
    head[i] = j >= n || j == 0 || kj != kp;
    tail[i] = j >= n || j == n - 1 || kj != kn;
    const bool on = j < n && load.active(kj);
    v[i] = on ? load(a, j) : L::identity();
    act |= (int)on << i;
    kp = kj;
  }
  return act;
}

// Per (chunk, axis): the chunk's aggregate in both directions.
template <class L>
__global__ void __launch_bounds__(kSegThreads) k_seg_chunks(const L load, const int* key, int n, int nc,
                                                            Seg<typename L::V>* fwd,
                                                            Seg<typename L::V>* bwd) {
  using V = typename L::V;
  __shared__ Seg<V> s_warp[kSegWarps];
  const int a = blockIdx.y, c = blockIdx.x;
  const int j0 = c * kSegChunk + threadIdx.x * kSegItems;
  int head[kSegItems], tail[kSegItems], node[kSegItems];
  V v[kSegItems], before[kSegItems], incl[kSegItems];
  const int act = seg_load(load, key, n, a, j0, head, tail, node, v);
  const size_t slot = (size_t)a * nc + c;
  if (!__syncthreads_or(act)) {
    if (threadIdx.x == 0) fwd[slot] = bwd[slot] = Seg<V>{1, L::identity()};
    return;
  }
  Seg<V> af = seg_scan_block<L, false, kSegItems, kSegWarps>(head, v, L::identity(), before, incl, s_warp);
  Seg<V> ab = seg_scan_block<L, true, kSegItems, kSegWarps>(tail, v, L::identity(), before, incl, s_warp);
  if (threadIdx.x == 0) {
    fwd[slot] = af;
    bwd[slot] = ab;
  }
}

// Per (axis, direction): chunk aggregates scanned in place over all chunks, 1024 at a time
// with a running carry; afterwards fwd[c] holds the forward result at chunk c's last
// position and bwd[c] the backward result at its first.
template <class O>
__global__ void __launch_bounds__(kCarryThreads) k_seg_carries(int nc, Seg<typename O::V>* fwd,
                                                               Seg<typename O::V>* bwd) {
  using V = typename O::V;
  __shared__ Seg<V> s_warp[kCarryThreads / 32];
  const bool rev = blockIdx.y != 0;
  Seg<V>* s = (rev ? bwd : fwd) + (size_t)blockIdx.x * nc;
  V carry = O::identity();
  const int tiles = (nc + kCarryThreads - 1) / kCarryThreads;
  for (int t = 0; t < tiles; ++t) {
    const int c = (rev ? tiles - 1 - t : t) * kCarryThreads + threadIdx.x;
    const Seg<V> x = c < nc ? s[c] : Seg<V>{1, O::identity()};
    int flag[1] = {x.flag};
    V v[1] = {x.v}, before[1], incl[1];
    Seg<V> agg = rev ? seg_scan_block<O, true, 1, kCarryThreads / 32>(flag, v, carry, before, incl, s_warp)
                     : seg_scan_block<O, false, 1, kCarryThreads / 32>(flag, v, carry, before, incl, s_warp);
    if (c < nc) s[c] = Seg<V>{x.flag, incl[0]};
    carry = agg.flag ? agg.v : O::combine(carry, agg.v);
  }
}

// Per (chunk, axis): both scans with the carries, each active position handed to `use`.
template <class L, class U>
__global__ void __launch_bounds__(kSegThreads) k_seg_apply(const L load, const U use, const int* key, int n,
                                                           int nc, const Seg<typename L::V>* fwd,
                                                           const Seg<typename L::V>* bwd) {
  using V = typename L::V;
  __shared__ Seg<V> s_warp[kSegWarps];
  const int a = blockIdx.y, c = blockIdx.x;
  const int j0 = c * kSegChunk + threadIdx.x * kSegItems;
  int head[kSegItems], tail[kSegItems], node[kSegItems];
  V v[kSegItems], fb[kSegItems], fi[kSegItems], bb[kSegItems], bi[kSegItems];
  const int act = seg_load(load, key, n, a, j0, head, tail, node, v);
  if (!__syncthreads_or(act)) return;
  const size_t slot = (size_t)a * nc + c;
  const V cf = c > 0 ? fwd[slot - 1].v : L::identity();
  const V cb = c + 1 < nc ? bwd[slot + 1].v : L::identity();
  seg_scan_block<L, false, kSegItems, kSegWarps>(head, v, cf, fb, fi, s_warp);
  seg_scan_block<L, true, kSegItems, kSegWarps>(tail, v, cb, bb, bi, s_warp);
#pragma unroll
  for (int i = 0; i < kSegItems; ++i)
    if (act >> i & 1) use(a, j0 + i, node[i], tail[i], fb[i], fi[i], bi[i]);
}

struct BoxOp {
  using V = Box;
  __device__ static Box identity() {
    Box b;
    for (int k = 0; k < 3; ++k) {
      b.mn[k] = CUDART_INF_F;
      b.mx[k] = -CUDART_INF_F;
    }
    return b;
  }
  __device__ static Box combine(const Box& x, const Box& y) { return BoxUnion()(x, y); }
};

struct CountOp {
  using V = TypeCounts;
  __device__ static TypeCounts identity() { return TypeCounts{0ULL, 0ULL}; }
  __device__ static TypeCounts combine(const TypeCounts& x, const TypeCounts& y) {
    return TypeCounts{x.a + y.a, x.b + y.b};
  }
};

// Primitive boxes in each axis order, for the nodes at the level.
struct BoxLoad : BoxOp {
  Prims P;
  IdxSet I;
  const int* level_of;
  int level;
  __device__ bool active(int node) const { return level_of[node] == level; }
  __device__ Box operator()(int a, int j) const { return P.box[I.a[a][j]]; }
};

// One-hot type counts in each axis order, for the level's nodes above kSeqNodeSize.
struct CountLoad : CountOp {
  Prims P;
  IdxSet I;
  Nodes N;
  const int* level_of;
  int level;
  __device__ bool active(int node) const {
    return level_of[node] == level && N.end[node] - N.start[node] > kSeqNodeSize;
  }
  __device__ TypeCounts operator()(int a, int j) const {
    int t = P.type[I.a[a][j]];
    unsigned long long one = 1ULL << (32 * (t & 1));
    return t < 2 ? TypeCounts{one, 0ULL} : TypeCounts{0ULL, one};
  }
};

// Count-based prefix and suffix weights of every position of a large node.
struct CountWeights {
  TypeWeights tw;
  double* pw[3];
  double* sw[3];
  __device__ void operator()(int a, int j, int, int, const TypeCounts&, const TypeCounts& upto,
                             const TypeCounts& from) const {
    pw[a][j] = counts_weight(upto, tw.w);
    sw[a][j] = counts_weight(from, tw.w);
  }
};

// Split cost of every position (GpuScene.java:1482-1485): cost[j] is the cost of putting
// positions [s, j) left; +inf marks positions that are not candidates.  The left bounds
// are the forward scan before j, the right bounds the backward scan at j, and the node's
// bounds their union (written once per node, at its last position, for the axis-0 pass).
// For nodes whose weights came from counts, bound[j] limits |cost[j] - the reference's cost|.
struct SplitCosts {
  Prims P;
  IdxSet I;
  Nodes N;
  const double* pw[3];
  const double* sw[3];
  double traversal;
  int certified;
  double* cost[3];
  double* bound[3];
  Box* node_box;  // node bounds at each node's last position
  __device__ void operator()(int a, int j, int node, int tail, const Box& left, const Box& upto,
                             const Box& right) const {
    if (a == 0 && tail) node_box[j] = upto;
    int s = N.start[node], e = N.end[node];
    double c = CUDART_INF;
    if (j > s && e - s > 1) {
      const int* idx = I.a[a];
      double ext = P.cen[a][idx[e - 1]] - P.cen[a][idx[s]];
      if (ext > 1.0e-12) {
        double an = surface_area(BoxUnion()(left, right)) * traversal;
        double al = surface_area(left);
        double ar = surface_area(right);
        double b = al * pw[a][j - 1];
        double d = ar * sw[a][j];
        c = (an + b) + d;
        if (certified && e - s > kSeqNodeSize) {
          const double u = 0x1p-53;
          double kl = (double)(j - s), kr = (double)(e - j);
          bound[a][j] = 2.0 * (al * pw[a][j - 1] * (kl * u) + ar * sw[a][j] * (kr * u) + 8.0 * u * c);
        }
      }
    }
    cost[a][j] = c;
  }
};

// Each active node's slot in the level's per-node arrays.
__global__ void k_node_slots(const int* active, int k, int* g_of_node) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < k) g_of_node[active[g]] = g;
}

// The winner's bound, and a cleared failure flag, per certified node.
__global__ void k_best_bound(const Nodes N, const int* active, int k, const double* best_cost,
                             const long long* best_flat, const double* bnd0, const double* bnd1,
                             const double* bnd2, double* best_bound, int* failed) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  failed[g] = 0;
  int node = active[g];
  int s = N.start[node], len = N.end[node] - s;
  if (len <= kSeqNodeSize || best_cost[g] == CUDART_INF) return;
  long long flat = best_flat[g];
  int axis = (int)(flat / len), pos = (int)(flat % len);
  const double* b = axis == 0 ? bnd0 : axis == 1 ? bnd1 : bnd2;
  best_bound[g] = b[s + pos];
}

// A certified node fails when some other candidate could, in the reference's rounding, cost
// as little as the winner.
__global__ void k_certify(const Nodes N, const int* key, const int* level_of, int level, int n,
                          const int* g_of_node, const double* cost0, const double* cost1,
                          const double* cost2, const double* bound0, const double* bound1,
                          const double* bound2, const double* best_cost, const long long* best_flat,
                          const double* best_bound, int* failed) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int axis = blockIdx.y;  // one axis per grid row
  const double* cost = axis == 0 ? cost0 : axis == 1 ? cost1 : cost2;
  const double* bound = axis == 0 ? bound0 : axis == 1 ? bound1 : bound2;
  int node = key[j];
  if (level_of[node] != level) return;
  int s = N.start[node], len = N.end[node] - s;
  if (len <= kSeqNodeSize) return;
  double c = cost[j];
  if (c == CUDART_INF) return;
  int g = g_of_node[node];
  if ((long long)axis * len + (j - s) == best_flat[g]) return;
  if (c - bound[j] <= best_cost[g] + best_bound[g]) failed[g] = 1;
}

__global__ void k_failed_list(const int* active, int k, const int* failed, int* out, int* count) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g < k && failed[g]) out[atomicAdd(count, 1)] = active[g];
}

struct Cand {
  double cost;
  long long flat;
};
__device__ __forceinline__ Cand better(Cand a, Cand b) {
  if (b.cost < a.cost || (b.cost == a.cost && b.flat < a.flat)) return b;
  return a;
}

// First minimum over (axis, position) for each active node, with a node's positions
// spread over fixed-size chunks so that the few huge nodes of the top levels use many blocks.  Every chunk reduces its positions
// (all three axes) to one (cost, flat) candidate; then the node's minimum cost and, among
// the chunks that reach it, the smallest flat index are taken with atomics.  The minimum
// of (cost, flat) in lexicographic order does not depend on the reduction order, so the
// choice is the reference's strict first minimum.
constexpr int kArgChunk = 4096;

__global__ void k_arg_chunk_counts(const Nodes N, const int* active, int k, int* counts,
                                   unsigned long long* best_bits, long long* best_flat) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = active[g];
  int len = N.end[node] - N.start[node] - 1;  // candidate positions s+1 .. e-1
  counts[g] = len > kArgChunk ? (len + kArgChunk - 1) / kArgChunk : 1;
  best_bits[g] = 0x7FF0000000000000ULL;  // +inf
  best_flat[g] = 0x7FFFFFFFFFFFFFFFLL;
}

__global__ void __launch_bounds__(256) k_argmin_chunks(const Nodes N, const int* active, int k,
                                                       const int* chunk_end, const double* cost0,
                                                       const double* cost1, const double* cost2,
                                                       double* part_cost, long long* part_flat,
                                                       int* part_node, unsigned long long* best_bits) {
  int b = blockIdx.x;
  // the node whose chunk range [chunk_end[g-1], chunk_end[g]) holds block b
  int lo = 0, hi = k;
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (chunk_end[mid] <= b) lo = mid + 1;
    else hi = mid;
  }
  int g = lo;
  if (g >= k) {
    if (threadIdx.x == 0) part_node[b] = -1;
    return;
  }
  int chunk = b - (g ? chunk_end[g - 1] : 0);
  int node = active[g];
  int s = N.start[node], e = N.end[node];
  int n = e - s;
  int j0 = s + 1 + chunk * kArgChunk;
  int j1 = min(e, j0 + kArgChunk);
  Cand m{CUDART_INF, 0x7FFFFFFFFFFFFFFFLL};
  const double* costs[3] = {cost0, cost1, cost2};
  for (int a = 0; a < 3; ++a)
    for (int j = j0 + threadIdx.x; j < j1; j += blockDim.x) {
      double c = costs[a][j];
      if (c != CUDART_INF) m = better(m, Cand{c, (long long)a * n + (j - s)});
    }
  __shared__ double sc[8];
  __shared__ long long sf[8];
  for (int off = 16; off > 0; off >>= 1) {
    double oc = __shfl_down_sync(0xFFFFFFFFu, m.cost, off);
    long long of = __shfl_down_sync(0xFFFFFFFFu, m.flat, off);
    m = better(m, Cand{oc, of});
  }
  int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) {
    sc[w] = m.cost;
    sf[w] = m.flat;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    Cand r = Cand{sc[0], sf[0]};
    for (int q = 1; q < (int)(blockDim.x >> 5); ++q) r = better(r, Cand{sc[q], sf[q]});
    part_cost[b] = r.cost;
    part_flat[b] = r.flat;
    part_node[b] = g;
    // costs are non-negative: their bit patterns order like the values
    atomicMin(best_bits + g, (unsigned long long)__double_as_longlong(r.cost));
  }
}

__global__ void k_argmin_flat(int blocks_total, const double* part_cost, const long long* part_flat,
                              const int* part_node, const double* best_cost, long long* best_flat) {
  int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= blocks_total) return;
  int g = part_node[b];
  if (g < 0) return;
  if (part_cost[b] == best_cost[g]) atomicMin(best_flat + g, part_flat[b]);
}

// ---- whole subtrees of at most kSubtreeSize primitives, one warp each
//
// The recursion of BvhBuildState.build (GpuScene.java:1424-1447) below such a node runs in
// one warp, depth first, with the node's three axis orders in shared memory: per node and
// axis the suffix boxes and weights (weights summed one by one in the reference's order,
// the same additions as its loop), then the prefix pass evaluating every split's cost in the
// reference's expression order, the first minimum over (axis, position), the leaf rule in
// the node's current order, and a stable partition of the other two axis orders.  Every
// number is the one the level loop would compute for the same node; the subtree only saves
// the per-level passes over all primitives (scans, gathers, argmin blocks) that dominate
// the deep levels.
constexpr int kSubtreeSize = kSeqNodeSize;
constexpr int kSubtreeThreads = 96;  // one warp per axis
#ifndef RTB_SUBTREE_BLOCKS_PER_SM
#define RTB_SUBTREE_BLOCKS_PER_SM 9  // 22.8 KB of shared memory and <= 72 registers each
#endif

struct SubtreeSmem {
  // The subtree's primitives get local slots 0..M-1 (axis 0's order at the root); the
  // axis orders hold slots, and the primitives' boxes and weights are staged by slot, so
  // the sweeps read shared memory only.
  int gid[kSubtreeSize];        // slot -> primitive
  Box lbox[kSubtreeSize];
  double lw[kSubtreeSize];
  unsigned char lside[kSubtreeSize];
  int idx[3][kSubtreeSize];     // the subtree's three axis orders (slots)
  union {  // the sweeps' terms, then (the sweeps done) the partition's scratch
    double sterm[3][kSubtreeSize];  // per axis: suffix area x suffix weight of the current node
    int tmp[3][kSubtreeSize];       // per axis: partition scratch
  };
  int4 stack[kSubtreeSize];     // pending nodes, depth first: node, start, end,
                                // depth << 2 | (order axis + 1)
  double best_cost[3];
  long long best_flat[3];
  int sp, child;
};

__device__ __forceinline__ Box empty_box() {
  Box b;
  for (int k = 0; k < 3; ++k) {
    b.mn[k] = CUDART_INF_F;
    b.mx[k] = -CUDART_INF_F;
  }
  return b;
}

// Inclusive union over lanes 0..lane (min / max are exact in any order), for the lanes
// below `count` (warp-uniform); lanes from `count` up hold empty boxes and are not needed.
__device__ __forceinline__ Box warp_union_scan(Box b, int lane, int count) {
  for (int off = 1; off < count; off <<= 1) {
    Box o;
    for (int k = 0; k < 3; ++k) {
      o.mn[k] = __shfl_up_sync(0xFFFFFFFFu, b.mn[k], off);
      o.mx[k] = __shfl_up_sync(0xFFFFFFFFu, b.mx[k], off);
    }
    if (lane >= off) b = BoxUnion()(b, o);
  }
  return b;
}

__device__ __forceinline__ Box warp_bcast(const Box& b, int src) {
  Box r;
  for (int k = 0; k < 3; ++k) {
    r.mn[k] = __shfl_sync(0xFFFFFFFFu, b.mn[k], src);
    r.mx[k] = __shfl_sync(0xFFFFFFFFu, b.mx[k], src);
  }
  return r;
}

// Running sums of the lanes' weights in lane order, continuing `acc`: lane q gets
// acc + w_0 + ... + w_q added one by one, for the lanes below `count` (warp-uniform).  The
// chain runs in groups of four lanes, each group's shuffles issued ahead of its additions;
// lanes past the node's end carry w = 0, and adding +0 to a non-negative sum leaves it
// unchanged, so the last group may run past `count`.
__device__ __forceinline__ double warp_sequential_sum(double w, double& acc, int lane, int count) {
  double mine = 0.0;
  for (int g = 0; g < count; g += 4) {
    double v[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) v[q] = __shfl_sync(0xFFFFFFFFu, w, g + q);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      acc = acc + v[q];
      mine = g + q == lane ? acc : mine;
    }
  }
  return mine;
}

__device__ __forceinline__ bool lex_less(double c, long long f, double bc, long long bf) {
  return c < bc || (c == bc && f < bf);
}

// One block of three warps per subtree root: warp a sweeps axis a of the current node,
// the block takes the first minimum over the three axes' winners, and the warps of the two
// other axes partition their orders.  Every decision is computed identically by all threads
// (or broadcast through shared memory), so the block's barriers are uniform.
__global__ void __launch_bounds__(kSubtreeThreads, RTB_SUBTREE_BLOCKS_PER_SM) k_subtrees(
    const Prims P, IdxSet I, Nodes N, const int* roots, const int* root_count, int leaf_size,
    double traversal, int* node_counter, int* stats, int* slot_of) {
  __shared__ SubtreeSmem sm;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if ((int)blockIdx.x >= *root_count) return;
  const int root = roots[blockIdx.x];
  const int rs = N.start[root], re = N.end[root], M = re - rs;
  for (int i = threadIdx.x; i < M; i += kSubtreeThreads) {
    int p = I.a[0][rs + i];
    sm.gid[i] = p;
    sm.lbox[i] = P.box[p];
    sm.lw[i] = P.w[p];
    slot_of[p] = i;  // each primitive belongs to one subtree
    sm.idx[0][i] = i;
  }
  __syncthreads();
  for (int a = 1; a < 3; ++a)
    for (int i = threadIdx.x; i < M; i += kSubtreeThreads) sm.idx[a][i] = slot_of[I.a[a][rs + i]];
  if (threadIdx.x == 0) {
    sm.stack[0] = make_int4(root, rs, re, (N.depth[root] << 2) | (N.order_axis[root] + 1));
    sm.sp = 1;
  }
  // the subtree's statistics, kept by thread 0 and added to the build's once at the end
  // (one atomic per block instead of four per leaf on the same four words)
  int leaves = 0, min_occ = 0x7FFFFFFF, max_occ = 0, max_depth = 0;
  __syncthreads();
  while (sm.sp > 0) {
    const int4 en = sm.stack[sm.sp - 1];
    __syncthreads();
    if (threadIdx.x == 0) sm.sp--;
    const int node = en.x, s = en.y, e = en.z, m = e - s, lo = s - rs;
    const int oa = (en.w & 3) - 1, depth = en.w >> 2;
    // node bounds (every warp computes the same union): a butterfly over the lanes that hold
    // positions, then lane 0's union to all
    Box nb = empty_box();
    for (int i = lane; i < m; i += 32) nb = BoxUnion()(nb, sm.lbox[sm.idx[0][lo + i]]);
    int span = 1;
    while (span < min(m, 32)) span <<= 1;
    for (int off = 1; off < span; off <<= 1) {
      Box o;
      for (int k = 0; k < 3; ++k) {
        o.mn[k] = __shfl_xor_sync(0xFFFFFFFFu, nb.mn[k], off);
        o.mx[k] = __shfl_xor_sync(0xFFFFFFFFu, nb.mx[k], off);
      }
      nb = BoxUnion()(nb, o);
    }
    if (span < 32) nb = warp_bcast(nb, 0);
    const double node_a = surface_area(nb) * traversal;
    // this warp's axis
    double best = CUDART_INF;
    long long best_flat = 0x7FFFFFFFFFFFFFFFLL;
    const int a = warp;
    const int* ix = sm.idx[a] + lo;
    if (m > 1 && P.cen[a][sm.gid[ix[m - 1]]] - P.cen[a][sm.gid[ix[0]]] > 1.0e-12) {
      // suffix boxes and weights, from the last position down (GpuScene.java:1476-1480)
      Box carry = empty_box();
      double acc = 0.0;
      for (int base = 0; base < m; base += 32) {
        const int cnt = min(32, m - base);
        int q = m - 1 - (base + lane);
        Box b = q >= 0 ? sm.lbox[ix[q]] : empty_box();
        double w = q >= 0 ? sm.lw[ix[q]] : 0.0;
        b = BoxUnion()(warp_union_scan(b, lane, cnt), carry);
        double sw = warp_sequential_sum(w, acc, lane, cnt);
        if (q >= 0) sm.sterm[a][lo + q] = surface_area(b) * sw;
        carry = warp_bcast(b, cnt - 1);
      }
      __syncwarp();
      // prefix pass and the cost of putting local positions [0, i) left (1470-1475, 1482-1485)
      carry = empty_box();
      acc = 0.0;
      for (int base = 0; base < m; base += 32) {
        const int cnt = min(32, m - base);
        int li = base + lane;
        Box b = li < m ? sm.lbox[ix[li]] : empty_box();
        double w = li < m ? sm.lw[ix[li]] : 0.0;
        b = BoxUnion()(warp_union_scan(b, lane, cnt), carry);
        double pw = warp_sequential_sum(w, acc, lane, cnt);
        int i = li + 1;  // split after li
        if (i < m) {
          double bl = surface_area(b) * pw;
          double d = sm.sterm[a][lo + i];
          double c = (node_a + bl) + d;
          long long flat = (long long)a * m + i;
          if (lex_less(c, flat, best, best_flat)) {
            best = c;
            best_flat = flat;
          }
        }
        carry = warp_bcast(b, cnt - 1);
      }
      for (int off = 16; off > 0; off >>= 1) {
        double oc = __shfl_xor_sync(0xFFFFFFFFu, best, off);
        long long of = __shfl_xor_sync(0xFFFFFFFFu, best_flat, off);
        if (lex_less(oc, of, best, best_flat)) {
          best = oc;
          best_flat = of;
        }
      }
    }
    if (lane == 0) {
      sm.best_cost[a] = best;
      sm.best_flat[a] = best_flat;
    }
    __syncthreads();
    best = sm.best_cost[0];
    best_flat = sm.best_flat[0];
    for (int k = 1; k < 3; ++k)
      if (lex_less(sm.best_cost[k], sm.best_flat[k], best, best_flat)) {
        best = sm.best_cost[k];
        best_flat = sm.best_flat[k];
      }
    // leaf rule (GpuScene.java:1435-1441), the weight sum in the node's current order
    bool leaf = m == 1 || best == CUDART_INF;
    if (!leaf && m <= leaf_size) {
      double wsum = 0.0;
      for (int j = 0; j < m; ++j) wsum = wsum + (oa < 0 ? P.w[s + j] : sm.lw[sm.idx[oa][lo + j]]);
      if (!(best < surface_area(nb) * wsum)) leaf = true;
    }
    if (threadIdx.x == 0) {
      N.bounds[node] = nb;
      N.split_axis[node] = -1;
    }
    if (leaf) {
      if (threadIdx.x == 0) {
        N.leaf[node] = 1;
        leaves++;
        min_occ = min(min_occ, m);
        max_occ = max(max_occ, m);
        max_depth = max(max_depth, depth);
      }
      __syncthreads();
      continue;
    }
    const int axis = (int)(best_flat / m), pos = (int)(best_flat % m);
    if (threadIdx.x == 0) {
      int l = atomicAdd(node_counter, 2), r = l + 1;
      N.leaf[node] = 0;
      N.left[node] = l;
      N.right[node] = r;
      N.split_axis[node] = axis;
      N.split_pos[node] = pos;
      N.start[l] = s;
      N.end[l] = s + pos;
      N.start[r] = s + pos;
      N.end[r] = e;
      N.order_axis[l] = N.order_axis[r] = axis;
      N.depth[l] = N.depth[r] = depth + 1;
      N.leaf[l] = N.leaf[r] = 0;
      const int meta = ((depth + 1) << 2) | (axis + 1);
      sm.stack[sm.sp] = make_int4(r, s + pos, e, meta);
      sm.stack[sm.sp + 1] = make_int4(l, s, s + pos, meta);
      sm.sp += 2;
    }
    // stable partition of the other two axis orders by side
    if (warp == axis)
      for (int i = lane; i < m; i += 32) sm.lside[sm.idx[axis][lo + i]] = i >= pos ? 1 : 0;
    __syncthreads();
    if (warp != axis) {
      int* t = sm.tmp[a];
      int nl = 0;
      for (int base = 0; base < m; base += 32) {
        int li = base + lane;
        bool in = li < m;
        int p = in ? sm.idx[a][lo + li] : 0;
        bool left = in && sm.lside[p] == 0;
        unsigned bal = __ballot_sync(0xFFFFFFFFu, left);
        if (left) t[nl + __popc(bal & ((1u << lane) - 1u))] = p;
        nl += __popc(bal);
      }
      int nr = 0;
      for (int base = 0; base < m; base += 32) {
        int li = base + lane;
        bool in = li < m;
        int p = in ? sm.idx[a][lo + li] : 0;
        bool right = in && sm.lside[p] != 0;
        unsigned bal = __ballot_sync(0xFFFFFFFFu, right);
        if (right) t[pos + nr + __popc(bal & ((1u << lane) - 1u))] = p;
        nr += __popc(bal);
      }
      __syncwarp();
      for (int i = lane; i < m; i += 32) sm.idx[a][lo + i] = t[i];
    }
    __syncthreads();
  }
  for (int a = 0; a < 3; ++a)
    for (int i = threadIdx.x; i < M; i += kSubtreeThreads) I.a[a][rs + i] = sm.gid[sm.idx[a][i]];
  if (threadIdx.x == 0 && leaves > 0) {
    atomicAdd(stats + 0, leaves);
    atomicMin(stats + 1, min_occ);
    atomicMax(stats + 2, max_occ);
    atomicMax(stats + 3, max_depth);
  }
}

// Nodes per depth, then all nodes listed level by level (the finishing passes walk them;
// the order inside a level is free, every node of a level being independent of the
// others).  Both passes count in shared memory first, a warp's lanes of equal depth
// together, so that each block adds once per depth to the few global counters instead of
// once per node; depths from kDepthShared up go to the global counters directly.
constexpr int kDepthShared = 256;

__global__ void __launch_bounds__(256) k_depth_hist(const Nodes N, int count, int* hist) {
  __shared__ int sh[kDepthShared];
  for (int i = threadIdx.x; i < kDepthShared; i += blockDim.x) sh[i] = 0;
  __syncthreads();
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = node < count ? N.depth[node] : -1;
  const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
  if (d >= 0 && (threadIdx.x & 31) == __ffs(peers) - 1) {
    if (d < kDepthShared) atomicAdd(sh + d, __popc(peers));
    else atomicAdd(hist + d, __popc(peers));
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kDepthShared; i += blockDim.x)
    if (sh[i]) atomicAdd(hist + i, sh[i]);
}

__global__ void __launch_bounds__(256) k_depth_scatter(const Nodes N, int count, int* cursor,
                                                       int* all_nodes) {
  __shared__ int cnt[kDepthShared], base[kDepthShared];
  for (int i = threadIdx.x; i < kDepthShared; i += blockDim.x) cnt[i] = 0;
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int node = blockIdx.x * blockDim.x + threadIdx.x;
  const int d = node < count ? N.depth[node] : -1;
  const unsigned peers = __match_any_sync(0xFFFFFFFFu, d);
  const int leader = __ffs(peers) - 1;
  int local = -1;  // rank among the block's nodes of depth d
  if (d >= 0 && d < kDepthShared) {
    int first = 0;
    if (lane == leader) first = atomicAdd(cnt + d, __popc(peers));
    local = first;
  }
  local = __shfl_sync(0xFFFFFFFFu, local, leader) + __popc(peers & ((1u << lane) - 1u));
  __syncthreads();
  for (int i = threadIdx.x; i < kDepthShared; i += blockDim.x)
    if (cnt[i]) base[i] = atomicAdd(cursor + i, cnt[i]);
  __syncthreads();
  if (d >= kDepthShared) all_nodes[atomicAdd(cursor + d, 1)] = node;
  else if (d >= 0) all_nodes[base[d] + local] = node;
}

// Leaf-or-split decision per active node (GpuScene.java:1424-1447).
__global__ void k_decide(const Prims P, IdxSet I, Nodes N, const int* active, int k,
                         const double* best_cost, const long long* best_flat, const Box* node_box,
                         int leaf_size, int* node_counter, int* next_active, int* next_count,
                         int* level_of, int level, int* stats, int* largest_child, int* small_roots,
                         int* small_count) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = active[g];
  int s = N.start[node], e = N.end[node];
  int n = e - s;
  Box bounds = node_box[e - 1];
  N.bounds[node] = bounds;
  N.split_axis[node] = -1;
  bool leaf = n == 1 || best_cost[g] == CUDART_INF;
  if (!leaf && n <= leaf_size) {
    double wsum = 0.0;
    for (int j = s; j < e; ++j) wsum = wsum + P.w[current_prim(I.a, N.order_axis[node], j)];
    double leaf_cost = surface_area(bounds) * wsum;
    if (!(best_cost[g] < leaf_cost)) leaf = true;
  }
  if (leaf) {
    N.leaf[node] = 1;
    atomicAdd(stats + 0, 1);                 // leaves
    atomicMin(stats + 1, n);                 // min occupancy
    atomicMax(stats + 2, n);                 // max occupancy
    atomicMax(stats + 3, N.depth[node]);     // max depth
    return;
  }
  long long flat = best_flat[g];
  int axis = (int)(flat / n);
  int pos = (int)(flat % n);
  int c = atomicAdd(node_counter, 2);
  int l = c, r = c + 1;
  N.leaf[node] = 0;
  N.left[node] = l;
  N.right[node] = r;
  N.split_axis[node] = axis;
  N.split_pos[node] = pos;
  N.start[l] = s;
  N.end[l] = s + pos;
  N.start[r] = s + pos;
  N.end[r] = e;
  N.order_axis[l] = N.order_axis[r] = axis;
  N.depth[l] = N.depth[r] = N.depth[node] + 1;
  N.leaf[l] = N.leaf[r] = 0;
  atomicMax(stats + 3, N.depth[node] + 1);
  // children of at most kSubtreeSize primitives leave the level loop: k_subtrees builds
  // their whole subtrees later (level_of -1 keeps the level kernels off their positions)
  int sizes[2] = {pos, n - pos}, kids[2] = {l, r};
  for (int h = 0; h < 2; ++h) {
    if (sizes[h] <= kSubtreeSize) {
      level_of[kids[h]] = -1;
      small_roots[atomicAdd(small_count, 1)] = kids[h];
    } else {
      level_of[kids[h]] = level + 1;
      next_active[atomicAdd(next_count, 1)] = kids[h];
      atomicMax(largest_child, sizes[h]);
    }
  }
}

// Stable partition of the three axis orders of every node split at this level, one axis
// per blockIdx.y: left flags, one exclusive sum over all 3n flags (a node's left rank is a
// difference inside its own axis range, so the other axes' counts cancel), then the scatter.
__global__ void k_left_flags3(IdxSet I, const Nodes N, const int* key, const int* level_of, int level,
                              int n, const unsigned char* side, int* flags) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int a = blockIdx.y;
  const int node = key[j];
  const bool split = level_of[node] == level && N.split_axis[node] >= 0;
  flags[(size_t)a * n + j] = split ? (side[I.a[a][j]] == 0) : 0;
}

__global__ void k_scatter3(IdxSet I, IdxSet T, const Nodes N, const int* key, const int* level_of,
                           int level, int n, const unsigned char* side, const int* lscan) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  const int a = blockIdx.y;
  const int node = key[j];
  const int p = I.a[a][j];
  int* out = T.a[a];
  if (!(level_of[node] == level && N.split_axis[node] >= 0)) {
    out[j] = p;
    return;
  }
  const int* ls = lscan + (size_t)a * n;
  const int s = N.start[node];
  const int lrank = ls[j] - ls[s];
  out[side[p] == 0 ? s + lrank : s + N.split_pos[node] + ((j - s) - lrank)] = p;
}

__global__ void k_sides(IdxSet I, const Nodes N, const int* key, const int* level_of, int level, int n,
                        unsigned char* side) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= n) return;
  int node = key[j];
  if (level_of[node] != level) return;
  int axis = N.split_axis[node];
  if (axis < 0) return;
  int p = I.a[axis][j];
  side[p] = (j - N.start[node]) >= N.split_pos[node] ? 1 : 0;
}



// ---- BvhRotator (GpuScene.java:968-1057) on the device
//
// A pass visits the tree bottom-up; at each interior node it compares the current node
// with the four rotations that swap a grandchild with the uncle, by areaCost (surface area
// times c_T per interior node plus surface area times the leaf's sequential weight sum per
// leaf), and keeps the first one cheaper by more than 1e-12.  The decision at a node only
// reads its own subtree, which the deeper levels have already settled, so each level runs
// in parallel.  The reference recomputes areaCost recursively for every candidate; here each
// node keeps its settled subtree's cost, and a candidate's cost adds the same terms in the
// same order ((A_node c_T + cost(left)) + cost(right)), so every comparison is the
// reference's to the bit.  A rotation reuses the child slot it restructures.

// Breadth-first levels of the current tree: children of the frontier.
__global__ void k_next_level(const Nodes N, const int* frontier, int k, int* next, int* next_count) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = frontier[g];
  if (N.leaf[node]) return;
  int q = atomicAdd(next_count, 2);
  next[q] = N.left[node];
  next[q + 1] = N.right[node];
}

__global__ void k_leaf_area_cost(const Prims P, IdxSet I, const Nodes N, const int* nodes, int k,
                                 double* rcost) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int node = nodes[g];
  if (!N.leaf[node]) return;
  double w = 0.0;
  for (int j = N.start[node]; j < N.end[node]; ++j) w = w + P.w[current_prim(I.a, N.order_axis[node], j)];
  rcost[node] = surface_area(N.bounds[node]) * w;
}

__device__ __forceinline__ Box box_union(const Box& a, const Box& b) { return BoxUnion()(a, b); }

__global__ void k_rotate_level(Nodes N, const int* nodes, int k, double traversal, double* rcost,
                               int* rotations) {
  int g = blockIdx.x * blockDim.x + threadIdx.x;
  if (g >= k) return;
  int n = nodes[g];
  if (N.leaf[n]) return;
  const double eps = 1.0e-12;
  int L = N.left[n], R = N.right[n];
  double top = surface_area(N.bounds[n]) * traversal;
  double x = top + rcost[L];
  double best = x + rcost[R];
  int choice = 0;
  double inner_best = 0.0;
  if (!N.leaf[L]) {
    int a = N.left[L], b = N.right[L], c = R;
    // join(a, join(b, c))
    double in1 = surface_area(box_union(N.bounds[b], N.bounds[c])) * traversal;
    in1 = in1 + rcost[b];
    in1 = in1 + rcost[c];
    double c1 = top + rcost[a];
    c1 = c1 + in1;
    if (c1 < best - eps) {
      best = c1;
      choice = 1;
      inner_best = in1;
    }
    // join(b, join(a, c))
    double in2 = surface_area(box_union(N.bounds[a], N.bounds[c])) * traversal;
    in2 = in2 + rcost[a];
    in2 = in2 + rcost[c];
    double c2 = top + rcost[b];
    c2 = c2 + in2;
    if (c2 < best - eps) {
      best = c2;
      choice = 2;
      inner_best = in2;
    }
  }
  if (!N.leaf[R]) {
    int a = L, b = N.left[R], c = N.right[R];
    // join(join(a, c), b)
    double in3 = surface_area(box_union(N.bounds[a], N.bounds[c])) * traversal;
    in3 = in3 + rcost[a];
    in3 = in3 + rcost[c];
    double c3 = top + in3;
    c3 = c3 + rcost[b];
    if (c3 < best - eps) {
      best = c3;
      choice = 3;
      inner_best = in3;
    }
    // join(join(a, b), c)
    double in4 = surface_area(box_union(N.bounds[a], N.bounds[b])) * traversal;
    in4 = in4 + rcost[a];
    in4 = in4 + rcost[b];
    double c4 = top + in4;
    c4 = c4 + rcost[c];
    if (c4 < best - eps) {
      best = c4;
      choice = 4;
      inner_best = in4;
    }
  }
  if (choice == 1 || choice == 2) {
    int a = N.left[L], b = N.right[L], c = R;
    int outer = choice == 1 ? a : b, p = choice == 1 ? b : a;
    N.left[n] = outer;
    N.right[n] = L;
    N.left[L] = p;
    N.right[L] = c;
    N.bounds[L] = box_union(N.bounds[p], N.bounds[c]);
    rcost[L] = inner_best;
  } else if (choice == 3 || choice == 4) {
    int a = L, b = N.left[R], c = N.right[R];
    int q = choice == 3 ? c : b, outer = choice == 3 ? b : c;
    N.left[n] = R;
    N.right[n] = outer;
    N.left[R] = a;
    N.right[R] = q;
    N.bounds[R] = box_union(N.bounds[a], N.bounds[q]);
    rcost[R] = inner_best;
  }
  rcost[n] = best;
  if (choice) atomicAdd(rotations, 1);
}

// Breadth-first levels of the tree under `roots`: nodes level by level in `all_nodes`,
// level starts in level_begin.  Returns false on a CUDA error.
bool tree_levels(const Nodes& N, int roots, int* all_nodes, int* counter, std::vector<int>& level_begin,
                 cudaStream_t sm) {
  std::vector<int> h(roots);
  for (int r = 0; r < roots; ++r) h[r] = r;
  cudaMemcpyAsync(all_nodes, h.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  level_begin.assign(1, 0);
  int begin = 0, k = roots;
  while (k > 0) {
    level_begin.push_back(begin + k);
    cudaMemsetAsync(counter, 0, 4, sm);
    k_next_level<<<blocks(k), 256, 0, sm>>>(N, all_nodes + begin, k, all_nodes + begin + k, counter);
    int next = 0;
    cudaMemcpyAsync(&next, counter, 4, cudaMemcpyDeviceToHost, sm);
    if (cudaStreamSynchronize(sm) != cudaSuccess) return false;
    begin += k;
    k = next;
  }
  return true;
}

}  // namespace

rtb_status build_bvh(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                     rtb_scene** out, rtb_bvh_stats* stats) {
  return build_bvh_options(ctx, desc, cfg, nullptr, out, stats);
}

rtb_status build_bvh_options(rtb_context* ctx, const rtb_scene_desc* desc, const rtb_build_config* cfg,
                             const rtb_build_options* options, rtb_scene** out, rtb_bvh_stats* stats) {
  if (!out) return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "null argument");
  if (cfg && (cfg->mode == 4 || cfg->mode == 5)) return build_bvh_sbvh(ctx, desc, cfg, options, out, stats);
  BuildCfg c;
  bool per_type = false;
  rtb_status st = build_setup(ctx, desc, cfg, c, per_type, true);
  if (st != RTB_OK) return st;
  int rotation_passes = options ? options->rotation_passes : 4;  // BvhBuildOptions.defaults
  bool rotate = cfg->mode == 6 || cfg->mode == 7;
  if (rotate && rotation_passes < 1)
    return fail(ctx, RTB_ERR_INVALID_ARGUMENT, "rotationPasses must be positive.");
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
  IdxSet I, T;
  for (int k = 0; k < 3; ++k) {
    I.a[k] = W.alloc<int>(n);
    T.a[k] = W.alloc<int>(n);
  }
  int cap = 2 * n + 8;
  Nodes N = alloc_nodes(W, cap);
  int* level_of = W.alloc<int>(cap);
  int* key = W.alloc<int>(n);
  Box* node_box = W.alloc<Box>(n);  // a node's bounds at its last position
  const int nc = (n + kSegChunk - 1) / kSegChunk;
  Seg<Box>* box_fwd = W.alloc<Seg<Box>>(3 * (size_t)nc);
  Seg<Box>* box_bwd = W.alloc<Seg<Box>>(3 * (size_t)nc);
  Seg<TypeCounts>* cnt_fwd = c.weighted ? W.alloc<Seg<TypeCounts>>(3 * (size_t)nc) : nullptr;
  Seg<TypeCounts>* cnt_bwd = c.weighted ? W.alloc<Seg<TypeCounts>>(3 * (size_t)nc) : nullptr;
  WeightChains chains;
  for (int a = 0; a < 3; ++a) {
    chains.w[a] = W.alloc<double>(n);
    chains.pw[a] = W.alloc<double>(n);
    chains.sw[a] = c.weighted || a == 0 ? W.alloc<double>(n) : chains.sw[0];
    if (!c.weighted && a > 0) chains.pw[a] = chains.pw[0];
  }
  double* cost[3];
  double* bound[3];
  for (int a = 0; a < 3; ++a) {
    cost[a] = W.alloc<double>(n);
    bound[a] = c.weighted ? W.alloc<double>(n) : nullptr;
  }
  int* g_of_node = W.alloc<int>(cap);
  int* failed = W.alloc<int>(cap);
  int* failed_list = W.alloc<int>(cap);
  double* best_bound = W.alloc<double>(cap);
  int* lists = W.alloc<int>(2);  // small count, failed count
  int* sub_roots = W.alloc<int>(cap);  // nodes whose subtrees k_subtrees builds
  int* depth_hist = W.alloc<int>(cap + 1);
  unsigned char* side = W.alloc<unsigned char>(n);
  int* flags = W.alloc<int>(3 * (size_t)n);  // left flags of the three axis orders
  int* lscan = W.alloc<int>(3 * (size_t)n);
  unsigned long long* skeys = W.alloc<unsigned long long>(n);
  unsigned long long* skeys2 = W.alloc<unsigned long long>(n);
  int* svals = W.alloc<int>(n);
  int* tkeys = W.alloc<int>(n);
  int* tkeys2 = W.alloc<int>(n);
  int* active = W.alloc<int>(cap);
  int* next_active = W.alloc<int>(cap);
  int* all_nodes = W.alloc<int>(cap);
  double* best_cost = W.alloc<double>(cap);
  long long* best_flat = W.alloc<long long>(cap);
  int* arg_counts = W.alloc<int>(cap);
  int* arg_ends = W.alloc<int>(cap);
  long long max_arg_blocks = n / kArgChunk + cap;
  double* part_cost = W.alloc<double>(max_arg_blocks);
  long long* part_flat = W.alloc<long long>(max_arg_blocks);
  int* part_node = W.alloc<int>(max_arg_blocks);
  int* counters = W.alloc<int>(8);  // node counter, next count, stats[4]
  int* root_start = W.alloc<int>(4);
  int* root_end = W.alloc<int>(4);
  size_t tmp_bytes = 0, b1 = 0, b3 = 0, b4 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b1, skeys, skeys2, svals, svals, n);
  cub::DeviceScan::ExclusiveSum(nullptr, b3, flags, lscan, std::max(3 * n, cap));
  cub::DeviceRadixSort::SortPairs(nullptr, b4, tkeys, tkeys2, svals, svals, n, 0, 2);
  tmp_bytes = std::max(b1, std::max(b3, b4));
  void* tmp = W.alloc<char>(tmp_bytes);
  if (!W.ok) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "BVH build workspace");

  cudaEventRecord(ctx->ev0, sm);
  upload_prims(desc, c, in, P, sm);

  // ---- axis orders: (centroid, order), then (type, centroid, order) for per-type forests
  for (int a = 0; a < 3; ++a) {
    k_keys<<<blocks(n), 256, 0, sm>>>(P, a, n, skeys, svals);
    size_t tb = tmp_bytes;
    cub::DeviceRadixSort::SortPairs(tmp, tb, skeys, skeys2, svals, I.a[a], n, 0, 64, sm);
    if (per_type) {
      k_type_keys<<<blocks(n), 256, 0, sm>>>(P, I.a[a], n, tkeys);
      tb = tmp_bytes;
      cub::DeviceRadixSort::SortPairs(tmp, tb, tkeys, tkeys2, I.a[a], T.a[a], n, 0, 2, sm);
      cudaMemcpyAsync(I.a[a], T.a[a], (size_t)n * 4, cudaMemcpyDeviceToDevice, sm);
    }
  }

  // ---- roots
  int h_rs[4], h_re[4];
  int roots = root_ranges(c, per_type, h_rs, h_re);
  int h_counters[8] = {roots, 0, 0, 0x7FFFFFFF, 0, 0, 0, 0};
  cudaMemcpyAsync(root_start, h_rs, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(root_end, h_re, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(N.start, h_rs, roots * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(N.end, h_re, roots * 4, cudaMemcpyHostToDevice, sm);
  // roots of at most kSubtreeSize primitives go straight to the subtree kernel
  std::vector<int> h_big, h_small, h_level(roots);
  for (int r = 0; r < roots; ++r) {
    bool small = h_re[r] - h_rs[r] <= kSubtreeSize;
    (small ? h_small : h_big).push_back(r);
    h_level[r] = small ? -1 : 0;
  }
  h_counters[7] = (int)h_small.size();
  if (!h_big.empty())
    cudaMemcpyAsync(active, h_big.data(), h_big.size() * 4, cudaMemcpyHostToDevice, sm);
  if (!h_small.empty())
    cudaMemcpyAsync(sub_roots, h_small.data(), h_small.size() * 4, cudaMemcpyHostToDevice, sm);
  cudaMemcpyAsync(counters, h_counters, sizeof(h_counters), cudaMemcpyHostToDevice, sm);
  cudaMemsetAsync(N.order_axis, 0xFF, (size_t)roots * 4, sm);  // -1: input order
  cudaMemsetAsync(N.depth, 0, (size_t)roots * 4, sm);
  cudaMemcpyAsync(level_of, h_level.data(), roots * 4, cudaMemcpyHostToDevice, sm);
  k_init_keys<<<blocks(n), 256, 0, sm>>>(key, root_start, root_end, roots, n);

  // ---- level loop
  TypeWeights tw;
  for (int t = 0; t < 4; ++t) tw.w[t] = c.weighted ? 1.0 + c.lambda * (c.measured[t] - 1.0) : 1.0;
  int sequential_nodes = 0;
  std::vector<int> level_begin = {0};
  int k = (int)h_big.size(), level = 0, total_nodes = roots;
  const dim3 seg_grid(nc, 3), carry_grid(3, 2);
  // split costs of every position on all three axes (and the level's node bounds)
  auto costs = [&](int certified) {
    BoxLoad L;
    L.P = P;
    L.I = I;
    L.level_of = level_of;
    L.level = level;
    SplitCosts U{P, I, N, {chains.pw[0], chains.pw[1], chains.pw[2]},
                 {chains.sw[0], chains.sw[1], chains.sw[2]}, c.traversal, certified,
                 {cost[0], cost[1], cost[2]}, {bound[0], bound[1], bound[2]}, node_box};
    k_seg_chunks<<<seg_grid, kSegThreads, 0, sm>>>(L, key, n, nc, box_fwd, box_bwd);
    k_seg_carries<BoxOp><<<carry_grid, kCarryThreads, 0, sm>>>(nc, box_fwd, box_bwd);
    k_seg_apply<<<seg_grid, kSegThreads, 0, sm>>>(L, U, key, n, nc, box_fwd, box_bwd);
  };
  auto argmin = [&]() {
    k_arg_chunk_counts<<<blocks(k), 256, 0, sm>>>(N, active, k, arg_counts,
                                                  (unsigned long long*)best_cost, best_flat);
    size_t tb = tmp_bytes;
    cub::DeviceScan::InclusiveSum(tmp, tb, arg_counts, arg_ends, k, sm);
    // chunks <= (positions / kArgChunk) + one per node; surplus blocks find no node
    long long nb = (long long)n / kArgChunk + k + 1;
    k_argmin_chunks<<<(unsigned)nb, 256, 0, sm>>>(N, active, k, arg_ends, cost[0], cost[1], cost[2],
                                                  part_cost, part_flat, part_node,
                                                  (unsigned long long*)best_cost);
    k_argmin_flat<<<blocks(nb), 256, 0, sm>>>((int)nb, part_cost, part_flat, part_node, best_cost,
                                              best_flat);
  };
  while (k > 0) {
    // Every node of the level loop holds more than kSubtreeSize >= kSeqNodeSize primitives
    // (smaller ones go to k_subtrees), so with non-unit weights all of them take the
    // certified count-based weights; only those whose certificate fails are summed
    // sequentially, below.
    static_assert(kSubtreeSize >= kSeqNodeSize, "level-loop nodes must all be certifiable");
    const bool certify = c.weighted;
    if (c.weighted) {
      cudaMemsetAsync(lists, 0, 2 * sizeof(int), sm);
      k_node_slots<<<blocks(k), 256, 0, sm>>>(active, k, g_of_node);
      {
        CountLoad L;
        L.P = P;
        L.I = I;
        L.N = N;
        L.level_of = level_of;
        L.level = level;
        CountWeights U{tw, {chains.pw[0], chains.pw[1], chains.pw[2]},
                       {chains.sw[0], chains.sw[1], chains.sw[2]}};
        k_seg_chunks<<<seg_grid, kSegThreads, 0, sm>>>(L, key, n, nc, cnt_fwd, cnt_bwd);
        k_seg_carries<CountOp><<<carry_grid, kCarryThreads, 0, sm>>>(nc, cnt_fwd, cnt_bwd);
        k_seg_apply<<<seg_grid, kSegThreads, 0, sm>>>(L, U, key, n, nc, cnt_fwd, cnt_bwd);
      }
    } else {
      k_weights_unit<<<blocks(n), 256, 0, sm>>>(N, key, level_of, level, n, chains.pw[0], chains.sw[0]);
    }
    costs(certify ? 1 : 0);
    argmin();
    if (certify) {
      // large nodes whose winner is not clear of the others' bounds: sequential weights,
      // their costs again, and the argmin again (unchanged for every other node)
      k_best_bound<<<blocks(k), 256, 0, sm>>>(N, active, k, best_cost, best_flat, bound[0], bound[1],
                                              bound[2], best_bound, failed);
      k_certify<<<dim3(blocks(n), 3), 256, 0, sm>>>(N, key, level_of, level, n, g_of_node, cost[0],
                                                    cost[1], cost[2], bound[0], bound[1], bound[2],
                                                    best_cost, best_flat, best_bound, failed);
      k_failed_list<<<blocks(k), 256, 0, sm>>>(active, k, failed, failed_list, lists + 1);
      int nfail = 0;
      cudaMemcpyAsync(&nfail, lists + 1, 4, cudaMemcpyDeviceToHost, sm);
      cudaError_t e = cudaStreamSynchronize(sm);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH build level");
      if (nfail > 0) {
        for (int a = 0; a < 3; ++a)
          k_gather_weights<<<blocks(n), 256, 0, sm>>>(P, I.a[a], n, const_cast<double*>(chains.w[a]));
        k_weights_seq<<<blocks(6LL * 32 * nfail, 128), 128, 0, sm>>>(chains, N, failed_list, nfail,
                                                                     nullptr);
        costs(0);
        argmin();
        sequential_nodes += nfail;
      }
    }
    cudaMemsetAsync(counters + 1, 0, 4, sm);
    cudaMemsetAsync(counters + 6, 0, 4, sm);
    k_decide<<<blocks(k), 256, 0, sm>>>(P, I, N, active, k, best_cost, best_flat, node_box, c.leaf_size,
                                        counters, next_active, counters + 1, level_of, level,
                                        counters + 2, counters + 6, sub_roots, counters + 7);
    k_sides<<<blocks(n), 256, 0, sm>>>(I, N, key, level_of, level, n, side);
    {
      const dim3 axes_grid(blocks(n), 3);
      k_left_flags3<<<axes_grid, 256, 0, sm>>>(I, N, key, level_of, level, n, side, flags);
      size_t tb = tmp_bytes;
      cub::DeviceScan::ExclusiveSum(tmp, tb, flags, lscan, 3 * n, sm);
      k_scatter3<<<axes_grid, 256, 0, sm>>>(I, T, N, key, level_of, level, n, side, lscan);
      for (int a = 0; a < 3; ++a) std::swap(I.a[a], T.a[a]);
    }
    k_update_keys<<<blocks(n), 256, 0, sm>>>(N, level_of, level, n, key);
    int next_info[6] = {0, 0, 0, 0, 0, 0};  // counters[1..6]: next count, ..., largest child
    cudaMemcpyAsync(next_info, counters + 1, sizeof(next_info), cudaMemcpyDeviceToHost, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH build level");
    int next = next_info[0];
    if (next > 0) std::swap(active, next_active);
    k = next;
    level++;
  }
  // ---- the subtrees below the level loop, then every node listed by depth
  {
    int h[8];
    cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, sm);
    cudaError_t e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH build levels");
    if (h[7] > 0)
      k_subtrees<<<(unsigned)h[7], kSubtreeThreads, 0, sm>>>(
          P, I, N, sub_roots, counters + 7, c.leaf_size, c.traversal, counters, counters + 2, flags);
    cudaMemcpyAsync(h, counters, sizeof(h), cudaMemcpyDeviceToHost, sm);
    e = cudaStreamSynchronize(sm);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH subtrees");
    total_nodes = h[0];
    int depths = h[5] + 1;
    if (total_nodes < 1 || total_nodes > cap || depths < 1 || depths > cap)
      return fail(ctx, RTB_ERR_DEVICE_CHECK, "BVH node count out of range");
    cudaMemsetAsync(depth_hist, 0, (size_t)depths * 4, sm);
    k_depth_hist<<<blocks(total_nodes), 256, 0, sm>>>(N, total_nodes, depth_hist);
    std::vector<int> hist(depths);
    cudaMemcpyAsync(hist.data(), depth_hist, (size_t)depths * 4, cudaMemcpyDeviceToHost, sm);
    e = cudaStreamSynchronize(sm);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH depth histogram");
    level_begin.assign(1, 0);
    for (int d = 0; d < depths; ++d) level_begin.push_back(level_begin.back() + hist[d]);
    cudaMemcpyAsync(depth_hist, level_begin.data(), (size_t)depths * 4, cudaMemcpyHostToDevice, sm);
    k_depth_scatter<<<blocks(total_nodes), 256, 0, sm>>>(N, total_nodes, depth_hist, all_nodes);
  }
  int rotation_count = 0;
  if (rotate) {
    double* rcost = W.alloc<double>(cap);
    int* rot = W.alloc<int>(2);
    if (!W.ok) return fail(ctx, RTB_ERR_OUT_OF_MEMORY, "BVH rotation workspace");
    bool leaves_done = false;
    for (int pass = 0; pass < rotation_passes; ++pass) {
      if (!tree_levels(N, roots, all_nodes, rot + 1, level_begin, sm))
        return cuda_fail(ctx, cudaGetLastError(), "BVH levels");
      int levels = (int)level_begin.size() - 1;
      if (!leaves_done) {
        k_leaf_area_cost<<<blocks(total_nodes), 256, 0, sm>>>(P, I, N, all_nodes, total_nodes, rcost);
        leaves_done = true;
      }
      cudaMemsetAsync(rot, 0, 4, sm);
      for (int L = levels - 1; L >= 0; --L) {
        int b = level_begin[L], cnt = level_begin[L + 1] - b;
        k_rotate_level<<<blocks(cnt), 256, 0, sm>>>(N, all_nodes + b, cnt, c.traversal, rcost, rot);
      }
      int h_rot = 0;
      cudaMemcpyAsync(&h_rot, rot, 4, cudaMemcpyDeviceToHost, sm);
      cudaError_t e = cudaStreamSynchronize(sm);
      if (e != cudaSuccess) return cuda_fail(ctx, e, "BVH rotation pass");
      rotation_count += h_rot;
      if (h_rot == 0) break;
    }
    if (!tree_levels(N, roots, all_nodes, rot + 1, level_begin, sm))
      return cuda_fail(ctx, cudaGetLastError(), "BVH levels");
    // the rotated tree's depth replaces the build's
    int depth = (int)level_begin.size() - 2;
    cudaMemcpyAsync(counters + 5, &depth, 4, cudaMemcpyHostToDevice, sm);
    cudaStreamSynchronize(sm);
  }
  rtb_status fs = finish_build(ctx, desc, cfg, W, c, P, I, N, all_nodes, level_begin, roots, total_nodes,
                               counters, out, stats);
  if (fs == RTB_OK && stats) {
    stats->rotation_count = rotation_count;
    stats->sequential_nodes = sequential_nodes;
  }
  return fs;
}

}  // namespace rtb
