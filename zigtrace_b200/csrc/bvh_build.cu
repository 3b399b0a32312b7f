/*
 * bvh_build.cu -- Bvh.build (src/bvh.zig:41-262) on the device.
 *
 * The result is the reference's tree node for node: the same binned-SAH
 * splits (12 bins, leaf size 4, depth 64), the same permutation of the
 * primitive indices and the same node numbering.  Only the schedule is the
 * device's own:
 *
 *   large nodes (more than 32 primitives), level by level: per-node bounds
 *     and bins reduced with 64-bit atomics on an order-preserving integer
 *     image of the f64 values (min/max are exact in any order); one thread
 *     per node runs the reference's bin sweep and split choice; the
 *     in-place partition (bvh.zig:175-182, a Lomuto partition) is
 *     reproduced in parallel from a prefix count of the elements that go
 *     left (see lomuto note below);
 *   small subtrees (at most 32 primitives): one warp builds the whole
 *     subtree depth first, one primitive per lane, with ballots for the
 *     partition and shared memory for the bins;
 *   numbering: Builder.makeChildren appends a node pair each time a node is
 *     split, in depth-first order, so an internal node whose split is the
 *     g-th (0-based, preorder) has its children at 2g+1 and 2g+2.  Counting
 *     the internal nodes of every subtree bottom-up and assigning preorder
 *     ranks top-down gives every node its reference index.
 *
 * Lomuto note.  With s_j the range before partitioning, L(j) "goes left",
 * rank(j) the number of L elements before j and mid the number of L
 * elements, the loop `if L(j) { swap(range[mid], range[j]); mid += 1 }`
 * leaves: positions q < mid: the L element of rank q; positions q >= mid:
 * s_q when s_q is not L, else G(rank(q)), where G(k) = s_k if s_k is not L,
 * else G(rank(k)).  (An L element at q swaps with the front of the block of
 * non-L elements, which sits at position rank(q); that slot holds s_k when
 * it was never written, or else what an earlier L element placed there.)
 * G is resolved by pointer jumping.
 *
 * Nodes that need splitMedian (more than 4 primitives and no bin split:
 * all centroids coincide or the bounds have no area) and boxes with
 * non-finite coordinates are left to the host builder: the build reports
 * ZT_DEVICE_BUILD_FALLBACK and the caller runs the host build instead, as it
 * does when no CUDA device or too little device memory is available.
 * Bounds agree with the host build up to the sign of zero (min and max of
 * +0 and -0 may return either); nothing downstream distinguishes the two.
 */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "scene_host.h"

namespace zt {

namespace {

constexpr int kBins = 12;              /* bvh.zig:16 bin_count */
constexpr uint32_t kLeafSize = 4;      /* bvh.zig: max_leaf_size */
constexpr uint32_t kMaxLevel = 64;     /* bvh.zig: max_depth */
constexpr double kTravCost = 1.0;      /* bvh.zig: traversal_cost */
constexpr uint32_t kSmall = 32;        /* subtrees at most this large are built by one warp */
constexpr int kAcc = 12 + 3 * kBins * 7; /* per-node accumulators: bounds, cbounds, bins */

typedef unsigned long long u64;

/* Order-preserving map of non-NaN doubles to u64 (-0 sorts below +0). */
__device__ __forceinline__ u64 ord(double d) {
  const u64 u = (u64)__double_as_longlong(d);
  return (u & 0x8000000000000000ull) ? ~u : (u | 0x8000000000000000ull);
}
__device__ __forceinline__ double unord(u64 u) {
  return __longlong_as_double((long long)((u & 0x8000000000000000ull) ? (u & ~0x8000000000000000ull) : ~u));
}
#define ORD_POS_INF 0xFFF0000000000000ull /* ord(+inf) */
#define ORD_NEG_INF 0x000FFFFFFFFFFFFFull /* ord(-inf) */

struct DBox { double mn[3], mx[3]; };

__device__ __forceinline__ DBox dbox_empty() {
  DBox b;
  for (int k = 0; k < 3; ++k) { b.mn[k] = INFINITY; b.mx[k] = -INFINITY; }
  return b;
}
__device__ __forceinline__ void dbox_merge(DBox& a, const DBox& b) { /* aabb.zig:21-23 */
  for (int k = 0; k < 3; ++k) { a.mn[k] = fmin(a.mn[k], b.mn[k]); a.mx[k] = fmax(a.mx[k], b.mx[k]); }
}
__device__ __forceinline__ double dbox_area(const DBox& a) { /* aabb.zig:53-57 */
  if (a.mn[0] > a.mx[0] || a.mn[1] > a.mx[1] || a.mn[2] > a.mx[2]) return 0;
  const double ex = a.mx[0] - a.mn[0], ey = a.mx[1] - a.mn[1], ez = a.mx[2] - a.mn[2];
  return 2.0 * (ex * ey + ey * ez + ez * ex);
}
__device__ __forceinline__ uint32_t bin_of(double c, double lo, double extent) { /* bvh.zig:258-262 */
  const double f = (c - lo) / extent * (double)kBins;
  return (uint32_t)fmax(0.0, fmin(f, (double)(kBins - 1)));
}

struct Split { int axis; uint32_t bin; double cost; bool valid; };

/* Builder.findSplit's sweeps (bvh.zig:211-256) for one axis, over its 12
 * bins already reduced (bb[b] boxes, bn[b] counts): the best split of the
 * axis, the first bin of the lowest cost. */
template <typename BinBox>
__device__ Split sweep_axis(const BinBox& bb, const uint32_t* bn, int axis, double parent_area) {
  Split best{0, 0, 0.0, false};
  double right_area[kBins];
  uint32_t right_n[kBins];
  DBox acc = dbox_empty();
  uint32_t acc_n = 0;
  for (int i = kBins - 1; i >= 0; --i) {
    dbox_merge(acc, bb(i));
    acc_n += bn[i];
    right_area[i] = dbox_area(acc);
    right_n[i] = acc_n;
  }
  acc = dbox_empty();
  acc_n = 0;
  for (int b = 0; b < kBins - 1; ++b) {
    dbox_merge(acc, bb(b));
    acc_n += bn[b];
    const uint32_t rn = right_n[b + 1];
    if (acc_n == 0 || rn == 0) continue;
    const double cost = kTravCost + (dbox_area(acc) * (double)acc_n + right_area[b + 1] * (double)rn) / parent_area;
    if (!best.valid || cost < best.cost) best = Split{axis, (uint32_t)b, cost, true};
  }
  return best;
}

/* The candidates of the three axes in axis order, as findSplit's single
 * loop keeps them: a later axis wins only with a strictly lower cost. */
__device__ __forceinline__ void keep_better(Split& best, const Split& c) {
  if (c.valid && (!best.valid || c.cost < best.cost)) best = c;
}

/* findSplit over all three axes (one thread). */
__device__ Split sweep(const DBox* bin_box, const uint32_t* bin_n, const bool* axis_ok, double parent_area) {
  Split best{0, 0, 0.0, false};
  if (parent_area <= 0) return best;
  for (int axis = 0; axis < 3; ++axis) {
    if (!axis_ok[axis]) continue;
    const DBox* bb = bin_box + axis * kBins;
    keep_better(best, sweep_axis([&](int b) { return bb[b]; }, bin_n + axis * kBins, axis, parent_area));
  }
  return best;
}

/* Shape.bounds (geometry.zig:54-57, 101-103; Aabb.pad, aabb.zig:30-39) and
 * the centroid; false for a non-finite coordinate. */
__global__ void k_prim_boxes(const zt_shape* __restrict__ shapes, uint32_t n, DBox* __restrict__ boxes,
                             double* __restrict__ cent, uint32_t* __restrict__ idx, int* __restrict__ bad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const zt_shape s = shapes[i];
  DBox b;
  if (s.kind == ZT_SPHERE) {
    const double r = fabs(s.p[3]);
    for (int k = 0; k < 3; ++k) { b.mn[k] = s.p[k] - r; b.mx[k] = s.p[k] + r; }
  } else {
    for (int k = 0; k < 3; ++k) {
      b.mn[k] = fmin(s.p[k], s.p[3 + k]);
      b.mx[k] = fmax(s.p[k], s.p[3 + k]);
      b.mn[k] = fmin(b.mn[k], s.p[6 + k]);
      b.mx[k] = fmax(b.mx[k], s.p[6 + k]);
    }
    const double delta = 1e-6;
    for (int k = 0; k < 3; ++k)
      if (b.mx[k] - b.mn[k] < delta) { b.mn[k] -= delta / 2; b.mx[k] += delta / 2; }
  }
  bool fin = true;
  for (int k = 0; k < 3; ++k) {
    fin = fin && isfinite(b.mn[k]) && isfinite(b.mx[k]);
    cent[3 * (size_t)i + k] = (b.mn[k] + b.mx[k]) * 0.5;
  }
  if (!fin) atomicExch(bad, 1);
  boxes[i] = b;
  idx[i] = i;
}

/* ------------------------------------------------------------------------
 * Large nodes, one level at a time.
 * ---------------------------------------------------------------------- */
struct LargeNode {
  uint32_t first, count, level;
  uint32_t leaf;        /* 1: stays a leaf (level limit) */
  int32_t child[2];     /* >= 0: large node id; < 0: -1 - subtree id */
  uint32_t axis, bin;   /* the split */
  double lo, extent;    /* centroid range on the split axis */
  uint32_t mid;         /* elements going left */
  uint32_t internal;    /* internal nodes in this subtree */
  uint32_t index, rank; /* reference node index and preorder split rank */
  DBox bounds;
};

struct Subtree {
  uint32_t first, count, level;
  uint32_t internal;    /* internal nodes of the subtree (set by the warp build) */
  uint32_t index, rank; /* reference index of its root and the rank of its first split */
};

/* Per-node accumulator block: [0..6) bounds (mn ord, mx ord), [6..12)
 * centroid bounds, then per axis and bin: count, 3 mn ord, 3 mx ord. */
__global__ void k_acc_init(u64* __restrict__ acc, uint32_t m) {
  const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= (uint64_t)m * kAcc) return;
  const int j = (int)(i % kAcc);
  u64 v;
  if (j < 12) v = (j % 6) < 3 ? ORD_POS_INF : ORD_NEG_INF;
  else {
    const int r = (j - 12) % 7;
    v = r == 0 ? 0 : (r <= 3 ? ORD_POS_INF : ORD_NEG_INF);
  }
  acc[i] = v;
}

/* node_of[p] = a for every position of active node a. */
__global__ void k_mark(const LargeNode* __restrict__ nodes, const uint32_t* __restrict__ active, uint32_t m,
                       int32_t* __restrict__ node_of) {
  const uint32_t a = blockIdx.x;
  if (a >= m) return;
  const LargeNode& nd = nodes[active[a]];
  for (uint32_t p = threadIdx.x; p < nd.count; p += blockDim.x) node_of[nd.first + p] = (int32_t)a;
}

__device__ __forceinline__ void warp_min_max(u64& mn, u64& mx, unsigned mask) {
  for (int o = 16; o > 0; o >>= 1) {
    const u64 a = __shfl_xor_sync(mask, mn, o), b = __shfl_xor_sync(mask, mx, o);
    mn = a < mn ? a : mn;
    mx = b > mx ? b : mx;
  }
}

/* Bounds and centroid bounds of each active node. */
__global__ void k_bounds(const int32_t* __restrict__ node_of, const uint32_t* __restrict__ idx,
                         const DBox* __restrict__ boxes, const double* __restrict__ cent, uint32_t n,
                         u64* __restrict__ acc) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t a = p < n ? node_of[p] : -1;
  const int32_t a0 = __shfl_sync(0xffffffffu, a, 0);
  const bool uniform = __all_sync(0xffffffffu, a == a0) && a0 >= 0;
  u64 v[12];
  if (a >= 0) {
    const uint32_t e = idx[p];
    const DBox b = boxes[e];
    for (int k = 0; k < 3; ++k) {
      v[k] = ord(b.mn[k]);
      v[3 + k] = ord(b.mx[k]);
      const u64 c = ord(cent[3 * (size_t)e + k]);
      v[6 + k] = c;
      v[9 + k] = c;
    }
  } else {
    for (int k = 0; k < 3; ++k) { v[k] = v[6 + k] = ORD_POS_INF; v[3 + k] = v[9 + k] = ORD_NEG_INF; }
  }
  if (uniform) {
    for (int k = 0; k < 3; ++k) {
      warp_min_max(v[k], v[3 + k], 0xffffffffu);
      warp_min_max(v[6 + k], v[9 + k], 0xffffffffu);
    }
    if ((threadIdx.x & 31) != 0) return;
  } else if (a < 0) {
    return;
  }
  u64* A = acc + (size_t)(uniform ? a0 : a) * kAcc;
  for (int k = 0; k < 3; ++k) {
    atomicMin(A + k, v[k]);
    atomicMax(A + 3 + k, v[3 + k]);
    atomicMin(A + 6 + k, v[6 + k]);
    atomicMax(A + 9 + k, v[9 + k]);
  }
}

/* Bin counts and bin bounds of each active node, through shared memory
 * when a whole block of positions belongs to one node. */
__global__ void __launch_bounds__(256) k_bins(const int32_t* __restrict__ node_of, const uint32_t* __restrict__ idx,
                                              const DBox* __restrict__ boxes, const double* __restrict__ cent,
                                              uint32_t n, u64* __restrict__ acc) {
  __shared__ u64 sb[3 * kBins * 7];
  __shared__ int32_t s_a0;
  __shared__ int s_uniform;
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  const int32_t a = p < n ? node_of[p] : -1;
  if (threadIdx.x == 0) {
    s_a0 = a;
    s_uniform = 1;
  }
  __syncthreads();
  if (a != s_a0) s_uniform = 0;
  for (int i = threadIdx.x; i < 3 * kBins * 7; i += blockDim.x) {
    const int r = i % 7;
    sb[i] = r == 0 ? 0 : (r <= 3 ? ORD_POS_INF : ORD_NEG_INF);
  }
  __syncthreads();
  const bool uniform = s_uniform && s_a0 >= 0;
  if (a >= 0) {
    const u64* A = acc + (size_t)a * kAcc;
    const uint32_t e = idx[p];
    const DBox b = boxes[e];
    for (int axis = 0; axis < 3; ++axis) {
      const double lo = unord(A[6 + axis]), extent = unord(A[9 + axis]) - lo;
      if (!(extent > 0)) continue;
      const uint32_t bin = bin_of(cent[3 * (size_t)e + axis], lo, extent);
      u64* B = uniform ? sb + (axis * kBins + bin) * 7 : (u64*)A + 12 + (axis * kBins + bin) * 7;
      atomicAdd(B, 1ull);
      for (int k = 0; k < 3; ++k) {
        atomicMin(B + 1 + k, ord(b.mn[k]));
        atomicMax(B + 4 + k, ord(b.mx[k]));
      }
    }
  }
  if (!uniform) return;
  __syncthreads();
  u64* A = acc + (size_t)s_a0 * kAcc + 12;
  for (int i = threadIdx.x; i < 3 * kBins * 7; i += blockDim.x) {
    const int r = i % 7;
    if (r == 0) {
      if (sb[i]) atomicAdd(A + i, sb[i]);
    } else if (r <= 3) {
      if (sb[i] != ORD_POS_INF) atomicMin(A + i, sb[i]);
    } else if (sb[i] != ORD_NEG_INF) {
      atomicMax(A + i, sb[i]);
    }
  }
}

/* One thread per active node: bounds, leaf test and split choice
 * (Builder.subdivide, bvh.zig:148-185). */
__global__ void k_decide(LargeNode* __restrict__ nodes, const uint32_t* __restrict__ active, uint32_t m,
                         const u64* __restrict__ acc, int* __restrict__ fallback) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= m) return;
  LargeNode& nd = nodes[active[a]];
  const u64* A = acc + (size_t)a * kAcc;
  DBox bounds, cb;
  for (int k = 0; k < 3; ++k) {
    bounds.mn[k] = unord(A[k]);
    bounds.mx[k] = unord(A[3 + k]);
    cb.mn[k] = unord(A[6 + k]);
    cb.mx[k] = unord(A[9 + k]);
  }
  nd.bounds = bounds;
  nd.leaf = 0;
  if (nd.count <= 1 || nd.level >= kMaxLevel) {
    nd.leaf = 1;
    return;
  }
  DBox bin_box[3 * kBins];
  uint32_t bin_n[3 * kBins];
  bool axis_ok[3];
  for (int axis = 0; axis < 3; ++axis) {
    axis_ok[axis] = cb.mx[axis] - cb.mn[axis] > 0;
    for (int b = 0; b < kBins; ++b) {
      const u64* B = A + 12 + (axis * kBins + b) * 7;
      bin_n[axis * kBins + b] = (uint32_t)B[0];
      for (int k = 0; k < 3; ++k) {
        bin_box[axis * kBins + b].mn[k] = unord(B[1 + k]);
        bin_box[axis * kBins + b].mx[k] = unord(B[4 + k]);
      }
    }
  }
  const Split s = sweep(bin_box, bin_n, axis_ok, dbox_area(bounds));
  if (!s.valid) { /* count > 4 here: splitMedian, left to the host */
    atomicExch(fallback, 1);
    nd.leaf = 1;
    return;
  }
  if (nd.count <= kLeafSize && s.cost >= (double)nd.count) {
    nd.leaf = 1;
    return;
  }
  nd.axis = (uint32_t)s.axis;
  nd.bin = s.bin;
  nd.lo = cb.mn[s.axis];
  nd.extent = cb.mx[s.axis] - nd.lo;
}

/* Goes-left flags of the positions of splitting nodes. */
__global__ void k_flags(const int32_t* __restrict__ node_of, const uint32_t* __restrict__ active,
                        const LargeNode* __restrict__ nodes, const uint32_t* __restrict__ idx,
                        const double* __restrict__ cent, uint32_t n, uint32_t* __restrict__ flag) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t a = node_of[p];
  uint32_t f = 0;
  if (a >= 0) {
    const LargeNode& nd = nodes[active[a]];
    if (!nd.leaf) f = bin_of(cent[3 * (size_t)idx[p] + nd.axis], nd.lo, nd.extent) <= nd.bin;
  }
  flag[p] = f;
}

/* Exclusive scan of n u32 values in three passes (1024 per block). */
constexpr int kScanBlock = 1024;

__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t* sh, uint32_t& total) {
  const int t = threadIdx.x, lane = t & 31, w = t >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[w] = x;
  __syncthreads();
  if (w == 0) {
    uint32_t s = lane < (int)(blockDim.x / 32) ? sh[lane] : 0;
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(0xffffffffu, s, o);
      if (lane >= o) s += y;
    }
    sh[lane] = s;
  }
  __syncthreads();
  const uint32_t incl = x + (w > 0 ? sh[w - 1] : 0);
  total = sh[blockDim.x / 32 - 1];
  __syncthreads();
  return incl - v;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_reduce(const uint32_t* __restrict__ in, uint32_t n,
                                                            uint32_t* __restrict__ block_sum) {
  __shared__ uint32_t sh[32];
  const uint32_t p = blockIdx.x * kScanBlock + threadIdx.x;
  uint32_t total;
  block_exclusive_scan(p < n ? in[p] : 0, sh, total);
  if (threadIdx.x == 0) block_sum[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanBlock) k_scan_sums(uint32_t* __restrict__ block_sum, uint32_t nb) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (uint32_t base = 0; base < nb; base += kScanBlock) {
    const uint32_t p = base + threadIdx.x;
    uint32_t total;
    const uint32_t ex = block_exclusive_scan(p < nb ? block_sum[p] : 0, sh, total);
    if (p < nb) block_sum[p] = ex + carry;
    carry += total;
  }
}

__global__ void __launch_bounds__(kScanBlock) k_scan_apply(const uint32_t* __restrict__ in, uint32_t n,
                                                           const uint32_t* __restrict__ block_sum,
                                                           uint32_t* __restrict__ out) {
  __shared__ uint32_t sh[32];
  const uint32_t p = blockIdx.x * kScanBlock + threadIdx.x;
  uint32_t total;
  const uint32_t ex = block_exclusive_scan(p < n ? in[p] : 0, sh, total);
  if (p <= n) out[p] = ex + block_sum[blockIdx.x]; /* out has n + 1 entries */
}

/* rank(p) for positions of splitting nodes; mid per node. */
__global__ void k_jump_init(const int32_t* __restrict__ node_of, const uint32_t* __restrict__ active,
                            const LargeNode* __restrict__ nodes, const uint32_t* __restrict__ flag,
                            const uint32_t* __restrict__ pre, uint32_t n, uint32_t* __restrict__ nxt) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t a = node_of[p];
  uint32_t v = p;
  if (a >= 0) {
    const LargeNode& nd = nodes[active[a]];
    if (!nd.leaf && flag[p]) v = nd.first + (pre[p] - pre[nd.first]);
  }
  nxt[p] = v;
}

__global__ void k_jump(const uint32_t* __restrict__ in, uint32_t n, uint32_t* __restrict__ out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < n) out[p] = in[in[p]];
}

__global__ void k_set_mid(LargeNode* __restrict__ nodes, const uint32_t* __restrict__ active, uint32_t m,
                          const uint32_t* __restrict__ pre) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= m) return;
  LargeNode& nd = nodes[active[a]];
  if (!nd.leaf) nd.mid = pre[nd.first + nd.count] - pre[nd.first];
}

/* The partitioned ranges (Lomuto note above); other positions copied. */
__global__ void k_scatter(const int32_t* __restrict__ node_of, const uint32_t* __restrict__ active,
                          const LargeNode* __restrict__ nodes, const uint32_t* __restrict__ flag,
                          const uint32_t* __restrict__ pre, const uint32_t* __restrict__ root, uint32_t n,
                          const uint32_t* __restrict__ idx, uint32_t* __restrict__ out) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t a = node_of[p];
  if (a < 0 || nodes[active[a]].leaf) {
    out[p] = idx[p];
    return;
  }
  const LargeNode& nd = nodes[active[a]];
  const uint32_t q = p - nd.first;
  const uint32_t r = pre[p] - pre[nd.first];
  if (flag[p]) out[nd.first + r] = idx[p];
  if (q >= nd.mid) out[p] = flag[p] ? idx[root[nd.first + r]] : idx[p];
}

/* Children of splitting nodes: large ones to the next level, small ones to
 * the warp-built subtrees. */
__global__ void k_children(LargeNode* __restrict__ nodes, const uint32_t* __restrict__ active, uint32_t m,
                           uint32_t* __restrict__ n_nodes, uint32_t* __restrict__ next, uint32_t* __restrict__ n_next,
                           Subtree* __restrict__ subs, uint32_t* __restrict__ n_subs) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= m) return;
  LargeNode& nd = nodes[active[a]];
  if (nd.leaf) {
    nd.child[0] = nd.child[1] = 0;
    return;
  }
  const uint32_t fc[2] = {nd.first, nd.first + nd.mid}, cc[2] = {nd.mid, nd.count - nd.mid};
  for (int side = 0; side < 2; ++side) {
    if (cc[side] > kSmall) {
      const uint32_t id = atomicAdd(n_nodes, 1u);
      LargeNode& c = nodes[id];
      c.first = fc[side];
      c.count = cc[side];
      c.level = nd.level + 1;
      c.leaf = 0;
      next[atomicAdd(n_next, 1u)] = id;
      nd.child[side] = (int32_t)id;
    } else {
      const uint32_t id = atomicAdd(n_subs, 1u);
      subs[id].first = fc[side];
      subs[id].count = cc[side];
      subs[id].level = nd.level + 1;
      nd.child[side] = -1 - (int32_t)id;
    }
  }
}

/* ------------------------------------------------------------------------
 * Small subtrees: one warp each, depth first.
 * ---------------------------------------------------------------------- */
struct LNode {       /* one node of a warp-built subtree, in visit (preorder) order */
  DBox bounds;
  uint32_t first, count;
  int32_t lrank;     /* preorder rank of its split within the subtree, -1 for a leaf */
  int32_t parent;    /* slot of the parent, -1 for the subtree root */
  uint32_t side;
};

constexpr int kWarpsPerBlock = 4;

__global__ void __launch_bounds__(32 * kWarpsPerBlock, 8) k_small(Subtree* __restrict__ subs, uint32_t n_subs,
                                                              uint32_t* __restrict__ idx,
                                                              const DBox* __restrict__ boxes,
                                                              const double* __restrict__ cent,
                                                              LNode* __restrict__ lnodes, int* __restrict__ fallback) {
  struct Entry { uint32_t first, count, level; int32_t parent; uint32_t side; };
  __shared__ Entry stack[kWarpsPerBlock][33];
  __shared__ u64 sbox[kWarpsPerBlock][32][6];
  __shared__ uint32_t sbin[kWarpsPerBlock][32];
  __shared__ double sbb[kWarpsPerBlock][3 * kBins][6];
  __shared__ uint32_t sbn[kWarpsPerBlock][3 * kBins];
  const int w = threadIdx.x / 32, lane = threadIdx.x % 32;
  const uint32_t s = blockIdx.x * kWarpsPerBlock + w;
  if (s >= n_subs) return;
  Subtree& st = subs[s];
  LNode* out = lnodes + 2 * (size_t)st.first; /* 2 * count - 1 slots of this subtree */
  int sp = 0, slots = 0, ranks = 0;
  if (lane == 0) stack[w][0] = Entry{st.first, st.count, st.level, -1, 0};
  sp = 1;
  __syncwarp();
  while (sp > 0) {
    --sp;
    const Entry en = stack[w][sp];
    __syncwarp();
    const uint32_t c = en.count;
    const int slot = slots++;
    const bool live = (uint32_t)lane < c;
    const uint32_t e = live ? idx[en.first + lane] : 0;
    DBox b;
    double ce[3];
    u64 v[12];
    if (live) {
      b = boxes[e];
      for (int k = 0; k < 3; ++k) {
        ce[k] = cent[3 * (size_t)e + k];
        v[k] = ord(b.mn[k]);
        v[3 + k] = ord(b.mx[k]);
        v[6 + k] = v[9 + k] = ord(ce[k]);
      }
    } else {
      for (int k = 0; k < 3; ++k) { v[k] = v[6 + k] = ORD_POS_INF; v[3 + k] = v[9 + k] = ORD_NEG_INF; }
    }
    for (int k = 0; k < 3; ++k) {
      warp_min_max(v[k], v[3 + k], 0xffffffffu);
      warp_min_max(v[6 + k], v[9 + k], 0xffffffffu);
    }
    DBox bounds, cb;
    for (int k = 0; k < 3; ++k) {
      bounds.mn[k] = unord(v[k]);
      bounds.mx[k] = unord(v[3 + k]);
      cb.mn[k] = unord(v[6 + k]);
      cb.mx[k] = unord(v[9 + k]);
    }
    LNode rec;
    rec.bounds = bounds;
    rec.first = en.first;
    rec.count = c;
    rec.lrank = -1;
    rec.parent = en.parent;
    rec.side = en.side;
    bool split = !(c <= 1 || en.level >= kMaxLevel);
    Split sp_best{0, 0, 0.0, false};
    if (split) {
      /* bins: each lane's box into shared memory, then one lane per (axis, bin) */
      if (live)
        for (int k = 0; k < 3; ++k) {
          sbox[w][lane][k] = ord(b.mn[k]);
          sbox[w][lane][3 + k] = ord(b.mx[k]);
        }
      bool axis_ok[3];
      for (int axis = 0; axis < 3; ++axis) {
        const double lo = cb.mn[axis], extent = cb.mx[axis] - lo;
        axis_ok[axis] = extent > 0;
        __syncwarp();
        if (live) sbin[w][lane] = axis_ok[axis] ? bin_of(ce[axis], lo, extent) : 0;
        __syncwarp();
        if (lane < kBins) {
          u64 mn[3] = {ORD_POS_INF, ORD_POS_INF, ORD_POS_INF}, mx[3] = {ORD_NEG_INF, ORD_NEG_INF, ORD_NEG_INF};
          uint32_t cnt = 0;
          for (uint32_t j = 0; j < c; ++j) {
            if (sbin[w][j] != (uint32_t)lane) continue;
            ++cnt;
            for (int k = 0; k < 3; ++k) {
              mn[k] = sbox[w][j][k] < mn[k] ? sbox[w][j][k] : mn[k];
              mx[k] = sbox[w][j][3 + k] > mx[k] ? sbox[w][j][3 + k] : mx[k];
            }
          }
          sbn[w][axis * kBins + lane] = cnt;
          for (int k = 0; k < 3; ++k) {
            sbb[w][axis * kBins + lane][k] = unord(mn[k]);
            sbb[w][axis * kBins + lane][3 + k] = unord(mx[k]);
          }
        }
      }
      __syncwarp();
      /* one lane per axis runs findSplit's sweep; lane 0 keeps the best in
       * axis order */
      const double parent_area = dbox_area(bounds);
      Split mine{0, 0, 0.0, false};
      if (lane < 3 && parent_area > 0 && axis_ok[lane]) {
        const int base = lane * kBins;
        mine = sweep_axis(
            [&](int b) {
              DBox r;
              for (int k = 0; k < 3; ++k) {
                r.mn[k] = sbb[w][base + b][k];
                r.mx[k] = sbb[w][base + b][3 + k];
              }
              return r;
            },
            sbn[w] + base, lane, parent_area);
      }
      for (int a = 0; a < 3; ++a) {
        Split c;
        c.valid = __shfl_sync(0xffffffffu, mine.valid, a);
        c.axis = __shfl_sync(0xffffffffu, mine.axis, a);
        c.bin = __shfl_sync(0xffffffffu, mine.bin, a);
        c.cost = __shfl_sync(0xffffffffu, mine.cost, a);
        keep_better(sp_best, c);
      }
      if (!sp_best.valid) {
        if (c > kLeafSize && lane == 0) atomicExch(fallback, 1); /* splitMedian: host */
        split = false;
      } else if (c <= kLeafSize && sp_best.cost >= (double)c) {
        split = false;
      }
    }
    if (split) {
      rec.lrank = ranks++;
      const int axis = sp_best.axis;
      const double lo = cb.mn[axis], extent = cb.mx[axis] - lo;
      const bool L = live && bin_of(ce[axis], lo, extent) <= sp_best.bin;
      const unsigned ball = __ballot_sync(0xffffffffu, L);
      const uint32_t mid = __popc(ball);
      const uint32_t rank = __popc(ball & ((1u << lane) - 1u));
      /* G by pointer jumping: root(p) = p for non-L, else root(rank(p)) */
      uint32_t nx = L ? rank : (uint32_t)lane;
      for (int it = 0; it < 5; ++it) nx = __shfl_sync(0xffffffffu, nx, nx);
      const uint32_t g_elem = __shfl_sync(0xffffffffu, e, nx); /* G(lane) */
      const int src = (uint32_t)lane < mid ? (int)__fns(ball, 0, lane + 1) : lane; /* the L element of rank lane */
      const uint32_t from_left = __shfl_sync(0xffffffffu, e, src);
      const uint32_t from_g = __shfl_sync(0xffffffffu, g_elem, rank);
      const uint32_t newe = (uint32_t)lane < mid ? from_left : (L ? from_g : e);
      if (live) idx[en.first + lane] = newe;
      __syncwarp();
      if (lane == 0) { /* right first so the left child is visited next */
        stack[w][sp] = Entry{en.first + mid, c - mid, en.level + 1, slot, 1};
        stack[w][sp + 1] = Entry{en.first, mid, en.level + 1, slot, 0};
      }
      sp += 2;
      __syncwarp();
    }
    if (lane == 0) out[slot] = rec;
    __syncwarp();
  }
  if (lane == 0) st.internal = (uint32_t)ranks;
}

/* ------------------------------------------------------------------------
 * Numbering and output.
 * ---------------------------------------------------------------------- */
__global__ void k_count_internal(LargeNode* __restrict__ nodes, const uint32_t* __restrict__ level_ids, uint32_t m,
                                 const Subtree* __restrict__ subs) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= m) return;
  LargeNode& nd = nodes[level_ids[a]];
  if (nd.leaf) {
    nd.internal = 0;
    return;
  }
  uint32_t t = 1;
  for (int side = 0; side < 2; ++side) {
    const int32_t c = nd.child[side];
    t += c >= 0 ? nodes[c].internal : subs[-1 - c].internal;
  }
  nd.internal = t;
}

__device__ __forceinline__ void put_node(HostNode* out, uint32_t i, const DBox& b, uint32_t first, uint32_t count) {
  HostNode h;
  for (int k = 0; k < 3; ++k) { h.bmin[k] = b.mn[k]; h.bmax[k] = b.mx[k]; }
  h.first = first;
  h.count = count;
  out[i] = h;
}

/* Large nodes of one level: own record, children's index and rank. */
__global__ void k_emit_large(LargeNode* __restrict__ nodes, const uint32_t* __restrict__ level_ids, uint32_t m,
                             Subtree* __restrict__ subs, HostNode* __restrict__ out) {
  const uint32_t a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= m) return;
  LargeNode& nd = nodes[level_ids[a]];
  if (nd.leaf) {
    put_node(out, nd.index, nd.bounds, nd.first, nd.count);
    return;
  }
  put_node(out, nd.index, nd.bounds, 2 * nd.rank + 1, 0);
  uint32_t next_rank = nd.rank + 1;
  for (int side = 0; side < 2; ++side) {
    const int32_t c = nd.child[side];
    const uint32_t index = 2 * nd.rank + 1 + side;
    if (c >= 0) {
      nodes[c].index = index;
      nodes[c].rank = next_rank;
      next_rank += nodes[c].internal;
    } else {
      subs[-1 - c].index = index;
      subs[-1 - c].rank = next_rank;
      next_rank += subs[-1 - c].internal;
    }
  }
}

/* Warp-built subtrees: place each node of the subtree (2 * internal + 1
 * slots, in visit order). */
__global__ void k_emit_small(const Subtree* __restrict__ subs, uint32_t n_subs, const LNode* __restrict__ lnodes,
                             HostNode* __restrict__ out) {
  const uint32_t s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n_subs) return;
  const Subtree st = subs[s];
  const LNode* ln = lnodes + 2 * (size_t)st.first;
  const uint32_t n_slots = 2 * st.internal + 1;
  for (uint32_t k = 0; k < n_slots; ++k) {
    const LNode r = ln[k];
    const uint32_t i = r.parent < 0 ? st.index : 2 * (st.rank + (uint32_t)ln[r.parent].lrank) + 1 + r.side;
    if (r.lrank >= 0) put_node(out, i, r.bounds, 2 * (st.rank + (uint32_t)r.lrank) + 1, 0);
    else put_node(out, i, r.bounds, r.first, r.count);
  }
}

}  // namespace

/* Host driver.  Returns ZT_OK with s->nodes / s->indices filled, or
 * ZT_DEVICE_BUILD_FALLBACK when the host builder must be used. */
zt_status device_build_bvh(zt_scene* s, double* build_ms) {
  const size_t n = s->shapes.size();
  s->nodes.clear();
  s->indices.clear();
  if (n == 0) return ZT_OK;
  if (n > 0x7FFFFFFFull) return fail(ZT_ERR_TOO_MANY_PRIMITIVES, "TooManyPrimitives: more than 2^31 bounded shapes");
  const uint32_t N = (uint32_t)n;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaEventRecord(ev0, 0);

  /* one allocation for everything */
  const uint32_t max_large = 2 * (N / (kSmall + 1)) + 2;
  const uint32_t max_subs = 2 * max_large + 2;
  auto up = [](size_t b) { return (b + 255) & ~(size_t)255; };
  size_t off = 0;
  const size_t o_shapes = off; off += up(n * sizeof(zt_shape));
  const size_t o_boxes = off; off += up(n * sizeof(DBox));
  const size_t o_cent = off; off += up(3 * n * sizeof(double));
  const size_t o_idx = off; off += up(n * 4);
  const size_t o_idx2 = off; off += up(n * 4);
  const size_t o_node_of = off; off += up(n * 4);
  const size_t o_flag = off; off += up(n * 4);
  const size_t o_pre = off; off += up((n + 1) * 4);
  const size_t o_nxt = off; off += up(n * 4);
  const size_t o_nxt2 = off; off += up(n * 4);
  const size_t o_bsum = off; off += up(((n + kScanBlock) / kScanBlock + 1) * 4);
  const size_t o_large = off; off += up((size_t)max_large * sizeof(LargeNode));
  const size_t o_subs = off; off += up((size_t)max_subs * sizeof(Subtree));
  const size_t o_lists = off; off += up((size_t)2 * max_large * 4);
  const size_t o_ctl = off; off += up(16 * 4);
  const size_t o_acc = off; off += up((size_t)(N / (kSmall + 1) + 1) * kAcc * 8);
  const size_t o_lnodes = off; off += up(2 * n * sizeof(LNode));
  const size_t o_out = off; off += up((2 * n - 1) * sizeof(HostNode));
  unsigned char* mem = nullptr;
  cudaError_t e = cudaMalloc((void**)&mem, off);
  if (e != cudaSuccess) { /* no device, or not enough device memory: the host builds it */
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    cudaGetLastError();
    return ZT_DEVICE_BUILD_FALLBACK;
  }
  zt_shape* d_shapes = (zt_shape*)(mem + o_shapes);
  DBox* d_boxes = (DBox*)(mem + o_boxes);
  double* d_cent = (double*)(mem + o_cent);
  uint32_t* d_idx = (uint32_t*)(mem + o_idx);
  uint32_t* d_idx2 = (uint32_t*)(mem + o_idx2);
  int32_t* d_node_of = (int32_t*)(mem + o_node_of);
  uint32_t* d_flag = (uint32_t*)(mem + o_flag);
  uint32_t* d_pre = (uint32_t*)(mem + o_pre);
  uint32_t* d_nxt = (uint32_t*)(mem + o_nxt);
  uint32_t* d_nxt2 = (uint32_t*)(mem + o_nxt2);
  uint32_t* d_bsum = (uint32_t*)(mem + o_bsum);
  LargeNode* d_large = (LargeNode*)(mem + o_large);
  Subtree* d_subs = (Subtree*)(mem + o_subs);
  uint32_t* d_list[2] = {(uint32_t*)(mem + o_lists), (uint32_t*)(mem + o_lists) + max_large};
  uint32_t* d_ctl = (uint32_t*)(mem + o_ctl); /* 0 n_large, 1 n_next, 2 n_subs, 3 bad, 4 fallback */
  u64* d_acc = (u64*)(mem + o_acc);
  LNode* d_lnodes = (LNode*)(mem + o_lnodes);
  HostNode* d_out = (HostNode*)(mem + o_out);

  zt_status rc = ZT_OK;
  auto ck = [&](cudaError_t err, const char* what) {
    if (err != cudaSuccess && rc == ZT_OK) rc = fail(ZT_ERR_CUDA, std::string("device BVH build: ") + what + ": " +
                                                                    cudaGetErrorString(err));
    return rc == ZT_OK;
  };
  const unsigned G = (N + 255) / 256;
  std::vector<std::vector<uint32_t>> levels; /* large node ids per level, for the numbering passes */
  uint32_t n_subs = 0;
  do {
    if (!ck(cudaMemcpy(d_shapes, s->shapes.data(), n * sizeof(zt_shape), cudaMemcpyHostToDevice), "upload shapes"))
      break;
    if (!ck(cudaMemset(d_ctl, 0, 16 * 4), "clear")) break;
    k_prim_boxes<<<G, 256>>>(d_shapes, N, d_boxes, d_cent, d_idx, (int*)(d_ctl + 3));
    uint32_t ctl[8];
    if (!ck(cudaMemcpy(ctl, d_ctl, 8 * 4, cudaMemcpyDeviceToHost), "boxes")) break;
    if (ctl[3]) { rc = ZT_DEVICE_BUILD_FALLBACK; break; }
    /* the root: large, or a single warp subtree */
    std::vector<uint32_t> active;
    if (N > kSmall) {
      LargeNode root;
      memset(&root, 0, sizeof root);
      root.first = 0;
      root.count = N;
      root.level = 0;
      root.index = 0;
      root.rank = 0;
      if (!ck(cudaMemcpy(d_large, &root, sizeof root, cudaMemcpyHostToDevice), "root")) break;
      const uint32_t one = 1, zero = 0;
      if (!ck(cudaMemcpy(d_ctl, &one, 4, cudaMemcpyHostToDevice), "root count")) break;
      if (!ck(cudaMemcpy(d_list[0], &zero, 4, cudaMemcpyHostToDevice), "root list")) break;
      active.push_back(0);
    } else {
      Subtree root{0, N, 0, 0, 0, 0};
      if (!ck(cudaMemcpy(d_subs, &root, sizeof root, cudaMemcpyHostToDevice), "root")) break;
      const uint32_t one = 1;
      if (!ck(cudaMemcpy(d_ctl + 2, &one, 4, cudaMemcpyHostToDevice), "root count")) break;
    }
    int cur = 0;
    while (!active.empty() && rc == ZT_OK) {
      const uint32_t m = (uint32_t)active.size();
      levels.push_back(active);
      uint32_t* d_active = d_list[cur];
      ck(cudaMemset(d_node_of, 0xFF, n * 4), "node_of");
      k_acc_init<<<(unsigned)(((uint64_t)m * kAcc + 255) / 256), 256>>>(d_acc, m);
      k_mark<<<m, 256>>>(d_large, d_active, m, d_node_of);
      k_bounds<<<G, 256>>>(d_node_of, d_idx, d_boxes, d_cent, N, d_acc);
      k_bins<<<G, 256>>>(d_node_of, d_idx, d_boxes, d_cent, N, d_acc);
      k_decide<<<(m + 127) / 128, 128>>>(d_large, d_active, m, d_acc, (int*)(d_ctl + 4));
      k_flags<<<G, 256>>>(d_node_of, d_active, d_large, d_idx, d_cent, N, d_flag);
      const uint32_t nb = (N + kScanBlock) / kScanBlock;
      k_scan_reduce<<<nb, kScanBlock>>>(d_flag, N, d_bsum);
      k_scan_sums<<<1, kScanBlock>>>(d_bsum, nb);
      k_scan_apply<<<nb, kScanBlock>>>(d_flag, N, d_bsum, d_pre);
      k_set_mid<<<(m + 127) / 128, 128>>>(d_large, d_active, m, d_pre);
      k_jump_init<<<G, 256>>>(d_node_of, d_active, d_large, d_flag, d_pre, N, d_nxt);
      /* pointer jumping: chains are shorter than the largest node (< N) */
      uint32_t* a = d_nxt;
      uint32_t* b = d_nxt2;
      for (uint64_t len = 1; len < N; len <<= 1) {
        k_jump<<<G, 256>>>(a, N, b);
        std::swap(a, b);
      }
      k_scatter<<<G, 256>>>(d_node_of, d_active, d_large, d_flag, d_pre, a, N, d_idx, d_idx2);
      std::swap(d_idx, d_idx2);
      const uint32_t zero = 0;
      ck(cudaMemcpy(d_ctl + 1, &zero, 4, cudaMemcpyHostToDevice), "next count");
      k_children<<<(m + 127) / 128, 128>>>(d_large, d_active, m, d_ctl, d_list[cur ^ 1], d_ctl + 1, d_subs, d_ctl + 2);
      if (!ck(cudaGetLastError(), "level kernels")) break;
      if (!ck(cudaMemcpy(ctl, d_ctl, 8 * 4, cudaMemcpyDeviceToHost), "level")) break;
      if (ctl[4]) { rc = ZT_DEVICE_BUILD_FALLBACK; break; }
      active.resize(ctl[1]);
      if (ctl[1] && !ck(cudaMemcpy(active.data(), d_list[cur ^ 1], ctl[1] * 4, cudaMemcpyDeviceToHost), "next"))
        break;
      cur ^= 1;
    }
    if (rc != ZT_OK) break;
    if (!ck(cudaMemcpy(&n_subs, d_ctl + 2, 4, cudaMemcpyDeviceToHost), "subtrees")) break;
    if (n_subs) k_small<<<(n_subs + kWarpsPerBlock - 1) / kWarpsPerBlock, 32 * kWarpsPerBlock>>>(
        d_subs, n_subs, d_idx, d_boxes, d_cent, d_lnodes, (int*)(d_ctl + 4));
    if (!ck(cudaGetLastError(), "subtrees")) break;
    if (!ck(cudaMemcpy(ctl, d_ctl, 8 * 4, cudaMemcpyDeviceToHost), "subtree status")) break;
    if (ctl[4]) { rc = ZT_DEVICE_BUILD_FALLBACK; break; }
    /* numbering: internal counts bottom-up, ranks and records top-down */
    uint32_t* d_ids = d_list[0];
    for (size_t L = levels.size(); L-- > 0;) {
      const uint32_t m = (uint32_t)levels[L].size();
      ck(cudaMemcpy(d_ids, levels[L].data(), m * 4, cudaMemcpyHostToDevice), "ids");
      k_count_internal<<<(m + 127) / 128, 128>>>(d_large, d_ids, m, d_subs);
    }
    for (size_t L = 0; L < levels.size(); ++L) {
      const uint32_t m = (uint32_t)levels[L].size();
      ck(cudaMemcpy(d_ids, levels[L].data(), m * 4, cudaMemcpyHostToDevice), "ids");
      k_emit_large<<<(m + 127) / 128, 128>>>(d_large, d_ids, m, d_subs, d_out);
    }
    if (n_subs) k_emit_small<<<(n_subs + 127) / 128, 128>>>(d_subs, n_subs, d_lnodes, d_out);
    if (!ck(cudaGetLastError(), "numbering")) break;
    cudaEventRecord(ev1, 0);
    uint32_t internal = 0; /* of the whole tree: 2 * internal + 1 nodes */
    if (N > kSmall) {
      if (!ck(cudaMemcpy(&internal, &d_large[0].internal, 4, cudaMemcpyDeviceToHost), "node count")) break;
    } else if (!ck(cudaMemcpy(&internal, &d_subs[0].internal, 4, cudaMemcpyDeviceToHost), "node count")) {
      break;
    }
    s->nodes.resize(2 * (size_t)internal + 1);
    s->indices.resize(n);
    if (!ck(cudaMemcpy(s->nodes.data(), d_out, s->nodes.size() * sizeof(HostNode), cudaMemcpyDeviceToHost), "nodes"))
      break;
    if (!ck(cudaMemcpy(s->indices.data(), d_idx, n * 4, cudaMemcpyDeviceToHost), "indices")) break;
  } while (false);
  if (rc == ZT_OK && build_ms) {
    cudaEventSynchronize(ev1);
    float ms = 0;
    cudaEventElapsedTime(&ms, ev0, ev1);
    *build_ms = ms;
  }
  cudaFree(mem);
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
  if (rc != ZT_OK) {
    s->nodes.clear();
    s->indices.clear();
  }
  return rc;
}

}  // namespace zt
