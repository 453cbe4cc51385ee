// Device kd-tree builder (XYZGPU_BUILD_DEVICE): the binned-SAH build of
// kdbuild_host.cpp performed breadth first on the GPU, one level at a time,
// producing the identical flattened tree (same float operations in the same
// order, --fmad=false; integer histograms and scans are order independent).
//
// Per level (m nodes, R references, each node's references contiguous):
//   classify   nodes with >= kBigRefs references are listed ("big"): their
//              histograms, left / right counts and emit run on up to 128 CTAs
//              each (slices of the references), the SAH decision on one CTA
//              each; the rest get one warp each
//   decide     binned start/end histograms per axis in shared memory
//              (shared-memory atomics), exclusive prefix per axis, SAH cost of
//              every candidate plane, arg-min with the host's tie-break
//              (lowest axis, then lowest plane), exact left/right counts
//   scan       exclusive scan over nodes of (split, leaf refs, next refs,
//              empty leaf) -> child pair index, leaf offset, child ref offset
//   emit       node words, next-level node bounds and ranges, and a stable
//              scatter of references into the children (ballot / block scans,
//              and per-slice counts for big nodes, keep the parent's order) or
//              into the leaf reference array
// The host reads two small values per level (the big-node count and the scan
// totals) to size the next level; everything else stays on the device.
//
// Layout (kd_layout_depth_first, after either builder): the breadth-first
// array is permuted so that every subtree occupies one contiguous range, in
// depth-first order of child pairs: a pair (first, second) is followed by
// the first child's descendants, then the second's.  A ray descending into
// the first child finds that child's pair in the next bytes, usually the
// same 32-byte sector, and rays working in one region of space read one
// region of the array.  Node words keep their format; only child indices
// change.
#include <algorithm>
#include <vector>

#include "scene.h"

namespace xyzgpu {
namespace {

constexpr int kBigRefs = 2048;
constexpr int kBigThreads = 256;
constexpr int kBigSlicesMax = 128;     // CTAs per big node when emitting
constexpr int kBigSliceBudget = 1024;  // CTAs per emit launch (about)
constexpr int kWarpsPerBlock = 4;
constexpr int kScanThreads = 256;
constexpr int kScanPerThread = 8;
constexpr int kScanPerBlock = kScanThreads * kScanPerThread;

struct RefArrays {
  int32_t *tri;
  float *lo[3];
  float *hi[3];
};

struct LevelArrays {
  float4 *blo, *bhi;  // node bounds
  int32_t *begin, *count;
  int32_t *axis;      // -1: leaf
  float *plane;
  int32_t *nl, *nr;
  uint4 *scan;        // in: (split, leaf refs, next refs, empty leaf); out: exclusive prefix
};

struct BuildArgs {
  int leaf_max, max_depth, bins, depth;
  float ct, ci, eb;
};

XYZ_DEV float half_area3(float e0, float e1, float e2) { return e0 * e1 + e1 * e2 + e2 * e0; }
XYZ_DEV float comp4(float4 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

__global__ void k_init_refs(const float4 *__restrict__ tri, int n, RefArrays R) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float4 const a = tri[3 * i], b = tri[3 * i + 1], c = tri[3 * i + 2];
    // vertices as the intersection test sees them: v0, v0 + e1, v0 + e2
    float const v[3][3] = {{a.x, a.y, a.z}, {a.x + b.x, a.y + b.y, a.z + b.z},
                           {a.x + c.x, a.y + c.y, a.z + c.z}};
    R.tri[i] = i;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      R.lo[k][i] = fminf(fminf(v[0][k], v[1][k]), v[2][k]);
      R.hi[k][i] = fmaxf(fmaxf(v[0][k], v[1][k]), v[2][k]);
    }
  }
}

XYZ_DEV bool eligible(const BuildArgs &a, int n) { return n > a.leaf_max && a.depth < a.max_depth; }

__global__ void k_classify(LevelArrays L, int m, BuildArgs a, int32_t *big_list, int32_t *big_count) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    int const n = L.count[j];
    if (n >= kBigRefs && eligible(a, n)) big_list[atomicAdd(big_count, 1)] = j;
  }
}

// SAH over the exclusive prefix sums pre[a][0][i] (starts) and pre[a][1][i]
// (ends) of bins [0, i).  Candidate c = a * (B - 1) + (i - 1).  Returns the
// cost; +inf for invalid candidates.
XYZ_DEV float candidate_cost(const BuildArgs &A, int B, const uint32_t *pre, int c, int n, const float ext[3],
                             float4 lo4, float4 hi4, float sa, float *plane_out, int *nl_out) {
  int const a = c / (B - 1);
  int const i = c - a * (B - 1) + 1;
  if (!(ext[a] > 0.0f)) return INFINITY;
  float const lo = comp4(lo4, a);
  float const step = ext[a] / static_cast<float>(B);
  float const plane = lo + static_cast<float>(i) * step;
  uint32_t const nl = pre[(a * 2 + 0) * (kKdMaxBins + 1) + i];
  uint32_t const ended = pre[(a * 2 + 1) * (kKdMaxBins + 1) + i];
  int const nr = n - static_cast<int>(ended);
  float el[3] = {ext[0], ext[1], ext[2]};
  float er[3] = {ext[0], ext[1], ext[2]};
  el[a] = plane - lo;
  er[a] = comp4(hi4, a) - plane;
  float const sal = half_area3(el[0], el[1], el[2]);
  float const sar = half_area3(er[0], er[1], er[2]);
  float cost = A.ct + A.ci * (sal * static_cast<float>(nl) + sar * static_cast<float>(nr)) / sa;
  if (nl == 0 || nr == 0) cost = cost * (1.0f - A.eb);
  *plane_out = plane;
  *nl_out = static_cast<int>(nl);
  return cost;
}

XYZ_DEV void classify_ref(float lo, float hi, float plane, bool *l, bool *r) {
  bool const flat_on = (lo == plane) && (hi == plane);
  *l = (lo < plane) || flat_on;
  *r = (hi > plane) || flat_on;
}

XYZ_DEV int bin_of(float x, float lo, float scale, int B) {
  int b = static_cast<int>((x - lo) * scale);
  return min(max(b, 0), B - 1);
}

// Smaller (cost, candidate) first.
XYZ_DEV bool better(float c0, int i0, float c1, int i1) { return c0 < c1 || (c0 == c1 && i0 < i1); }

// ---- decide: one warp per small node
__global__ void __launch_bounds__(32 * kWarpsPerBlock)
    k_decide_small(LevelArrays L, int m, RefArrays R, BuildArgs A) {
  __shared__ uint32_t hist[kWarpsPerBlock][3 * 2 * (kKdMaxBins + 1)];
  int const lane = threadIdx.x & 31;
  int const wib = threadIdx.x >> 5;
  uint32_t *h = hist[wib];
  int const warp = blockIdx.x * kWarpsPerBlock + wib;
  int const nwarps = gridDim.x * kWarpsPerBlock;
  for (int j = warp; j < m; j += nwarps) {
    int const n = L.count[j];
    int const B = kd_node_bins(A.bins, n);
    if (n >= kBigRefs && eligible(A, n)) continue;  // a CTA decides this node
    if (!eligible(A, n)) {
      if (lane == 0) {
        L.axis[j] = -1;
        L.nl[j] = L.nr[j] = 0;
      }
      continue;
    }
    float4 const lo4 = L.blo[j], hi4 = L.bhi[j];
    float const ext[3] = {hi4.x - lo4.x, hi4.y - lo4.y, hi4.z - lo4.z};
    float const sa = half_area3(ext[0], ext[1], ext[2]);
    if (!(sa > 0.0f)) {
      if (lane == 0) {
        L.axis[j] = -1;
        L.nl[j] = L.nr[j] = 0;
      }
      continue;
    }
    // the six rows' first B + 1 entries (the rest is never read)
    for (int t = lane; t < 6 * (B + 1); t += 32) h[(t / (B + 1)) * (kKdMaxBins + 1) + t % (B + 1)] = 0u;
    __syncwarp();
    int const rb = L.begin[j];
    for (int a = 0; a < 3; ++a) {
      if (!(ext[a] > 0.0f)) continue;
      float const scale = static_cast<float>(B) / ext[a];
      float const lo = comp4(lo4, a);
      for (int r = lane; r < n; r += 32) {
        int const b0 = bin_of(R.lo[a][rb + r], lo, scale, B);
        int const b1 = bin_of(R.hi[a][rb + r], lo, scale, B);
        atomicAdd(&h[(a * 2 + 0) * (kKdMaxBins + 1) + b0], 1u);
        atomicAdd(&h[(a * 2 + 1) * (kKdMaxBins + 1) + b1], 1u);
      }
    }
    __syncwarp();
    // exclusive prefix of each of the six rows in place, the whole warp per
    // row: lane k holds bins 2k and 2k + 1 (B <= 64), an inclusive scan of
    // the pairs' sums over the lanes; row[B] gets the total
    for (int q = 0; q < 6; ++q) {
      uint32_t *row = h + q * (kKdMaxBins + 1);
      int const b0 = 2 * lane, b1 = 2 * lane + 1;
      uint32_t const v0 = b0 < B ? row[b0] : 0u, v1 = b1 < B ? row[b1] : 0u;
      uint32_t const pair = v0 + v1;
      uint32_t incl = pair;
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
        uint32_t const t = __shfl_up_sync(0xffffffffu, incl, off);
        if (lane >= off) incl += t;
      }
      __syncwarp();
      if (b0 < B) row[b0] = incl - pair;
      if (b1 < B) row[b1] = incl - pair + v0;
      if (lane == 31) row[B] = incl;
      __syncwarp();
    }
    float best = INFINITY;
    int best_c = 0x7fffffff;
    for (int c = lane; c < 3 * (B - 1); c += 32) {
      float pl;
      int nl;
      float const cost = candidate_cost(A, B, h, c, n, ext, lo4, hi4, sa, &pl, &nl);
      if (better(cost, c, best, best_c)) {
        best = cost;
        best_c = c;
      }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
      float const oc = __shfl_xor_sync(0xffffffffu, best, off);
      int const oi = __shfl_xor_sync(0xffffffffu, best_c, off);
      if (better(oc, oi, best, best_c)) {
        best = oc;
        best_c = oi;
      }
    }
    int axis = -1;
    float plane = 0.0f;
    if (best < A.ci * static_cast<float>(n)) {
      int nl_bin;
      candidate_cost(A, B, h, best_c, n, ext, lo4, hi4, sa, &plane, &nl_bin);
      axis = best_c / (B - 1);
    }
    int nl = 0, nr = 0;
    if (axis >= 0) {
      for (int r = lane; r < n; r += 32) {
        bool l, rr;
        classify_ref(R.lo[axis][rb + r], R.hi[axis][rb + r], plane, &l, &rr);
        nl += l;
        nr += rr;
      }
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) {
        nl += __shfl_xor_sync(0xffffffffu, nl, off);
        nr += __shfl_xor_sync(0xffffffffu, nr, off);
      }
    }
    if (lane == 0) {
      L.axis[j] = axis;
      L.plane[j] = plane;
      L.nl[j] = nl;
      L.nr[j] = nr;
    }
    __syncwarp();
  }
}

// ---- decide: one CTA per big node
// Big nodes use `slices` CTAs each for their O(n) passes; CTA g of a node
// takes the g-th contiguous slice of its references.
__device__ __forceinline__ void big_slice(int n, int slices, int g, int *b, int *e) {
  int const s = (n + slices - 1) / slices;
  *b = min(n, g * s);
  *e = min(n, *b + s);
}

constexpr int kHistWords = 3 * 2 * (kKdMaxBins + 1);

// Start / end bin histograms of a big node, one slice per CTA, added into the
// node's histogram in global memory (integer counts: the sum does not depend
// on the order of the slices).
__global__ void __launch_bounds__(kBigThreads) k_decide_big_hist(LevelArrays L, const int32_t *__restrict__ big_list,
                                                                 RefArrays R, BuildArgs A, int slices,
                                                                 uint32_t *__restrict__ gh) {
  __shared__ uint32_t h[kHistWords];
  int const ib = blockIdx.x / slices, g = blockIdx.x % slices;
  int const j = big_list[ib];
  int const n = L.count[j];
  int const B = kd_node_bins(A.bins, n);
  int const tid = threadIdx.x;
  float4 const lo4 = L.blo[j], hi4 = L.bhi[j];
  float const ext[3] = {hi4.x - lo4.x, hi4.y - lo4.y, hi4.z - lo4.z};
  if (!(half_area3(ext[0], ext[1], ext[2]) > 0.0f)) return;  // k_decide_big makes it a leaf
  for (int t = tid; t < kHistWords; t += kBigThreads) h[t] = 0u;
  __syncthreads();
  int b, e;
  big_slice(n, slices, g, &b, &e);
  int const rb = L.begin[j];
  for (int a = 0; a < 3; ++a) {
    if (!(ext[a] > 0.0f)) continue;
    float const scale = static_cast<float>(B) / ext[a];
    float const lo = comp4(lo4, a);
    for (int r = b + tid; r < e; r += kBigThreads) {
      int const b0 = bin_of(R.lo[a][rb + r], lo, scale, B);
      int const b1 = bin_of(R.hi[a][rb + r], lo, scale, B);
      atomicAdd(&h[(a * 2 + 0) * (kKdMaxBins + 1) + b0], 1u);
      atomicAdd(&h[(a * 2 + 1) * (kKdMaxBins + 1) + b1], 1u);
    }
  }
  __syncthreads();
  for (int t = tid; t < kHistWords; t += kBigThreads)
    if (h[t]) atomicAdd(&gh[static_cast<int64_t>(ib) * kHistWords + t], h[t]);
}

__global__ void __launch_bounds__(kBigThreads)
    k_decide_big(LevelArrays L, const int32_t *__restrict__ big_list, BuildArgs A,
                 const uint32_t *__restrict__ gh) {
  __shared__ uint32_t h[kHistWords];
  __shared__ float s_cost[kBigThreads / 32];
  __shared__ int s_idx[kBigThreads / 32];
  int const j = big_list[blockIdx.x];
  int const n = L.count[j];
  int const B = kd_node_bins(A.bins, n);
  int const tid = threadIdx.x;
  float4 const lo4 = L.blo[j], hi4 = L.bhi[j];
  float const ext[3] = {hi4.x - lo4.x, hi4.y - lo4.y, hi4.z - lo4.z};
  float const sa = half_area3(ext[0], ext[1], ext[2]);
  if (!(sa > 0.0f)) {
    if (tid == 0) {
      L.axis[j] = -1;
      L.nl[j] = L.nr[j] = 0;
    }
    return;
  }
  // the node's histograms, summed over its slices by k_decide_big_hist
  for (int t = tid; t < kHistWords; t += kBigThreads) h[t] = gh[static_cast<int64_t>(blockIdx.x) * kHistWords + t];
  __syncthreads();
  if (tid < 6) {
    uint32_t *row = h + tid * (kKdMaxBins + 1);
    uint32_t acc = 0u;
    for (int b = 0; b < B; ++b) {
      uint32_t const v = row[b];
      row[b] = acc;
      acc += v;
    }
    row[B] = acc;
  }
  __syncthreads();
  float best = INFINITY;
  int best_c = 0x7fffffff;
  for (int c = tid; c < 3 * (B - 1); c += kBigThreads) {
    float pl;
    int nl;
    float const cost = candidate_cost(A, B, h, c, n, ext, lo4, hi4, sa, &pl, &nl);
    if (better(cost, c, best, best_c)) {
      best = cost;
      best_c = c;
    }
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) {
    float const oc = __shfl_xor_sync(0xffffffffu, best, off);
    int const oi = __shfl_xor_sync(0xffffffffu, best_c, off);
    if (better(oc, oi, best, best_c)) {
      best = oc;
      best_c = oi;
    }
  }
  if ((tid & 31) == 0) {
    s_cost[tid >> 5] = best;
    s_idx[tid >> 5] = best_c;
  }
  __syncthreads();
  if (tid == 0) {
    for (int w = 1; w < kBigThreads / 32; ++w)
      if (better(s_cost[w], s_idx[w], best, best_c)) {
        best = s_cost[w];
        best_c = s_idx[w];
      }
    s_cost[0] = best;
    s_idx[0] = best_c;
  }
  __syncthreads();
  best = s_cost[0];
  best_c = s_idx[0];
  int axis = -1;
  float plane = 0.0f;
  if (best < A.ci * static_cast<float>(n)) {
    int nl_bin;
    candidate_cost(A, B, h, best_c, n, ext, lo4, hi4, sa, &plane, &nl_bin);
    axis = best_c / (B - 1);
  }
  // exact left / right counts: k_emit_big_count per slice, k_big_totals per node
  if (tid == 0) {
    L.axis[j] = axis;
    L.plane[j] = plane;
  }
}

__global__ void k_flags(LevelArrays L, int m, int force_leaves) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
    if (force_leaves) L.axis[j] = -1;
    int const split = L.axis[j] >= 0;
    int const n = L.count[j];
    L.scan[j] = make_uint4(split, split ? 0u : static_cast<uint32_t>(n),
                           split ? static_cast<uint32_t>(L.nl[j] + L.nr[j]) : 0u, (!split && n == 0) ? 1u : 0u);
  }
}

// ---- exclusive scan of uint4 (three kernels)
XYZ_DEV uint4 add4(uint4 a, uint4 b) { return make_uint4(a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w); }

XYZ_DEV uint4 block_exclusive(uint4 v, uint4 *total) {
  __shared__ uint4 warp_sums[kScanThreads / 32];
  int const lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  uint4 inc = v;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    uint4 o;
    o.x = __shfl_up_sync(0xffffffffu, inc.x, off);
    o.y = __shfl_up_sync(0xffffffffu, inc.y, off);
    o.z = __shfl_up_sync(0xffffffffu, inc.z, off);
    o.w = __shfl_up_sync(0xffffffffu, inc.w, off);
    if (lane >= off) inc = add4(inc, o);
  }
  if (lane == 31) warp_sums[w] = inc;
  __syncthreads();
  if (threadIdx.x == 0) {
    uint4 acc = make_uint4(0, 0, 0, 0);
    for (int k = 0; k < kScanThreads / 32; ++k) {
      uint4 const s = warp_sums[k];
      warp_sums[k] = acc;
      acc = add4(acc, s);
    }
    *total = acc;
  }
  __syncthreads();
  uint4 const ex = make_uint4(inc.x - v.x, inc.y - v.y, inc.z - v.z, inc.w - v.w);
  uint4 const r = add4(ex, warp_sums[w]);
  __syncthreads();
  return r;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_blocks(uint4 *data, int m, uint4 *block_sums) {
  __shared__ uint4 total;
  int const base = blockIdx.x * kScanPerBlock + threadIdx.x * kScanPerThread;
  uint4 loc[kScanPerThread];
  uint4 sum = make_uint4(0, 0, 0, 0);
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    loc[k] = base + k < m ? data[base + k] : make_uint4(0, 0, 0, 0);
    sum = add4(sum, loc[k]);
  }
  uint4 off = block_exclusive(sum, &total);
#pragma unroll
  for (int k = 0; k < kScanPerThread; ++k) {
    if (base + k < m) data[base + k] = off;
    off = add4(off, loc[k]);
  }
  if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_totals(uint4 *block_sums, int nb, uint4 *grand) {
  __shared__ uint4 total;
  uint4 carry = make_uint4(0, 0, 0, 0);
  for (int base = 0; base < nb; base += kScanThreads) {
    int const i = base + threadIdx.x;
    uint4 const v = i < nb ? block_sums[i] : make_uint4(0, 0, 0, 0);
    uint4 const ex = block_exclusive(v, &total);
    if (i < nb) block_sums[i] = add4(ex, carry);
    __syncthreads();
    carry = add4(carry, total);
    __syncthreads();
  }
  if (threadIdx.x == 0) *grand = carry;
}

__global__ void k_scan_add(uint4 *data, int m, const uint4 *block_sums) {
  int const i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < m) data[i] = add4(data[i], block_sums[i / kScanPerBlock]);
}

// ---- emit
struct EmitArgs {
  LevelArrays L, N;  // this level, next level
  RefArrays R, RN;   // this level's refs, next level's refs
  uint2 *nodes;
  int32_t *leaf_refs;
  int64_t level_base, next_base, leaf_base;
  int m;
};

XYZ_DEV void write_split_node(const EmitArgs &E, int j, int axis, float plane) {
  uint4 const sc = E.L.scan[j];
  int64_t const child = E.next_base + 2 * static_cast<int64_t>(sc.x);
  E.nodes[E.level_base + j] = make_uint2(__float_as_uint(plane),
                                         (static_cast<uint32_t>(child) << 2) | static_cast<uint32_t>(axis));
  int const c = 2 * static_cast<int>(sc.x);
  float4 lo = E.L.blo[j], hi = E.L.bhi[j];
  float4 hl = hi, lr = lo;
  if (axis == 0) hl.x = plane, lr.x = plane;
  if (axis == 1) hl.y = plane, lr.y = plane;
  if (axis == 2) hl.z = plane, lr.z = plane;
  E.N.blo[c] = lo;
  E.N.bhi[c] = hl;
  E.N.blo[c + 1] = lr;
  E.N.bhi[c + 1] = hi;
  E.N.begin[c] = static_cast<int32_t>(sc.z);
  E.N.count[c] = E.L.nl[j];
  E.N.begin[c + 1] = static_cast<int32_t>(sc.z) + E.L.nl[j];
  E.N.count[c + 1] = E.L.nr[j];
}

XYZ_DEV void write_ref(const RefArrays &D, int dst, const RefArrays &S, int src, int axis, float plane,
                       bool left) {
  D.tri[dst] = S.tri[src];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    float lo = S.lo[k][src], hi = S.hi[k][src];
    if (k == axis) {
      if (left)
        hi = fminf(hi, plane);
      else
        lo = fmaxf(lo, plane);
    }
    D.lo[k][dst] = lo;
    D.hi[k][dst] = hi;
  }
}

__global__ void __launch_bounds__(32 * kWarpsPerBlock) k_emit_small(EmitArgs E, BuildArgs A) {
  int const lane = threadIdx.x & 31;
  int const warp = blockIdx.x * kWarpsPerBlock + (threadIdx.x >> 5);
  int const nwarps = gridDim.x * kWarpsPerBlock;
  for (int j = warp; j < E.m; j += nwarps) {
    int const n = E.L.count[j];
    if (n >= kBigRefs && eligible(A, n)) continue;  // emitted by k_emit_big
    int const axis = E.L.axis[j];
    int const rb = E.L.begin[j];
    if (axis < 0) {
      uint4 const sc = E.L.scan[j];
      int64_t const off = E.leaf_base + sc.y;
      if (lane == 0)
        E.nodes[E.level_base + j] = make_uint2(static_cast<uint32_t>(off),
                                               (static_cast<uint32_t>(n) << 2) | kKdLeafTag);
      for (int r = lane; r < n; r += 32) E.leaf_refs[off + r] = E.R.tri[rb + r];
      continue;
    }
    float const plane = E.L.plane[j];
    if (lane == 0) write_split_node(E, j, axis, plane);
    int const lbase = static_cast<int>(E.L.scan[j].z);
    int const rbase = lbase + E.L.nl[j];
    int nl_run = 0, nr_run = 0;
    for (int r0 = 0; r0 < n; r0 += 32) {
      int const r = r0 + lane;
      bool l = false, rr = false;
      if (r < n) classify_ref(E.R.lo[axis][rb + r], E.R.hi[axis][rb + r], plane, &l, &rr);
      unsigned const ml = __ballot_sync(0xffffffffu, l);
      unsigned const mr = __ballot_sync(0xffffffffu, rr);
      unsigned const below = (1u << lane) - 1u;
      if (l) write_ref(E.RN, lbase + nl_run + __popc(ml & below), E.R, rb + r, axis, plane, true);
      if (rr) write_ref(E.RN, rbase + nr_run + __popc(mr & below), E.R, rb + r, axis, plane, false);
      nl_run += __popc(ml);
      nr_run += __popc(mr);
    }
  }
}

// Big nodes are emitted by `slices` CTAs each: CTA g of a node takes the g-th
// contiguous slice of its references.  A counting pass records each slice's
// left and right counts; the scatter pass starts each slice after the counts
// of the node's earlier slices and keeps the order within the slice, so the
// children receive the parent's references in the parent's order, as from a
// single CTA.

__global__ void __launch_bounds__(kBigThreads)
    k_emit_big_count(LevelArrays L, RefArrays R, const int32_t *__restrict__ big_list, int slices,
                     int2 *__restrict__ cnt) {
  __shared__ int s_red[2][kBigThreads / 32];
  int const j = big_list[blockIdx.x / slices], g = blockIdx.x % slices;
  int const axis = L.axis[j];
  if (axis < 0) return;  // leaf: its references are copied, not counted
  int const n = L.count[j], rb = L.begin[j];
  float const plane = L.plane[j];
  int b, e;
  big_slice(n, slices, g, &b, &e);
  int const tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  int cl = 0, cr = 0;
  for (int r = b + tid; r < e; r += kBigThreads) {
    bool l = false, rr = false;
    classify_ref(R.lo[axis][rb + r], R.hi[axis][rb + r], plane, &l, &rr);
    cl += l;
    cr += rr;
  }
  for (int o = 16; o > 0; o >>= 1) {
    cl += __shfl_down_sync(0xffffffffu, cl, o);
    cr += __shfl_down_sync(0xffffffffu, cr, o);
  }
  if (lane == 0) {
    s_red[0][w] = cl;
    s_red[1][w] = cr;
  }
  __syncthreads();
  if (tid == 0) {
    int tl = 0, tr = 0;
    for (int k = 0; k < kBigThreads / 32; ++k) {
      tl += s_red[0][k];
      tr += s_red[1][k];
    }
    cnt[blockIdx.x] = make_int2(tl, tr);
  }
}

// A big node's exact left / right reference counts: the sum of its slices'.
__global__ void k_big_totals(LevelArrays L, const int32_t *__restrict__ big_list, int slices,
                             const int2 *__restrict__ cnt) {
  int const j = big_list[blockIdx.x];
  int const lane = threadIdx.x;
  bool const split = L.axis[j] >= 0;
  int nl = 0, nr = 0;
  if (split)
    for (int k = lane; k < slices; k += 32) {
      int2 const c = cnt[blockIdx.x * slices + k];
      nl += c.x;
      nr += c.y;
    }
  for (int o = 16; o > 0; o >>= 1) {
    nl += __shfl_down_sync(0xffffffffu, nl, o);
    nr += __shfl_down_sync(0xffffffffu, nr, o);
  }
  if (lane == 0) {
    L.nl[j] = split ? nl : 0;
    L.nr[j] = split ? nr : 0;
  }
}

__global__ void __launch_bounds__(kBigThreads)
    k_emit_big(EmitArgs E, const int32_t *__restrict__ big_list, int slices, const int2 *__restrict__ cnt) {
  __shared__ int s_warp[2][kBigThreads / 32];
  __shared__ int s_run[2];
  int const first = (blockIdx.x / slices) * slices, g = blockIdx.x - first;
  int const j = big_list[blockIdx.x / slices];
  int const n = E.L.count[j];
  int const axis = E.L.axis[j];
  int const rb = E.L.begin[j];
  int const tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  int b, e;
  big_slice(n, slices, g, &b, &e);
  if (axis < 0) {
    uint4 const sc = E.L.scan[j];
    int64_t const off = E.leaf_base + sc.y;
    if (g == 0 && tid == 0)
      E.nodes[E.level_base + j] = make_uint2(static_cast<uint32_t>(off),
                                             (static_cast<uint32_t>(n) << 2) | kKdLeafTag);
    for (int r = b + tid; r < e; r += kBigThreads) E.leaf_refs[off + r] = E.R.tri[rb + r];
    return;
  }
  float const plane = E.L.plane[j];
  if (g == 0 && tid == 0) write_split_node(E, j, axis, plane);
  if (w == 0) {
    // references of the node's earlier slices
    int pl = 0, pr = 0;
    for (int k = lane; k < g; k += 32) {
      int2 const c = cnt[first + k];
      pl += c.x;
      pr += c.y;
    }
    for (int o = 16; o > 0; o >>= 1) {
      pl += __shfl_down_sync(0xffffffffu, pl, o);
      pr += __shfl_down_sync(0xffffffffu, pr, o);
    }
    if (lane == 0) {
      s_run[0] = pl;
      s_run[1] = pr;
    }
  }
  __syncthreads();
  int const lbase = static_cast<int>(E.L.scan[j].z);
  int const rbase = lbase + E.L.nl[j];
  for (int r0 = b; r0 < e; r0 += kBigThreads) {
    int const r = r0 + tid;
    bool l = false, rr = false;
    if (r < e) classify_ref(E.R.lo[axis][rb + r], E.R.hi[axis][rb + r], plane, &l, &rr);
    unsigned const ml = __ballot_sync(0xffffffffu, l);
    unsigned const mr = __ballot_sync(0xffffffffu, rr);
    if (lane == 0) {
      s_warp[0][w] = __popc(ml);
      s_warp[1][w] = __popc(mr);
    }
    __syncthreads();
    int pl = s_run[0], pr = s_run[1];
    for (int k = 0; k < w; ++k) {
      pl += s_warp[0][k];
      pr += s_warp[1][k];
    }
    unsigned const below = (1u << lane) - 1u;
    if (l) write_ref(E.RN, lbase + pl + __popc(ml & below), E.R, rb + r, axis, plane, true);
    if (rr) write_ref(E.RN, rbase + pr + __popc(mr & below), E.R, rb + r, axis, plane, false);
    __syncthreads();
    if (tid == 0) {
      for (int k = 0; k < kBigThreads / 32; ++k) {
        s_run[0] += s_warp[0][k];
        s_run[1] += s_warp[1][k];
      }
    }
    __syncthreads();
  }
}

// ---- device buffers
// Device buffer from the stream-ordered pool (the scene's build stream).
template <class T>
struct DevBuf {
  T *p = nullptr;
  int64_t cap = 0;
  cudaStream_t st = nullptr;
  ~DevBuf() {
    if (p) cudaFreeAsync(p, st);
  }
  // Grows to at least n elements, keeping the first `keep` elements.
  cudaError_t reserve(int64_t n, int64_t keep = 0) {
    if (n <= cap) return cudaSuccess;
    int64_t const nc = std::max<int64_t>(n, cap + cap / 2);
    T *q = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void **>(&q), nc * sizeof(T), st);
    if (e != cudaSuccess) return e;
    if (keep > 0 && p) {
      e = cudaMemcpyAsync(q, p, keep * sizeof(T), cudaMemcpyDeviceToDevice, st);
      if (e != cudaSuccess) {
        cudaFreeAsync(q, st);
        return e;
      }
    }
    if (p) cudaFreeAsync(p, st);
    p = q;
    cap = nc;
    return cudaSuccess;
  }
  T *release() {
    T *q = p;
    p = nullptr;
    cap = 0;
    return q;
  }
};

struct RefBufs {
  DevBuf<int32_t> tri;
  DevBuf<float> c[6];
  cudaError_t reserve(int64_t n) {
    cudaError_t e = tri.reserve(n);
    for (int k = 0; k < 6 && e == cudaSuccess; ++k) e = c[k].reserve(n);
    return e;
  }
  RefArrays view() {
    RefArrays r;
    r.tri = tri.p;
    for (int k = 0; k < 3; ++k) {
      r.lo[k] = c[k].p;
      r.hi[k] = c[3 + k].p;
    }
    return r;
  }
};

struct LevelBufs {
  DevBuf<float4> blo, bhi;
  DevBuf<int32_t> begin, count, axis, nl, nr;
  DevBuf<float> plane;
  DevBuf<uint4> scan;
  cudaError_t reserve(int64_t n) {
    cudaError_t e = blo.reserve(n);
    if (e == cudaSuccess) e = bhi.reserve(n);
    if (e == cudaSuccess) e = begin.reserve(n);
    if (e == cudaSuccess) e = count.reserve(n);
    if (e == cudaSuccess) e = axis.reserve(n);
    if (e == cudaSuccess) e = nl.reserve(n);
    if (e == cudaSuccess) e = nr.reserve(n);
    if (e == cudaSuccess) e = plane.reserve(n);
    if (e == cudaSuccess) e = scan.reserve(n);
    return e;
  }
  LevelArrays view() {
    return LevelArrays{blo.p, bhi.p, begin.p, count.p, axis.p, plane.p, nl.p, nr.p, scan.p};
  }
};

int grid_for(int64_t work, int threads, int device) {
  int64_t const want = (work + threads - 1) / threads;
  return static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t{sm_count(device)} * 16)));
}

// ---- depth-first layout
// Descendant counts of the nodes [begin, end) of one level (their children
// lie in deeper levels, counted before).
__global__ void k_layout_desc(const uint2 *__restrict__ nodes, int64_t begin, int64_t end, int32_t *desc) {
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint2 const nd = nodes[i];
    if ((nd.y & 3u) == kKdLeafTag) {
      desc[i] = 0;
    } else {
      uint32_t const c = nd.y >> 2;
      desc[i] = 2 + desc[c] + desc[c + 1];
    }
  }
}

__global__ void k_layout_root(int32_t *pos, int32_t *base) {
  pos[0] = 0;
  base[0] = 1;
}

// New positions of the children of the nodes [begin, end): the pair at
// base(parent); the first child's descendants from base + 2, the second's
// after them.
__global__ void k_layout_place(const uint2 *__restrict__ nodes, int64_t begin, int64_t end,
                               const int32_t *__restrict__ desc, int32_t *pos, int32_t *base) {
  for (int64_t i = begin + blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < end;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint2 const nd = nodes[i];
    if ((nd.y & 3u) == kKdLeafTag) continue;
    uint32_t const c = nd.y >> 2;
    int32_t const b = base[i];
    pos[c] = b;
    pos[c + 1] = b + 1;
    base[c] = b + 2;
    base[c + 1] = b + 2 + desc[c];
  }
}

__global__ void k_layout_scatter(const uint2 *__restrict__ nodes, int64_t n, const int32_t *__restrict__ pos,
                                 const int32_t *__restrict__ base, uint2 *__restrict__ out) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
    uint2 nd = nodes[i];
    if ((nd.y & 3u) != kKdLeafTag) nd.y = (static_cast<uint32_t>(base[i]) << 2) | (nd.y & 3u);
    out[pos[i]] = nd;
  }
}

}  // namespace

#define XYZ_BUILD_TRY(call)                                                                       \
  do {                                                                                            \
    cudaError_t const e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                        \
      return set_error(e_ == cudaErrorMemoryAllocation ? XYZGPU_E_NOMEM : XYZGPU_E_CUDA,          \
                       "kd-tree build: %s failed: %s", #call, cudaGetErrorString(e_));            \
  } while (0)

int kd_build_device(SceneImpl &s, const float4 *d_tri, int n, const BuildConfig &cfg, cudaStream_t st) {
  if (cfg.bins < 2 || cfg.bins > kKdMaxBins)
    return set_error(XYZGPU_E_INVALID, "kd-tree build: bins must be in [2, 64]");
  if (cfg.max_refs >= (int64_t{1} << 31))
    return set_error(XYZGPU_E_LIMIT, "kd-tree build: the reference budget exceeds 2^31 - 1 "
                                     "(lower max_refs_factor or the triangle count)");
  BuildArgs A;
  A.leaf_max = cfg.leaf_max_tris;
  A.max_depth = cfg.max_depth;
  A.bins = cfg.bins;
  A.ct = cfg.cost_traversal;
  A.ci = cfg.cost_intersect;
  A.eb = cfg.empty_bonus;
  int const dev = s.device;

  RefBufs refs[2];
  LevelBufs lv[2];
  DevBuf<uint2> nodes;
  DevBuf<int32_t> leaf_refs;
  DevBuf<int32_t> big_list, small_i32;
  DevBuf<int2> big_cnt;
  DevBuf<uint32_t> big_hist;
  DevBuf<uint4> block_sums, grand;
  for (int q = 0; q < 2; ++q) {
    refs[q].tri.st = st;
    for (auto &c : refs[q].c) c.st = st;
    for (auto *b : {&lv[q].begin, &lv[q].count, &lv[q].axis, &lv[q].nl, &lv[q].nr}) b->st = st;
    lv[q].blo.st = lv[q].bhi.st = st;
    lv[q].plane.st = st;
    lv[q].scan.st = st;
  }
  nodes.st = st;
  leaf_refs.st = st;
  big_list.st = small_i32.st = st;
  big_cnt.st = big_hist.st = st;
  block_sums.st = grand.st = st;
  XYZ_BUILD_TRY(refs[0].reserve(std::max(1, n)));
  XYZ_BUILD_TRY(lv[0].reserve(1));
  XYZ_BUILD_TRY(nodes.reserve(std::max<int64_t>(64, 2 * static_cast<int64_t>(n) / std::max(1, cfg.leaf_max_tris))));
  XYZ_BUILD_TRY(leaf_refs.reserve(std::max<int64_t>(64, 2 * static_cast<int64_t>(n))));
  XYZ_BUILD_TRY(small_i32.reserve(8));
  XYZ_BUILD_TRY(grand.reserve(1));

  if (n > 0) {
    k_init_refs<<<grid_for(n, 256, dev), 256, 0, st>>>(d_tri, n, refs[0].view());
    XYZ_BUILD_TRY(cudaGetLastError());
  }
  float4 const rlo = make_float4(s.dev.bmin.x, s.dev.bmin.y, s.dev.bmin.z, 0.0f);
  float4 const rhi = make_float4(s.dev.bmax.x, s.dev.bmax.y, s.dev.bmax.z, 0.0f);
  int32_t const zero = 0;
  XYZ_BUILD_TRY(cudaMemcpyAsync(lv[0].blo.p, &rlo, sizeof(float4), cudaMemcpyHostToDevice, st));
  XYZ_BUILD_TRY(cudaMemcpyAsync(lv[0].bhi.p, &rhi, sizeof(float4), cudaMemcpyHostToDevice, st));
  XYZ_BUILD_TRY(cudaMemcpyAsync(lv[0].begin.p, &zero, sizeof(int32_t), cudaMemcpyHostToDevice, st));
  XYZ_BUILD_TRY(cudaMemcpyAsync(lv[0].count.p, &n, sizeof(int32_t), cudaMemcpyHostToDevice, st));

  int64_t level_base = 0, leaf_total = 0, leaves = 0, empty = 0;
  int m = 1, depth = 0, cur = 0;
  std::vector<int64_t> level_start;
  for (depth = 0;; ++depth) {
    level_start.push_back(level_base);
    A.depth = depth;
    LevelArrays L = lv[cur].view();
    // big nodes
    XYZ_BUILD_TRY(big_list.reserve(m));
    XYZ_BUILD_TRY(cudaMemsetAsync(small_i32.p, 0, sizeof(int32_t), st));
    k_classify<<<grid_for(m, 256, dev), 256, 0, st>>>(L, m, A, big_list.p, small_i32.p);
    int32_t n_big = 0;
    XYZ_BUILD_TRY(cudaMemcpyAsync(&n_big, small_i32.p, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    XYZ_BUILD_TRY(cudaStreamSynchronize(st));
    RefArrays const R = refs[cur].view();
    k_decide_small<<<grid_for(int64_t{m} * 32, 32 * kWarpsPerBlock, dev), 32 * kWarpsPerBlock, 0, st>>>(L, m, R, A);
    // big nodes: sliced histograms, one CTA per node for the decision, sliced
    // left / right counts (kept for the emit) and their per-node totals;
    // slices per node: up to 128, about 1,024 CTAs per launch in all
    int const slices = n_big > 0 ? std::max(1, std::min(kBigSlicesMax, kBigSliceBudget / n_big)) : 1;
    if (n_big > 0) {
      XYZ_BUILD_TRY(big_hist.reserve(int64_t{n_big} * kHistWords));
      XYZ_BUILD_TRY(big_cnt.reserve(int64_t{n_big} * slices));
      XYZ_BUILD_TRY(cudaMemsetAsync(big_hist.p, 0, sizeof(uint32_t) * n_big * kHistWords, st));
      k_decide_big_hist<<<n_big * slices, kBigThreads, 0, st>>>(L, big_list.p, R, A, slices, big_hist.p);
      k_decide_big<<<n_big, kBigThreads, 0, st>>>(L, big_list.p, A, big_hist.p);
      k_emit_big_count<<<n_big * slices, kBigThreads, 0, st>>>(L, R, big_list.p, slices, big_cnt.p);
      k_big_totals<<<n_big, 32, 0, st>>>(L, big_list.p, slices, big_cnt.p);
    }
    XYZ_BUILD_TRY(cudaGetLastError());
    // flags + scan (twice if the reference budget is exceeded)
    uint4 tot = make_uint4(0, 0, 0, 0);
    for (int pass = 0; pass < 2; ++pass) {
      k_flags<<<grid_for(m, 256, dev), 256, 0, st>>>(L, m, pass);
      int const nb = static_cast<int>((m + kScanPerBlock - 1) / kScanPerBlock);
      XYZ_BUILD_TRY(block_sums.reserve(nb));
      k_scan_blocks<<<nb, kScanThreads, 0, st>>>(L.scan, m, block_sums.p);
      k_scan_totals<<<1, kScanThreads, 0, st>>>(block_sums.p, nb, grand.p);
      k_scan_add<<<(m + 255) / 256, 256, 0, st>>>(L.scan, m, block_sums.p);
      XYZ_BUILD_TRY(cudaGetLastError());
      XYZ_BUILD_TRY(cudaMemcpyAsync(&tot, grand.p, sizeof(uint4), cudaMemcpyDeviceToHost, st));
      XYZ_BUILD_TRY(cudaStreamSynchronize(st));
      if (static_cast<int64_t>(tot.z) <= cfg.max_refs) break;
    }
    int64_t const splits = tot.x;
    int64_t const next_m = 2 * splits;
    int64_t const next_base = level_base + m;
    if (next_base + next_m >= (int64_t{1} << 30))
      return set_error(XYZGPU_E_LIMIT, "kd-tree build: node count exceeds 2^30");
    XYZ_BUILD_TRY(nodes.reserve(next_base + std::max<int64_t>(next_m, 1), level_base));
    XYZ_BUILD_TRY(leaf_refs.reserve(leaf_total + std::max<int64_t>(tot.y, 1), leaf_total));
    XYZ_BUILD_TRY(lv[cur ^ 1].reserve(std::max<int64_t>(next_m, 1)));
    XYZ_BUILD_TRY(refs[cur ^ 1].reserve(std::max<int64_t>(tot.z, 1)));
    EmitArgs E;
    E.L = lv[cur].view();
    E.N = lv[cur ^ 1].view();
    E.R = refs[cur].view();
    E.RN = refs[cur ^ 1].view();
    E.nodes = nodes.p;
    E.leaf_refs = leaf_refs.p;
    E.level_base = level_base;
    E.next_base = next_base;
    E.leaf_base = leaf_total;
    E.m = m;
    k_emit_small<<<grid_for(int64_t{m} * 32, 32 * kWarpsPerBlock, dev), 32 * kWarpsPerBlock, 0, st>>>(E, A);
    // big_cnt was written by k_emit_big_count at decision time, before the
    // flag / scan passes, and holds valid per-slice counts only for nodes that
    // decided to split (axis >= 0); leaves never have theirs written.  The
    // second k_flags pass (reference budget exceeded) only turns nodes into
    // leaves (axis = -1), and k_emit_big takes its leaf branch for those
    // without reading cnt, so the counts stay valid for every node that reads
    // them here.
    if (n_big > 0) k_emit_big<<<n_big * slices, kBigThreads, 0, st>>>(E, big_list.p, slices, big_cnt.p);
    XYZ_BUILD_TRY(cudaGetLastError());
    leaves += m - splits;
    empty += tot.w;
    leaf_total += tot.y;
    level_base = next_base;
    if (next_m == 0) break;
    m = static_cast<int>(next_m);
    cur ^= 1;
  }
  XYZ_BUILD_TRY(cudaStreamSynchronize(st));
  level_start.push_back(level_base);
  s.n_nodes = level_base;
  s.n_refs = leaf_total;
  s.n_leaves = leaves;
  s.n_empty = empty;
  s.depth = depth;
  s.d_nodes = nodes.release();
  s.d_refs = leaf_refs.release();
  return kd_layout_depth_first(s, level_start, st);
}

int kd_layout_depth_first(SceneImpl &s, const std::vector<int64_t> &level_start, cudaStream_t st) {
  int64_t const n = s.n_nodes;
  if (n <= 1) return XYZGPU_OK;
  if (level_start.size() < 2 || level_start.front() != 0 || level_start.back() != n)
    return set_error(XYZGPU_E_INVALID, "kd-tree layout: level ranges do not cover the nodes");
  int const dev = s.device;
  DevBuf<int32_t> desc, pos, base;
  DevBuf<uint2> out;
  desc.st = pos.st = base.st = out.st = st;
  XYZ_BUILD_TRY(desc.reserve(n));
  XYZ_BUILD_TRY(pos.reserve(n));
  XYZ_BUILD_TRY(base.reserve(n));
  XYZ_BUILD_TRY(out.reserve(n));
  size_t const levels = level_start.size() - 1;
  for (size_t l = levels; l-- > 0;) {
    int64_t const b = level_start[l], e = level_start[l + 1];
    if (e > b) k_layout_desc<<<grid_for(e - b, 256, dev), 256, 0, st>>>(s.d_nodes, b, e, desc.p);
  }
  k_layout_root<<<1, 1, 0, st>>>(pos.p, base.p);
  for (size_t l = 0; l < levels; ++l) {
    int64_t const b = level_start[l], e = level_start[l + 1];
    if (e > b) k_layout_place<<<grid_for(e - b, 256, dev), 256, 0, st>>>(s.d_nodes, b, e, desc.p, pos.p, base.p);
  }
  k_layout_scatter<<<grid_for(n, 256, dev), 256, 0, st>>>(s.d_nodes, n, pos.p, base.p, out.p);
  XYZ_BUILD_TRY(cudaGetLastError());
  XYZ_BUILD_TRY(cudaFreeAsync(s.d_nodes, st));
  s.d_nodes = out.release();
  XYZ_BUILD_TRY(cudaStreamSynchronize(st));
  return XYZGPU_OK;
}

}  // namespace xyzgpu
