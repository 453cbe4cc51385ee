// Host implementation of the binned-SAH kd-tree build.  It is the
// specification of the device builder (kdbuild.cu), which performs the same
// float operations in the same order level by level, so both produce the
// identical flattened tree.
//
// Relation to the reference (xyz/geom/kdtree.cpp:207-357): the reference sweeps
// sorted open/close events of each node's triangle bounds on three axes and
// splits where n_l*SA_l + n_r*SA_r is smallest, until a node holds <= 16
// triangles or is deeper than 16; straddling triangles go to both children.
// This builder keeps the structure (axis-aligned planes, straddlers on both
// sides, one split per node) but evaluates the SAH with traversal and
// intersection constants on B bins per axis, clips each reference's bounds to
// its node, and stops on the SAH leaf test, the leaf size or the depth limit.
// Closest-hit results do not depend on the tree.
#include <algorithm>
#include <cmath>
#include <cstring>

#include "kdtree.h"

namespace xyzgpu {

int kd_resolve_max_depth(int requested, int n) {
  if (requested > 0) return std::min(requested, kKdMaxDepthLimit);
  double const d = 8.0 + 1.3 * std::log2(std::max(1, n));
  return std::min(kKdMaxDepthLimit, static_cast<int>(d));
}

void kd_root_bounds(const float *tri_v, int n, float bmin[3], float bmax[3]) {
  for (int k = 0; k < 3; ++k) {
    bmin[k] = INFINITY;
    bmax[k] = -INFINITY;
  }
  for (int i = 0; i < n; ++i) {
    for (int v = 0; v < 3; ++v) {
      for (int k = 0; k < 3; ++k) {
        float const x = tri_v[9 * i + 3 * v + k];
        if (x < bmin[k]) bmin[k] = x;
        if (x > bmax[k]) bmax[k] = x;
      }
    }
  }
  for (int k = 0; k < 3; ++k) {
    if (n == 0) {
      bmin[k] = bmax[k] = 0.0f;
    }
    float const ext = bmax[k] - bmin[k];
    float const pad = ext * 1e-5f + 1e-6f;
    bmin[k] = bmin[k] - pad;
    bmax[k] = bmax[k] + pad;
  }
}

namespace {

struct Box {
  float lo[3], hi[3];
};

struct LevelNode {
  Box bounds;
  int64_t ref_begin, ref_count;
};

struct SplitChoice {
  int axis;    // -1: leaf
  float plane;
  int64_t n_left, n_right;
};

inline float half_area(const float e[3]) { return e[0] * e[1] + e[1] * e[2] + e[2] * e[0]; }

// Best binned-SAH split of one node (same arithmetic as the device kernel).
SplitChoice choose_split(const LevelNode &nd, const Box *boxes, const BuildConfig &cfg,
                         int depth) {
  SplitChoice best{-1, 0.0f, 0, 0};
  int64_t const n = nd.ref_count;
  if (n <= cfg.leaf_max_tris || depth >= cfg.max_depth) return best;
  float ext[3];
  for (int k = 0; k < 3; ++k) ext[k] = nd.bounds.hi[k] - nd.bounds.lo[k];
  float const sa = half_area(ext);
  if (!(sa > 0.0f)) return best;
  int const B = kd_node_bins(cfg.bins, n);
  float best_cost = cfg.cost_intersect * static_cast<float>(n);
  uint32_t start[kKdMaxBins], end[kKdMaxBins];
  for (int a = 0; a < 3; ++a) {
    if (!(ext[a] > 0.0f)) continue;
    std::memset(start, 0, sizeof(start));
    std::memset(end, 0, sizeof(end));
    float const scale = static_cast<float>(B) / ext[a];
    float const lo = nd.bounds.lo[a];
    for (int64_t r = nd.ref_begin; r < nd.ref_begin + n; ++r) {
      int b0 = static_cast<int>((boxes[r].lo[a] - lo) * scale);
      int b1 = static_cast<int>((boxes[r].hi[a] - lo) * scale);
      b0 = std::min(std::max(b0, 0), B - 1);
      b1 = std::min(std::max(b1, 0), B - 1);
      start[b0]++;
      end[b1]++;
    }
    float const step = ext[a] / static_cast<float>(B);
    int64_t nl = 0, ended = 0;
    for (int i = 1; i < B; ++i) {
      nl += start[i - 1];
      ended += end[i - 1];
      int64_t const nr = n - ended;
      float const plane = lo + static_cast<float>(i) * step;
      float el[3] = {ext[0], ext[1], ext[2]};
      float er[3] = {ext[0], ext[1], ext[2]};
      el[a] = plane - lo;
      er[a] = nd.bounds.hi[a] - plane;
      float const sal = half_area(el);
      float const sar = half_area(er);
      float cost = cfg.cost_traversal +
                   cfg.cost_intersect * (sal * static_cast<float>(nl) + sar * static_cast<float>(nr)) / sa;
      if (nl == 0 || nr == 0) cost = cost * (1.0f - cfg.empty_bonus);
      if (cost < best_cost) {
        best_cost = cost;
        best.axis = a;
        best.plane = plane;
        best.n_left = nl;
        best.n_right = nr;
      }
    }
  }
  return best;
}

// Which sides of `plane` a clipped reference box goes to.
inline void classify(const Box &b, int a, float plane, bool *l, bool *r) {
  bool const flat_on = (b.lo[a] == plane) && (b.hi[a] == plane);
  *l = (b.lo[a] < plane) || flat_on;
  *r = (b.hi[a] > plane) || flat_on;
}

}  // namespace

bool kd_build_host(const float *tri_v, int n, const BuildConfig &cfg_in, KdTreeHost *out,
                   std::string *err) {
  BuildConfig cfg = cfg_in;
  if (cfg.bins < 2 || cfg.bins > kKdMaxBins) {
    *err = "bins must be in [2, 64]";
    return false;
  }
  cfg.max_depth = kd_resolve_max_depth(cfg.max_depth, n);
  if (cfg.max_refs <= 0) cfg.max_refs = static_cast<int64_t>(n) * 6 + 1024;

  kd_root_bounds(tri_v, n, out->bmin, out->bmax);
  out->nodes.clear();
  out->refs.clear();
  out->leaves = out->empty_leaves = 0;
  out->depth = 0;

  std::vector<int32_t> tri(n);
  std::vector<Box> box(n);
  for (int i = 0; i < n; ++i) {
    tri[i] = i;
    for (int k = 0; k < 3; ++k) {
      float const a = tri_v[9 * i + k], b = tri_v[9 * i + 3 + k], c = tri_v[9 * i + 6 + k];
      box[i].lo[k] = std::min(std::min(a, b), c);
      box[i].hi[k] = std::max(std::max(a, b), c);
    }
  }
  std::vector<LevelNode> level(1);
  for (int k = 0; k < 3; ++k) {
    level[0].bounds.lo[k] = out->bmin[k];
    level[0].bounds.hi[k] = out->bmax[k];
  }
  level[0].ref_begin = 0;
  level[0].ref_count = n;
  out->nodes.resize(2);

  int64_t level_base = 0;
  for (int depth = 0; !level.empty(); ++depth) {
    out->depth = depth;
    size_t const m = level.size();
    std::vector<SplitChoice> ch(m);
    int64_t next_refs = 0;
    for (size_t j = 0; j < m; ++j) {
      ch[j] = choose_split(level[j], box.data(), cfg, depth);
      if (ch[j].axis >= 0) {
        // exact counts follow the partition below; the binned counts bound them
        int64_t nl = 0, nr = 0;
        for (int64_t r = level[j].ref_begin; r < level[j].ref_begin + level[j].ref_count; ++r) {
          bool l, rr;
          classify(box[r], ch[j].axis, ch[j].plane, &l, &rr);
          nl += l;
          nr += rr;
        }
        ch[j].n_left = nl;
        ch[j].n_right = nr;
        next_refs += nl + nr;
      }
    }
    if (next_refs > cfg.max_refs) {
      for (auto &c : ch) c.axis = -1;  // reference budget exhausted: this level ends the tree
      next_refs = 0;
    }
    int64_t const next_base = level_base + static_cast<int64_t>(m);
    std::vector<LevelNode> next;
    std::vector<int32_t> ntri;
    std::vector<Box> nbox;
    ntri.reserve(next_refs);
    nbox.reserve(next_refs);
    int64_t n_split = 0;
    for (size_t j = 0; j < m; ++j) {
      LevelNode const &nd = level[j];
      uint32_t *w = &out->nodes[2 * (level_base + j)];
      if (ch[j].axis < 0) {
        w[0] = static_cast<uint32_t>(out->refs.size());
        w[1] = (static_cast<uint32_t>(nd.ref_count) << 2) | kKdLeafTag;
        out->leaves++;
        if (nd.ref_count == 0) out->empty_leaves++;
        for (int64_t r = nd.ref_begin; r < nd.ref_begin + nd.ref_count; ++r) out->refs.push_back(tri[r]);
        continue;
      }
      int const a = ch[j].axis;
      float const p = ch[j].plane;
      int64_t const child = next_base + 2 * n_split;
      ++n_split;
      std::memcpy(&w[0], &p, 4);
      w[1] = (static_cast<uint32_t>(child) << 2) | static_cast<uint32_t>(a);
      LevelNode left, right;
      left.bounds = nd.bounds;
      right.bounds = nd.bounds;
      left.bounds.hi[a] = p;
      right.bounds.lo[a] = p;
      left.ref_begin = static_cast<int64_t>(ntri.size());
      for (int64_t r = nd.ref_begin; r < nd.ref_begin + nd.ref_count; ++r) {
        bool l, rr;
        classify(box[r], a, p, &l, &rr);
        if (l) {
          Box b = box[r];
          b.hi[a] = std::min(b.hi[a], p);
          ntri.push_back(tri[r]);
          nbox.push_back(b);
        }
      }
      left.ref_count = static_cast<int64_t>(ntri.size()) - left.ref_begin;
      right.ref_begin = static_cast<int64_t>(ntri.size());
      for (int64_t r = nd.ref_begin; r < nd.ref_begin + nd.ref_count; ++r) {
        bool l, rr;
        classify(box[r], a, p, &l, &rr);
        if (rr) {
          Box b = box[r];
          b.lo[a] = std::max(b.lo[a], p);
          ntri.push_back(tri[r]);
          nbox.push_back(b);
        }
      }
      right.ref_count = static_cast<int64_t>(ntri.size()) - right.ref_begin;
      next.push_back(left);
      next.push_back(right);
    }
    if (static_cast<uint64_t>(next_base + 2 * n_split) >= (1ull << 30)) {
      *err = "kd-tree node count exceeds 2^30";
      return false;
    }
    out->nodes.resize(2 * (next_base + 2 * n_split));
    level.swap(next);
    tri.swap(ntri);
    box.swap(nbox);
    level_base = next_base;
  }
  return true;
}

}  // namespace xyzgpu
