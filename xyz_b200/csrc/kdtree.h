// Flattened kd-tree shared by the host builder, the device builder and the
// traversal kernels.
//
// The reference keeps a heap tree of virtual KDNode / KDLeaf / KDNull objects
// (xyz/geom/kdtree.cpp:20-177).  Here every node is 8 bytes, two uint32 words:
//   interior: w0 = split position (float bits)
//             w1 = (first_child << 2) | axis        axis in {0, 1, 2}
//             children are adjacent: first_child = below (lower coordinates),
//             first_child + 1 = above
//   leaf:     w0 = index of the leaf's first entry in the reference array
//             w1 = (count << 2) | 3                 count 0 = empty leaf
// Nodes are numbered breadth first, so the top levels form a prefix of the
// array.  A triangle that straddles a split plane is referenced from both
// sides, as in the reference (kdtree.cpp:323-339).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace xyzgpu {

constexpr uint32_t kKdLeafTag = 3u;
constexpr int kKdMaxDepthLimit = 60;  // traversal stack holds this many entries
constexpr int kKdMaxBins = 64;

#ifdef __CUDACC__
#define XYZ_KD_HD __host__ __device__
#else
#define XYZ_KD_HD
#endif

// SAH bins per axis for a node of n references: the configured count, fewer
// for small nodes (twice the references, at least 16), whose few references
// leave most of 64 bins empty.  The host and the device builder use the same
// rule, so their trees are identical.
inline XYZ_KD_HD int kd_node_bins(int bins, int64_t n) {
  int64_t const want = n * 2 < 16 ? 16 : n * 2;
  return want < bins ? static_cast<int>(want) : bins;
}

struct BuildConfig {
  int leaf_max_tris = 4;
  int max_depth = 0;  // resolved before building
  float cost_traversal = 1.0f;
  float cost_intersect = 1.5f;
  float empty_bonus = 0.2f;
  int bins = 32;
  int64_t max_refs = 0;  // resolved before building
};

struct KdTreeHost {
  std::vector<uint32_t> nodes;  // 2 words per node
  std::vector<int32_t> refs;
  float bmin[3], bmax[3];
  int depth = 0;
  int64_t leaves = 0, empty_leaves = 0;
};

// Root box of the tree: the triangles' bounds (v0, v0 + e1, v0 + e2 per
// triangle, the vertices exactly as the intersection test sees them), grown by
// 1e-5 of the extent (plus a tiny absolute margin) on both sides.
void kd_root_bounds(const float *tri_v, int n, float bmin[3], float bmax[3]);

// Binned-SAH kd-tree on the host.  tri_v: 9 floats per triangle (v0, v1, v2
// with v1 = v0 + e1, v2 = v0 + e2 evaluated in float).  The device builder
// implements the same algorithm level by level and produces the same tree.
bool kd_build_host(const float *tri_v, int n, const BuildConfig &cfg, KdTreeHost *out,
                   std::string *err);

int kd_resolve_max_depth(int requested, int n_triangles);

}  // namespace xyzgpu
