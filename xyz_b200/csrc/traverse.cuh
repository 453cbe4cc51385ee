// kd-tree closest-hit traversal for one ray (device).
//
// Semantics of the reference (xyz/geom/kdtree.cpp:82-150, 366-372):
//   * at an interior node, the plane distance e splits [t_min, t_max]; the near
//     child is the side holding the origin; e > t_max or e < 0 -> near only,
//     e < t_min -> far only, otherwise near on [t_min, e] then far on
//     [e, t_max];
//   * a leaf tests all its triangles with the double-faced Moller-Trumbore test
//     (xyz/geom/triangle.cpp:127-165): |det| < 1e-6 rejects, t must lie in the
//     interval (inclusive), barycentrics f, g >= 0 and f + g <= 1; an accepted
//     hit shrinks t_max, so among equal t the later triangle of a leaf wins;
//   * traversal stops at the first leaf (front to back) that produced a hit.
// Differences, all of which leave the closest hit unchanged: the ray is first
// clipped to the scene box, and triangles are tested against the ray's whole
// remaining interval [t_min, best_t] rather than the node's clipped interval,
// stopping once best_t <= the leaf's exit distance (robust to a hit that
// rounds across a split plane).  The plane distance uses a precomputed
// reciprocal of the direction.  A ray that starts exactly on a split plane
// continues on the side its direction points to.
#pragma once

#include <type_traits>

#include "common.cuh"

namespace xyzgpu {

struct TraceCount {
  uint32_t nodes, leaves, tris;
};

struct RayHit {
  float t, f, g;
  int32_t id;    // triangle id, -1 = miss
  int32_t back;  // 1 = hit from the back side (det > 0)
};

// FindIntersectionDF on a packed triangle; updates best_t on acceptance.
XYZ_DEV bool hit_triangle(const float4 *__restrict__ tri, int32_t i, f3 o, f3 d, float tmin,
                          RayHit &h) {
  float4 const a = __ldg(&tri[3 * i + 0]);
  float4 const b = __ldg(&tri[3 * i + 1]);
  float4 const c = __ldg(&tri[3 * i + 2]);
  f3 const e2xe1 = mk3(a.w, b.w, c.w);
  float const det = dot3(d, e2xe1);
  if (fabsf(det) < kEpsilon) return false;
  float const inv_det = __frcp_rn(det);
  f3 const vmo = sub3(xyz3(a), o);
  float const t = inv_det * dot3(vmo, e2xe1);
  if ((t < tmin) || (h.t < t)) return false;
  f3 const dxvmo = cross3(d, vmo);
  float const f = inv_det * dot3(xyz3(c), dxvmo);
  if ((f < 0.0f) || (f > 1.0f)) return false;
  float const g = inv_det * -dot3(xyz3(b), dxvmo);
  if ((g < 0.0f) || ((f + g) > 1.0f)) return false;
  h.t = t;
  h.f = f;
  h.g = g;
  h.id = i;
  h.back = det > 0.0f;
  return true;
}

// A deferred far child: its node and exit distance.  Its entry distance is
// not stored: in front-to-back order the far child pushed last is popped
// right after the subtree that ends at its split plane, so the entry equals
// the exit distance of the leaf just finished (8 bytes per entry keep the
// local-memory stack small; it competes with node fetches for L1).
struct __align__(8) StackEntry {
  uint32_t node;
  float tf;
};

// Persistent closest-hit loop over rays [0, n) taken from a shared work
// counter, with per-lane refill: after every leaf visit the lanes whose ray
// has finished are counted with a ballot; once enough are idle, one atomicAdd
// by the first of them fetches that many new rays, and each takes its index
// from a popcount of the lanes below it.  A lane therefore never idles while its warp finishes long
// rays, which keeps the warp's lanes busy on incoherent secondary and shadow
// rays (the warp-per-batch scheme leaves most lanes waiting for the slowest
// ray of the batch).  Every lane of the warp must call this.
//   Sink::load(i, o, d, tmin, tmax)   ray i
//   Sink::store(i, hit)               result of ray i
//   Sink::scene(i)                    (kBatch) the scene of ray i; rays of one
//                                     queue may belong to different scenes
//   Sink::target(i)                   (sinks with kTarget) the triangle whose
//                                     being the closest hit is the only
//                                     question the caller asks (next-event
//                                     estimation's visibility test,
//                                     xyz/bsdf/lambert.cpp:151-155)
//
// Target queries end early, with the same answer the full closest-hit search
// gives: the target's own hit distance t_own is computed first, with the
// same arithmetic the traversal would apply to it.  If the target is not hit
// at all, it cannot be the closest hit and the ray needs no traversal.  Once
// any triangle is accepted at t < t_own, the final closest hit has t < t_own
// too, so it is not the target whatever the remaining nodes hold, and the ray
// stops (the store then sees a non-target id).  Nothing else changes: the
// target itself and hits at t >= t_own go through the unchanged closest-hit
// rules, so ties and rounding across split planes resolve as before.
constexpr int kRefillIdle = 12;

template <class S, class = void>
struct SinkHasTarget : std::false_type {};
template <class S>
struct SinkHasTarget<S, std::void_t<decltype(S::kTarget)>> : std::bool_constant<S::kTarget> {};
// One iteration of the persistent loop descends at most this many nodes; a lane
// still above its next leaf resumes there in the next iteration, so the warp's
// leaf tests do not wait for its longest descent (counting renders descend
// without the cap).
#ifndef XYZ_DESCEND_STEPS
#define XYZ_DESCEND_STEPS 8
#endif
constexpr int kDescendSteps = XYZ_DESCEND_STEPS;

template <bool kCount, bool kBatch = false, class Sink>
XYZ_DEV void trace_persistent(const DevScene &S, int n, int *fetch, Sink &sink, TraceCount &tc) {
  constexpr bool kTarget = SinkHasTarget<Sink>::value;
  int const lane = threadIdx.x & 31;
  unsigned const lanes_below = (1u << lane) - 1u;
  int ray = -1;
  bool exhausted = false;
  f3 o{}, d{};
  float inv[3] = {0.0f, 0.0f, 0.0f};
  float tmin = 0.0f;
  RayHit h{};
  float stop_t = 0.0f;  // target queries: the target's own hit distance
  uint32_t node = 0;
  float tn = 0.0f, tf = 0.0f;
  int sp = 0;
  StackEntry stack[kKdMaxDepthLimit];
  const DevScene *lane_scene = &S;
  for (;;) {
    bool const need = ray < 0 && !exhausted;
    // refill once at least kRefillIdle lanes are idle: refilling after every
    // finished ray costs more than it gains (measured on B200: 8..20 idle lanes
    // is best, 1 and 32 are 10 % slower)
    unsigned const idle = __ballot_sync(0xffffffffu, ray < 0);
    unsigned const want = (__popc(idle) >= kRefillIdle) ? __ballot_sync(0xffffffffu, need) : 0u;
    if (want) {
      int const leader = __ffs(want) - 1;
      int base = 0;
      if (lane == leader) base = atomicAdd(fetch, __popc(want));
      base = __shfl_sync(0xffffffffu, base, leader);
      if (need) {
        int const i = base + __popc(want & lanes_below);
        if (i >= n) {
          exhausted = true;
        } else {
          float tmax;
          sink.load(i, o, d, tmin, tmax);
          if constexpr (kBatch) lane_scene = sink.scene(i);
          const DevScene &SL = kBatch ? *lane_scene : S;
          h.t = tmax;
          h.id = -1;
          h.f = h.g = 0.0f;
          h.back = 0;
          bool skip = false;
          if constexpr (kTarget) {
            RayHit own = h;
            skip = !hit_triangle(SL.tri, sink.target(i), o, d, tmin, own);
            stop_t = own.t;
            if (kCount) tc.tris++;
          }
          inv[0] = __frcp_rn(d.x);
          inv[1] = __frcp_rn(d.y);
          inv[2] = __frcp_rn(d.z);
          float const org[3] = {o.x, o.y, o.z};
          float const lo[3] = {SL.bmin.x, SL.bmin.y, SL.bmin.z};
          float const hi[3] = {SL.bmax.x, SL.bmax.y, SL.bmax.z};
          float t0 = tmin, t1 = tmax;
#pragma unroll
          for (int k = 0; k < 3; ++k) {
            float const ta = (lo[k] - org[k]) * inv[k];
            float const tb = (hi[k] - org[k]) * inv[k];
            t0 = fmaxf(t0, fminf(ta, tb));
            t1 = fminf(t1, fmaxf(ta, tb));
          }
          if (skip) {
            // the target is not hit: the answer is "not the target" (h.id = -1)
            sink.store(i, h);
          } else if (!(t0 <= t1)) {
            sink.store(i, h);  // misses the scene box
          } else {
            ray = i;
            node = 0;
            tn = t0;
            tf = t1;
            sp = 0;
          }
        }
      }
    }
    if (__all_sync(0xffffffffu, exhausted && ray < 0)) break;
    if (ray < 0) continue;
    const uint2 *__restrict__ nodes = kBatch ? lane_scene->nodes : S.nodes;
    // descend to a leaf
    uint2 nd = __ldg(&nodes[node]);
    if (kCount) tc.nodes++;
    int steps = 0;
    while ((nd.y & 3u) != kKdLeafTag && (kCount || steps < kDescendSteps)) {
      ++steps;
      uint32_t const ax = nd.y & 3u;
      float const split = __uint_as_float(nd.x);
      uint32_t const child = nd.y >> 2;
      float const oa = ax == 0 ? o.x : (ax == 1 ? o.y : o.z);
      float const ia = ax == 0 ? inv[0] : (ax == 1 ? inv[1] : inv[2]);
      float const da = ax == 0 ? d.x : (ax == 1 ? d.y : d.z);
      float const tp = (split - oa) * ia;
      uint32_t const above_first = (oa < split || (oa == split && da <= 0.0f)) ? 0u : 1u;
      uint32_t const first = child + above_first;
      uint32_t const second = child + (above_first ^ 1u);
      if ((tp > tf) || (tp <= 0.0f)) {
        node = first;
      } else if (tp < tn) {
        node = second;
      } else {
        stack[sp] = StackEntry{second, tf};
        ++sp;
        node = first;
        tf = tp;
      }
      nd = __ldg(&nodes[node]);
      if (kCount) tc.nodes++;
    }
    if ((nd.y & 3u) != kKdLeafTag) continue;  // resumes at `node` in the next iteration
    // test the leaf
    uint32_t const cnt = nd.y >> 2;
    if (kCount) {
      tc.leaves++;
      tc.tris += cnt;
    }
    const int32_t *__restrict__ refs = kBatch ? lane_scene->refs : S.refs;
    const float4 *__restrict__ tris = kBatch ? lane_scene->tri : S.tri;
    int32_t t_next = cnt > 0 ? __ldg(&refs[nd.x]) : 0;
    for (uint32_t j = 0; j < cnt; ++j) {
      int32_t const t = t_next;
      if (j + 1 < cnt) t_next = __ldg(&refs[nd.x + j + 1]);
      hit_triangle(tris, t, o, d, tmin, h);
      if (kTarget && h.t < stop_t) break;
    }
    // next leaf (entered at this leaf's exit), or done
    bool const done = (h.id >= 0 && h.t <= tf) || sp == 0 || (kTarget && h.t < stop_t);
    if (!done) {
      --sp;
      StackEntry const e = stack[sp];
      node = e.node;
      tn = tf;
      tf = e.tf;
    }
    if (done) {
      sink.store(ray, h);
      ray = -1;
    }
  }
}

}  // namespace xyzgpu
