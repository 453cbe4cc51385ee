// Wavefront path tracer: xyzgpu_render.
//
// One call renders spp samples of every pixel.  Paths are processed in waves of
// up to `capacity` paths (sample-major: slot = s_local * n_pixels + p_local), and
// a wave runs a fixed sequence of kernels over SoA queues in HBM:
//
//   raygen                      camera rays of every path of the wave
//   repeat max_depth times:
//     trace (extension queue)   closest hit of each live path's ray
//     shade                     one vertex of Scene::EvalutePathTracing
//                               (xyz/core/scene_pathtracing.cpp:46-143):
//                               shading basis, emitter hit with MIS, depth cap,
//                               next-event estimation (-> shadow queue),
//                               Russian roulette, Lambert sampling
//                               (-> next extension queue)
//     trace (shadow queue)      closest hit from the light point; the vertex
//                               receives the NEE term if that hit is its own
//                               triangle (xyz/bsdf/lambert.cpp:151-172)
//   film                        film[p] += path radiance, samples in order
//
// Queue lengths live in device memory, so the host issues the whole sequence
// without synchronising; kernels whose queue is empty return at once.
// Queue appends are compacted per warp: a ballot over the lanes that append,
// one atomicAdd by the first of them, and each lane's offset from a popcount of
// the lanes below it.
//
// Every path reads its own Philox stream (include/xyzgpu.h), so the result does
// not depend on the wave size or on the order in which queues are filled.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "scene.h"
#include "spectral.h"
#include "traverse.cuh"

namespace xyzgpu {
namespace {

constexpr int kThreads = 128;
constexpr int kCountStride = 8;  // int32 counters per iteration
// per-iteration counter slots
constexpr int kCExt = 0;        // extension rays entering iteration b
constexpr int kCShadow = 1;     // shadow rays produced in iteration b
constexpr int kCFetchExt = 2;   // work counter of the extension trace
constexpr int kCFetchSh = 3;    // work counter of the shadow trace
constexpr int kCVisible = 4;    // shadow rays that reached their vertex

struct CamDev {
  f3 eye, right, up, back;
  float film, aspect, L, V, R;
  int pinhole;
};

struct WaveArgs {
  DevScene S;
  CamDev cam;
  int W, H;
  int kmax;         // the reference's kMax = max_depth + 1
  int rr_start;
  float rr_threshold;
  uint64_t seed;
  int64_t p0;       // first pixel of the wave
  int64_t npix;     // pixels in the wave
  uint32_t s0;      // first sample index of the wave
  int nsamp;        // samples per pixel in the wave
  int64_t npaths;   // npix * nsamp
  float4 *beta;
  uint32_t *misc;
  float4 *radiance;
  float4 *q_o[2];
  float4 *q_d[2];
  int32_t *q_slot[2];
  float4 *hits;
  float4 *s_o, *s_d, *s_pb;
  int32_t *s_target;
  int32_t *counts;
  // spectral modes (XYZGPU_SPECTRAL_*): beta and radiance hold one channel per
  // hero wavelength, fSamplingNext moves to `fsn` and the shadow slot to `s_slot`
  int spectral, hero;
  uint32_t wl_dim;  // dimension of the hero wavelength draw
  float *fsn;
  int32_t *s_slot;
  // path-replay adjoint (xyzgpu_adjoint): each path's radiance from the primal
  // pass, dLoss/dfilm, and the gradient accumulators
  float4 *ltot;
  const float *dfilm;
  float *g_alb;
  float *g_em;
};

XYZ_DEV uint32_t pack_misc(uint32_t dim, uint32_t k, uint32_t specular) {
  return (dim & 0xffffu) | ((k & 0x7fffu) << 16) | (specular << 31);
}

XYZ_DEV void slot_to_pixel_sample(const WaveArgs &A, int64_t slot, uint32_t *pixel,
                                  uint32_t *sample) {
  int64_t const sl = slot / A.npix;
  int64_t const pl = slot - sl * A.npix;
  *pixel = static_cast<uint32_t>(A.p0 + pl);
  *sample = A.s0 + static_cast<uint32_t>(sl);
}

// Warp-aggregated append: returns this lane's index in the queue (valid when
// `want`).  All 32 lanes must call it.
XYZ_DEV int32_t warp_append(int32_t *counter, bool want) {
  unsigned const m = __ballot_sync(0xffffffffu, want);
  if (m == 0u) return -1;
  int const lane = threadIdx.x & 31;
  int const leader = __ffs(m) - 1;
  int32_t base = 0;
  if (lane == leader) base = atomicAdd(counter, __popc(m));
  base = __shfl_sync(0xffffffffu, base, leader);
  return base + __popc(m & ((1u << lane) - 1u));
}

// ------------------------------------------------------------------ raygen
// Scene::EvalutePathTracing lines 14-38 and the pixel jitter of
// PathTracer::run (integrator.cpp:124-125); camera rays per
// ThinLensCamera::GetPrimaryRay* (thinlenscamera.cpp:111-124, 159-205).
__global__ void __launch_bounds__(kThreads) k_raygen(WaveArgs A) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; slot < A.npaths;
       slot += stride) {
    uint32_t pixel, sample;
    slot_to_pixel_sample(A, slot, &pixel, &sample);
    uint32_t w[4];
    philox4x32_10(pixel, sample, 0u, 0u, static_cast<uint32_t>(A.seed),
                  static_cast<uint32_t>(A.seed >> 32), w);
    float const jx = u01_from_bits(w[0]);
    float const jy = u01_from_bits(w[1]);
    int const px = static_cast<int>(pixel % static_cast<uint32_t>(A.W));
    int const py = static_cast<int>(pixel / static_cast<uint32_t>(A.W));
    float const x = (static_cast<float>(px) + jx) / static_cast<float>(A.W);
    float const y = (static_cast<float>(py) + jy) / static_cast<float>(A.H);
    CamDev const &C = A.cam;
    f3 o, d;
    uint32_t dim;
    if (C.pinhole) {
      o = C.eye;
      float const lx = static_cast<float>((static_cast<double>(x) - 0.5) * static_cast<double>(C.film) *
                                          static_cast<double>(C.aspect));
      float const ly = static_cast<float>((static_cast<double>(y) - 0.5) * static_cast<double>(C.film));
      float const lz = -C.V;
      d = normalize3(add3(add3(scl3(C.right, lx), scl3(C.up, ly)), scl3(C.back, lz)));
      dim = 4;
    } else {
      uint32_t w2[4];
      philox4x32_10(pixel, sample, 1u, 0u, static_cast<uint32_t>(A.seed),
                    static_cast<uint32_t>(A.seed >> 32), w2);
      // SampleLensPosition(s, t): g++ evaluates the two draws right to left,
      // so t = dimension 4 and s = dimension 5 (SampleDisk, thinlenscamera.cpp:4-15).
      float const ct = u01_from_bits(w2[0]);
      float const cs = u01_from_bits(w2[1]);
      float const radius = C.R * sqrtf(cs);
      float const ang = static_cast<float>((2.0 * kPi) * static_cast<double>(ct));
      float const lensx = radius * cosf(ang);
      float const lensy = radius * sinf(ang);
      o = add3(add3(C.eye, scl3(C.right, lensx)), scl3(C.up, lensy));
      float const fps = C.film * C.L / C.V;
      float const lx = static_cast<float>((static_cast<double>(x) - 0.5) * static_cast<double>(fps) *
                                              static_cast<double>(C.aspect) -
                                          static_cast<double>(lensx));
      float const ly = static_cast<float>((static_cast<double>(y) - 0.5) * static_cast<double>(fps) -
                                          static_cast<double>(lensy));
      float const lz = -C.L;
      d = normalize3(add3(add3(scl3(C.right, lx), scl3(C.up, ly)), scl3(C.back, lz)));
      dim = 6;
    }
    A.q_o[0][slot] = make_float4(o.x, o.y, o.z, kRayTMin);
    A.q_d[0][slot] = make_float4(d.x, d.y, d.z, __int_as_float(0x7f800000));
    A.q_slot[0][slot] = static_cast<int32_t>(slot);
    if (A.spectral) {
      A.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, 1.0f);
      A.fsn[slot] = 0.0f;
      dim += 1;  // the hero wavelength draw follows the camera's
    } else {
      A.beta[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
    }
    A.misc[slot] = pack_misc(dim, 1u, 1u);
    A.radiance[slot] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) A.counts[kCExt] = static_cast<int32_t>(A.npaths);
}

// ------------------------------------------------------------------ trace
// Persistent warps with per-lane refill over a device-sized queue
// (trace_persistent).  kShadow: the ray starts at a light point and the
// vertex's NEE term is added when the closest hit is the vertex's own triangle.
struct ExtSink {
  const float4 *__restrict__ qo;
  const float4 *__restrict__ qd;
  float4 *__restrict__ hits;
  XYZ_DEV void load(int i, f3 &o, f3 &d, float &tmin, float &tmax) const {
    float4 const a = qo[i], b = qd[i];
    o = xyz3(a);
    d = xyz3(b);
    tmin = a.w;
    tmax = b.w;
  }
  XYZ_DEV void store(int i, const RayHit &h) {
    int32_t const code = h.id >= 0 ? ((h.id << 1) | h.back) : -1;
    hits[i] = make_float4(h.t, h.f, h.g, __int_as_float(code));
  }
};

template <bool kSpec, bool kAdj>
struct ShadowSink {
  const WaveArgs *A;
  uint32_t visible;
  XYZ_DEV void load(int i, f3 &o, f3 &d, float &tmin, float &tmax) const {
    float4 const a = A->s_o[i], b = A->s_d[i];
    o = xyz3(a);
    d = xyz3(b);
    tmin = kRayTMin;
    tmax = a.w;
  }
  XYZ_DEV void store(int i, const RayHit &h) {
    if (h.id < 0 || h.id != A->s_target[i]) return;
    // Lambert::CalculateWeightedDirectLighting, lambert.cpp:157-172
    float const G = A->s_d[i].w / (h.t * h.t);  // nk2 * nk3 / t^2
    float const dimp = static_cast<float>(kInvPi * static_cast<double>(G));
    float const dexp = 1.0f / A->S.light_area;
    float const dens = dimp / dexp;
    double const wgt = (static_cast<double>(G) * (kInvPi * kInvPi)) *
                       static_cast<double>(1.0f / (1.0f + dens * dens));
    float4 pb = A->s_pb[i];
    int32_t const slot = kSpec ? A->s_slot[i] : __float_as_int(pb.w);
    if (kAdj) {
      // replay: pb is the unit-emission power; the light's scale is applied
      // here and the unit contribution goes to that light's emission gradient
      int32_t const ml = A->s_slot[i];
      float const e = __ldg(&A->S.emission[ml]);
      uint32_t pixel, sample;
      slot_to_pixel_sample(*A, slot, &pixel, &sample);
      float const *df = A->dfilm + 3 * static_cast<int64_t>(pixel);
      float const g = df[0] * static_cast<float>(static_cast<double>(pb.x) * wgt) +
                      df[1] * static_cast<float>(static_cast<double>(pb.y) * wgt) +
                      df[2] * static_cast<float>(static_cast<double>(pb.z) * wgt);
      if (g != 0.0f) atomicAdd(&A->g_em[ml], g);
      pb.x *= e;
      pb.y *= e;
      pb.z *= e;
    }
    float4 L = A->radiance[slot];
    L.x += static_cast<float>(static_cast<double>(pb.x) * wgt);
    L.y += static_cast<float>(static_cast<double>(pb.y) * wgt);
    L.z += static_cast<float>(static_cast<double>(pb.z) * wgt);
    if (kSpec) L.w += static_cast<float>(static_cast<double>(pb.w) * wgt);
    A->radiance[slot] = L;
    ++visible;
  }
};

template <bool kShadow, bool kCount, bool kAdj = false>
__global__ void __launch_bounds__(kThreads) k_trace_queue(WaveArgs A, int b,
                                                          unsigned long long *prof) {
  int32_t *const cnt = A.counts + b * kCountStride;
  int const n = kShadow ? cnt[kCShadow] : cnt[kCExt];
  int const lane = threadIdx.x & 31;
  int const qi = b & 1;
  TraceCount tc{0u, 0u, 0u};
  uint32_t visible = 0;
  if (kShadow && kAdj) {
    ShadowSink<false, true> sink{&A, 0u};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else if (kShadow && A.spectral) {
    ShadowSink<true, false> sink{&A, 0u};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else if (kShadow) {
    ShadowSink<false, false> sink{&A, 0u};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else {
    ExtSink sink{A.q_o[qi], A.q_d[qi], A.hits};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchExt], sink, tc);
  }
  if (kShadow) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) visible += __shfl_down_sync(0xffffffffu, visible, off);
    if (lane == 0 && visible) atomicAdd(&cnt[kCVisible], static_cast<int32_t>(visible));
  }
  if (kCount) {
    unsigned long long v[3] = {tc.nodes, tc.leaves, tc.tris};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      unsigned long long x = v[k];
#pragma unroll
      for (int off = 16; off > 0; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
      if (lane == 0) atomicAdd(&prof[(kShadow ? 3 : 0) + k], x);
    }
  }
}

// Adds the wave's queue lengths to the render's running totals.
constexpr int kTallyIterBase = 16;
constexpr int kTallyWords = kTallyIterBase + 2 * XYZGPU_PROFILE_MAX_ITERS;

__global__ void k_tally(WaveArgs A, int iters, unsigned long long *tally) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  unsigned long long e = 0, sh = 0, vis = 0;
  for (int b = 0; b < iters; ++b) {
    unsigned long long const eb = A.counts[b * kCountStride + kCExt];
    unsigned long long const sb = A.counts[b * kCountStride + kCShadow];
    e += eb;
    sh += sb;
    vis += A.counts[b * kCountStride + kCVisible];
    if (b < XYZGPU_PROFILE_MAX_ITERS) {
      tally[kTallyIterBase + b] += eb;
      tally[kTallyIterBase + XYZGPU_PROFILE_MAX_ITERS + b] += sb;
    }
  }
  tally[0] += e;
  tally[1] += sh;
  tally[2] += vis;
}

// ------------------------------------------------------------------ shade
struct LightSample {
  f3 pos, sn, gn;
  int32_t mat;  // the light triangle's material
};

// Scene::SampleLightPosition + Triangle::Sample (scene.cpp:42-78,
// triangle.cpp:232-263).  g++ evaluates SampleLightPosition(next(), next())
// right to left: t = dimension 2, s = dimension 3.
XYZ_DEV LightSample sample_light(const DevScene &S, uint64_t seed, uint32_t pixel, uint32_t sample) {
  uint32_t w[4];
  philox4x32_10(pixel, sample, 0u, 0u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), w);
  float const lt = u01_from_bits(w[2]);
  float const ls = u01_from_bits(w[3]);
  float const total = __ldg(&S.cdf[S.n_lights]);
  float const u = ls * total;
  int lo = 0, hi = S.n_lights + 1;  // upper_bound over cdf[0 .. n_lights]
  while (lo < hi) {
    int const mid = (lo + hi) >> 1;
    if (!(u < __ldg(&S.cdf[mid])))
      lo = mid + 1;
    else
      hi = mid;
  }
  int const n = min(max(lo - 1, 0), S.n_lights - 1);
  float const c0 = __ldg(&S.cdf[n]), c1 = __ldg(&S.cdf[n + 1]);
  float const v = (u - c0) / (c1 - c0);
  int32_t const li = __ldg(&S.lights[n]);
  float const ss = sqrtf(v);
  float const uu = ss * (1.0f - lt);
  float const vv = ss * lt;
  float4 const a = __ldg(&S.tri[3 * li]), b = __ldg(&S.tri[3 * li + 1]), c = __ldg(&S.tri[3 * li + 2]);
  LightSample L;
  L.pos = add3(add3(xyz3(a), scl3(xyz3(b), uu)), scl3(xyz3(c), vv));
  float4 const g4 = __ldg(&S.tri_ng[li]);
  L.gn = xyz3(g4);
  L.mat = __float_as_int(g4.w);
  if (S.tri_sn) {
    f3 const n0 = xyz3(__ldg(&S.tri_sn[3 * li])), s1 = xyz3(__ldg(&S.tri_sn[3 * li + 1])),
             s2 = xyz3(__ldg(&S.tri_sn[3 * li + 2]));
    L.sn = normalize3(add3(add3(n0, scl3(s1, uu)), scl3(s2, vv)));
  } else {
    f3 const z = mk3(0.0f, 0.0f, 0.0f);
    L.sn = normalize3(add3(add3(L.gn, scl3(z, uu)), scl3(z, vv)));
  }
  return L;
}

// kAdj: the replay pass of xyzgpu_adjoint (same path, plus gradients).
template <bool kAdj>
__global__ void __launch_bounds__(kThreads) k_shade(WaveArgs A, int b) {
  int32_t *const cnt = A.counts + b * kCountStride;
  int32_t *const cnt_next = A.counts + (b + 1) * kCountStride;
  int const n = cnt[kCExt];
  int const lane = threadIdx.x & 31;
  int const qi = b & 1, qo = qi ^ 1;
  int const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int const nwarps = (gridDim.x * blockDim.x) >> 5;
  DevScene const &S = A.S;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    int const i = base + lane;
    bool push_ext = false, push_sh = false;
    int32_t slot = 0, tri = 0;
    f3 pos{}, dir{}, lpos{}, vin{}, pbv{};
    float nk2nk3 = 0.0f;
    float4 beta4{};
    uint32_t misc = 0;
    int32_t light_mat = 0;
    if (i < n) {
      slot = A.q_slot[qi][i];
      float4 const h = A.hits[i];
      int32_t const code = __float_as_int(h.w);
      if (code >= 0) {
        tri = code >> 1;
        int const back = code & 1;
        float4 const o4 = A.q_o[qi][i], d4 = A.q_d[qi][i];
        f3 const d = xyz3(d4);
        // Triangle::ShadingBasis (triangle.cpp:194-219)
        float4 const g4 = __ldg(&S.tri_ng[tri]);
        f3 gn = xyz3(g4);
        int32_t const m = __float_as_int(g4.w);
        f3 sn;
        if (S.tri_sn) {
          f3 const n0 = xyz3(__ldg(&S.tri_sn[3 * tri])), s1 = xyz3(__ldg(&S.tri_sn[3 * tri + 1])),
                   s2 = xyz3(__ldg(&S.tri_sn[3 * tri + 2]));
          sn = normalize3(add3(add3(n0, scl3(s1, h.y)), scl3(s2, h.z)));
        } else {
          f3 const z = mk3(0.0f, 0.0f, 0.0f);
          sn = normalize3(add3(add3(gn, scl3(z, h.y)), scl3(z, h.z)));
        }
        if (back) {
          gn = neg3(gn);
          sn = neg3(sn);
        }
        f3 tan = mk3(-sn.z, 0.0f, sn.x), bin;
        float const l2 = dot3(tan, tan);
        if (l2 > 0.0f) {
          tan = scl3(tan, 1.0f / sqrtf(l2));
          bin = cross3(tan, sn);
        } else {
          bin = mk3(0.0f, 0.0f, (sn.y > 0.0f) ? 1.0f : -1.0f);
          tan = cross3(sn, bin);
        }
        if (!(-dot3(d, sn) <= 0.0f)) {
          pos = add3(xyz3(o4), scl3(d, h.x));
          float4 const m4 = __ldg(&S.mat[m]);
          bool const is_light = m4.w != 0.0f;
          beta4 = A.beta[slot];
          f3 beta = xyz3(beta4);
          misc = A.misc[slot];
          uint32_t dim = misc & 0xffffu;
          uint32_t k = (misc >> 16) & 0x7fffu;
          uint32_t const specular = misc >> 31;
          bool alive = true;
          if (is_light && !back) {
            // emitter hit (scene_pathtracing.cpp:84-111); the material's
            // emission scale multiplies the light's power (1 unless set)
            f3 pb = mul3(S.power, beta);
            float const e = __ldg(&S.emission[m]);
            f3 const pb_unit = pb;
            pb = scl3(pb, e);
            double const wl = kInvPi / static_cast<double>(S.light_area);
            double mis = 1.0;
            if (!specular) {
              float const cosv = fabsf(dot3(d, sn));
              float const d2 = h.x * h.x;
              float const dimp = beta4.w * cosv / d2;
              float const dexp = 1.0f / S.light_area;
              float const dens = dexp / dimp;
              mis = static_cast<double>(1.0f / (1.0f + dens * dens));
            }
            if (kAdj) {
              double const w = specular ? wl : wl * mis;
              uint32_t px, smp;
              slot_to_pixel_sample(A, slot, &px, &smp);
              float const *df = A.dfilm + 3 * static_cast<int64_t>(px);
              float const g = df[0] * static_cast<float>(static_cast<double>(pb_unit.x) * w) +
                              df[1] * static_cast<float>(static_cast<double>(pb_unit.y) * w) +
                              df[2] * static_cast<float>(static_cast<double>(pb_unit.z) * w);
              if (g != 0.0f) atomicAdd(&A.g_em[m], g);
            }
            float4 L = A.radiance[slot];
            if (specular) {
              L.x += static_cast<float>(static_cast<double>(pb.x) * wl);
              L.y += static_cast<float>(static_cast<double>(pb.y) * wl);
              L.z += static_cast<float>(static_cast<double>(pb.z) * wl);
            } else {
              L.x += static_cast<float>(static_cast<double>(pb.x) * wl * mis);
              L.y += static_cast<float>(static_cast<double>(pb.y) * wl * mis);
              L.z += static_cast<float>(static_cast<double>(pb.z) * wl * mis);
            }
            A.radiance[slot] = L;
            alive = false;
          }
          if (alive) {
            ++k;
            if (static_cast<int>(k) >= A.kmax) alive = false;
          }
          uint32_t pixel = 0, sample = 0;
          if (alive) {
            slot_to_pixel_sample(A, slot, &pixel, &sample);
            if (!is_light) {
              // next-event estimation (lambert.cpp:125-156)
              beta = mul3(beta, xyz3(m4));
              if (kAdj) {
                // Every contribution from here on carries this vertex's albedo
                // once: d/d albedo_c = (L_total - L_so_far)_c / albedo_c.
                float4 const lt = A.ltot[slot], lr = A.radiance[slot];
                float const *df = A.dfilm + 3 * static_cast<int64_t>(pixel);
                float const gx = df[0] * (lt.x - lr.x), gy = df[1] * (lt.y - lr.y),
                            gz = df[2] * (lt.z - lr.z);
                if (gx != 0.0f && m4.x != 0.0f) atomicAdd(&A.g_alb[3 * m], gx / m4.x);
                if (gy != 0.0f && m4.y != 0.0f) atomicAdd(&A.g_alb[3 * m + 1], gy / m4.y);
                if (gz != 0.0f && m4.z != 0.0f) atomicAdd(&A.g_alb[3 * m + 2], gz / m4.z);
              }
              if (S.n_lights > 0) {
                LightSample const ls = sample_light(S, A.seed, pixel, sample);
                f3 const v = normalize3(sub3(pos, ls.pos));
                float const nk3 = dot3(v, ls.gn);
                if (!((nk3 <= 0.0f) || (dot3(v, ls.sn) <= 0.0f))) {
                  float const nk2 = -dot3(v, sn);
                  if (!((nk2 <= 0.0f) || (-dot3(v, gn) <= 0.0f))) {
                    push_sh = true;
                    lpos = ls.pos;
                    vin = v;
                    nk2nk3 = nk2 * nk3;
                    pbv = mul3(S.power, beta);
                    light_mat = ls.mat;
                    if (!kAdj) pbv = scl3(pbv, __ldg(&S.emission[ls.mat]));
                  }
                }
              }
            }
            PathRng rng;
            rng.init(A.seed, pixel, sample, dim);
            // Russian roulette (scene_pathtracing.cpp:128-137)
            if (static_cast<int>(k) - 1 >= A.rr_start) {
              float const ty = beta.y;
              if (ty < A.rr_threshold) {
                float const q = ty / A.rr_threshold;
                if (rng.next() >= q) {
                  alive = false;
                } else {
                  beta = scl3(beta, 1.0f / q);
                }
              }
            }
            if (alive && is_light) alive = false;  // Light::NextScatteringDirection
            if (alive) {
              // Lambert::NextScatteringDirection / ComputeDiffusedVector
              // (lambert.cpp:176-187, stdafx.hpp:50-63); g++ passes the first
              // draw to fMuPhi and the second to fMuTheta.
              float const mu_phi = rng.next();
              float const mu_theta = rng.next();
              float const phi = static_cast<float>(2.0 * kPi) * mu_phi;
              float const cos_t = sqrtf(mu_theta);
              float const sin_t = sqrtf(1.0f - mu_theta);
              dir = add3(add3(scl3(tan, sin_t * cosf(phi)), scl3(bin, sin_t * sinf(phi))),
                         scl3(sn, cos_t));
              float const fsn = static_cast<float>(kInvPi * static_cast<double>(cos_t));
              if (dot3(dir, gn) > 0.0f) {
                push_ext = true;
                beta4 = make_float4(beta.x, beta.y, beta.z, fsn);
                misc = pack_misc(rng.dim, k, 0u);
              }
            }
          }
        }
      }
    }
    int32_t const js = warp_append(&cnt[kCShadow], push_sh);
    if (push_sh) {
      A.s_o[js] = make_float4(lpos.x, lpos.y, lpos.z, __int_as_float(0x7f800000));
      A.s_d[js] = make_float4(vin.x, vin.y, vin.z, nk2nk3);
      A.s_pb[js] = make_float4(pbv.x, pbv.y, pbv.z, __int_as_float(slot));
      A.s_target[js] = tri;
      if (kAdj) A.s_slot[js] = light_mat;
    }
    int32_t const je = warp_append(&cnt_next[kCExt], push_ext);
    if (push_ext) {
      A.q_o[qo][je] = make_float4(pos.x, pos.y, pos.z, kRayTMin);
      A.q_d[qo][je] = make_float4(dir.x, dir.y, dir.z, __int_as_float(0x7f800000));
      A.q_slot[qo][je] = slot;
      A.beta[slot] = beta4;
      A.misc[slot] = misc;
    }
  }
}


// ------------------------------------------------------------ spectral shade
// One vertex of the reference's spectral estimator, tgir::Scene::
// EvaluteRussianRoulette (renderer/core/SceneStrategy.cpp:60-145), for H hero
// wavelengths: the geometry is the XYZ kernel's; the throughput, emitted power
// and albedo are per wavelength; next-event estimation comes before the depth
// cap and Russian roulette looks at the first wavelength's throughput, as in
// that estimator.
struct HeroSet {
  int bin[kMaxHero];
  float p[kMaxHero];
};

XYZ_DEV HeroSet hero_set(const WaveArgs &A, uint32_t pixel, uint32_t sample) {
  uint32_t w[4];
  philox4x32_10(pixel, sample, A.wl_dim >> 2, 0u, static_cast<uint32_t>(A.seed),
                static_cast<uint32_t>(A.seed >> 32), w);
  uint32_t const j = A.wl_dim & 3u;
  float const uh = u01_from_bits(j == 0 ? w[0] : (j == 1 ? w[1] : (j == 2 ? w[2] : w[3])));
  HeroSet hs;
#pragma unroll
  for (int k = 0; k < kMaxHero; ++k) {
    float const u = hero_u(uh, k, A.hero);
    hs.bin[k] = hero_bin(u);
    hs.p[k] = hero_sample_param(u);
  }
  return hs;
}

// Value of a 31-bin spectrum at hero wavelength k.
XYZ_DEV float spd_value(const WaveArgs &A, const float *spd, const HeroSet &hs, int k) {
  if (A.spectral == XYZGPU_SPECTRAL_BINNED) return spd[hs.bin[k]];
  return spectrum_sample(hs.p[k], [&](int i) { return spd[i]; });
}

XYZ_DEV float4 spd_values(const WaveArgs &A, const float *spd, const HeroSet &hs) {
  float v[kMaxHero] = {0.0f, 0.0f, 0.0f, 0.0f};
  for (int k = 0; k < A.hero; ++k) v[k] = spd_value(A, spd, hs, k);
  return make_float4(v[0], v[1], v[2], v[3]);
}

XYZ_DEV float4 mul4(float4 a, float4 b) { return make_float4(a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w); }

__global__ void __launch_bounds__(kThreads) k_shade_spectral(WaveArgs A, int b) {
  int32_t *const cnt = A.counts + b * kCountStride;
  int32_t *const cnt_next = A.counts + (b + 1) * kCountStride;
  int const n = cnt[kCExt];
  int const lane = threadIdx.x & 31;
  int const qi = b & 1, qo = qi ^ 1;
  int const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int const nwarps = (gridDim.x * blockDim.x) >> 5;
  DevScene const &S = A.S;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    int const i = base + lane;
    bool push_ext = false, push_sh = false;
    int32_t slot = 0, tri = 0;
    f3 pos{}, dir{}, lpos{}, vin{};
    float4 pb4{}, beta{};
    float nk2nk3 = 0.0f, fsn_out = 0.0f;
    uint32_t misc = 0;
    if (i < n) {
      slot = A.q_slot[qi][i];
      float4 const h = A.hits[i];
      int32_t const code = __float_as_int(h.w);
      if (code >= 0) {
        tri = code >> 1;
        int const back = code & 1;
        float4 const o4 = A.q_o[qi][i], d4 = A.q_d[qi][i];
        f3 const d = xyz3(d4);
        float4 const g4 = __ldg(&S.tri_ng[tri]);
        f3 gn = xyz3(g4);
        int32_t const m = __float_as_int(g4.w);
        f3 sn;
        if (S.tri_sn) {
          f3 const n0 = xyz3(__ldg(&S.tri_sn[3 * tri])), s1 = xyz3(__ldg(&S.tri_sn[3 * tri + 1])),
                   s2 = xyz3(__ldg(&S.tri_sn[3 * tri + 2]));
          sn = normalize3(add3(add3(n0, scl3(s1, h.y)), scl3(s2, h.z)));
        } else {
          f3 const z = mk3(0.0f, 0.0f, 0.0f);
          sn = normalize3(add3(add3(gn, scl3(z, h.y)), scl3(z, h.z)));
        }
        if (back) {
          gn = neg3(gn);
          sn = neg3(sn);
        }
        f3 tan = mk3(-sn.z, 0.0f, sn.x), bin;
        float const l2 = dot3(tan, tan);
        if (l2 > 0.0f) {
          tan = scl3(tan, 1.0f / sqrtf(l2));
          bin = cross3(tan, sn);
        } else {
          bin = mk3(0.0f, 0.0f, (sn.y > 0.0f) ? 1.0f : -1.0f);
          tan = cross3(sn, bin);
        }
        if (!(-dot3(d, sn) <= 0.0f)) {
          pos = add3(xyz3(o4), scl3(d, h.x));
          bool const is_light = __ldg(&S.mat[m]).w != 0.0f;
          beta = A.beta[slot];
          float const fsn_in = A.fsn[slot];
          misc = A.misc[slot];
          uint32_t dim = misc & 0xffffu;
          uint32_t k = (misc >> 16) & 0x7fffu;
          uint32_t const specular = misc >> 31;
          uint32_t pixel = 0, sample = 0;
          slot_to_pixel_sample(A, slot, &pixel, &sample);
          HeroSet const hs = hero_set(A, pixel, sample);
          float4 const phi = spd_values(A, S.spd_light, hs);
          bool alive = true;
          if (is_light && !back) {
            // SceneStrategy.cpp:100-120
            float const e = __ldg(&S.emission[m]);
            float4 pb = mul4(phi, beta);
            pb = make_float4(pb.x * e, pb.y * e, pb.z * e, pb.w * e);
            double const wl = kInvPi / static_cast<double>(S.light_area);
            double mis = 1.0;
            if (!specular) {
              float const cosv = fabsf(dot3(d, sn));
              float const dimp = fsn_in * cosv / (h.x * h.x);
              float const dens = (1.0f / S.light_area) / dimp;
              mis = static_cast<double>(1.0f / (1.0f + dens * dens));
            }
            float4 L = A.radiance[slot];
            L.x += static_cast<float>(static_cast<double>(pb.x) * wl * mis);
            L.y += static_cast<float>(static_cast<double>(pb.y) * wl * mis);
            L.z += static_cast<float>(static_cast<double>(pb.z) * wl * mis);
            L.w += static_cast<float>(static_cast<double>(pb.w) * wl * mis);
            A.radiance[slot] = L;
            alive = false;
          }
          if (alive) {
            if (!is_light) {
              // next-event estimation before the depth cap (SceneStrategy.cpp:122-123,
              // renderer/bsdf/Lambert.cpp:98-137)
              float4 const alb = spd_values(A, S.spd_albedo + kSpecBins * m, hs);
              beta = mul4(beta, alb);
              if (S.n_lights > 0) {
                LightSample const ls = sample_light(S, A.seed, pixel, sample);
                f3 const v = normalize3(sub3(pos, ls.pos));
                float const nk3 = dot3(v, ls.gn);
                if (!((nk3 <= 0.0f) || (dot3(v, ls.sn) <= 0.0f))) {
                  float const nk2 = -dot3(v, sn);
                  if (!((nk2 <= 0.0f) || (-dot3(v, gn) <= 0.0f))) {
                    push_sh = true;
                    lpos = ls.pos;
                    vin = v;
                    nk2nk3 = nk2 * nk3;
                    pb4 = mul4(phi, beta);
                    float const e = __ldg(&S.emission[ls.mat]);
                    pb4 = make_float4(pb4.x * e, pb4.y * e, pb4.z * e, pb4.w * e);
                  }
                }
              }
            }
            ++k;
            if (static_cast<int>(k) >= A.kmax) alive = false;
          }
          if (alive) {
            PathRng rng;
            rng.init(A.seed, pixel, sample, dim);
            // Russian roulette on the first wavelength's throughput (SceneStrategy.cpp:131-140)
            if (static_cast<int>(k) - 1 >= A.rr_start) {
              float const t = beta.x;
              if (t < A.rr_threshold) {
                float const q = t / A.rr_threshold;
                if (rng.next() >= q) {
                  alive = false;
                } else {
                  float const r = 1.0f / q;
                  beta = make_float4(beta.x * r, beta.y * r, beta.z * r, beta.w * r);
                }
              }
            }
            if (alive && is_light) alive = false;
            if (alive) {
              float const mu_phi = rng.next();
              float const mu_theta = rng.next();
              float const ph = static_cast<float>(2.0 * kPi) * mu_phi;
              float const cos_t = sqrtf(mu_theta);
              float const sin_t = sqrtf(1.0f - mu_theta);
              dir = add3(add3(scl3(tan, sin_t * cosf(ph)), scl3(bin, sin_t * sinf(ph))), scl3(sn, cos_t));
              fsn_out = static_cast<float>(kInvPi * static_cast<double>(cos_t));
              if (dot3(dir, gn) > 0.0f) {
                push_ext = true;
                misc = pack_misc(rng.dim, k, 0u);
              }
            }
          }
        }
      }
    }
    int32_t const js = warp_append(&cnt[kCShadow], push_sh);
    if (push_sh) {
      A.s_o[js] = make_float4(lpos.x, lpos.y, lpos.z, __int_as_float(0x7f800000));
      A.s_d[js] = make_float4(vin.x, vin.y, vin.z, nk2nk3);
      A.s_pb[js] = pb4;
      A.s_slot[js] = slot;
      A.s_target[js] = tri;
    }
    int32_t const je = warp_append(&cnt_next[kCExt], push_ext);
    if (push_ext) {
      A.q_o[qo][je] = make_float4(pos.x, pos.y, pos.z, kRayTMin);
      A.q_d[qo][je] = make_float4(dir.x, dir.y, dir.z, __int_as_float(0x7f800000));
      A.q_slot[qo][je] = slot;
      A.beta[slot] = beta;
      A.fsn[slot] = fsn_out;
      A.misc[slot] = misc;
    }
  }
}

// Spectral film: XYZ of each path from its hero wavelengths, added in sample
// order.  Binned: (L_j * 31) * CMF[bin_j] as hi::spd2xyz(i, L) (spectrum.cpp:
// 561-567); continuous: (L_j * 34) * CMF(lambda_j); summed over j, then / H.
__global__ void __launch_bounds__(kThreads) k_film_spectral(WaveArgs A, float *__restrict__ film) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  float const scale = A.spectral == XYZGPU_SPECTRAL_BINNED ? static_cast<float>(kSpecBins) : 34.0f;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.npix; p += stride) {
    float *f = film + 3 * (A.p0 + p);
    float fx = f[0], fy = f[1], fz = f[2];
    for (int s = 0; s < A.nsamp; ++s) {
      int64_t const slot = static_cast<int64_t>(s) * A.npix + p;
      float4 const L4 = A.radiance[slot];
      float const L[kMaxHero] = {L4.x, L4.y, L4.z, L4.w};
      uint32_t pixel, sample;
      slot_to_pixel_sample(A, slot, &pixel, &sample);
      HeroSet const hs = hero_set(A, pixel, sample);
      float acc[3] = {0.0f, 0.0f, 0.0f};
      for (int k = 0; k < A.hero; ++k) {
        float const v = L[k] * scale;
        for (int c = 0; c < 3; ++c) {
          float const cmf = A.spectral == XYZGPU_SPECTRAL_BINNED
                                ? c_cmf[c][hs.bin[k]]
                                : spectrum_sample(hs.p[k], [&](int i) { return c_cmf[c][i]; });
          acc[c] += v * cmf;
        }
      }
      float const inv_h = static_cast<float>(A.hero);
      fx += acc[0] / inv_h;
      fy += acc[1] / inv_h;
      fz += acc[2] / inv_h;
    }
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
  }
}

// ------------------------------------------------------------------ film
// film[p] += color for each sample in increasing sample order
// (PathTracer::run, integrator.cpp:119-127).
__global__ void __launch_bounds__(kThreads) k_film(WaveArgs A, float *__restrict__ film) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t p = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; p < A.npix; p += stride) {
    float *f = film + 3 * (A.p0 + p);
    float fx = f[0], fy = f[1], fz = f[2];
    for (int s = 0; s < A.nsamp; ++s) {
      float4 const L = A.radiance[static_cast<int64_t>(s) * A.npix + p];
      fx += L.x;
      fy += L.y;
      fz += L.z;
    }
    f[0] = fx;
    f[1] = fy;
    f[2] = fz;
  }
}

// Adjoint: keeps each path's primal radiance for the replay pass.
__global__ void __launch_bounds__(kThreads) k_adj_stash(WaveArgs A) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < A.npaths; i += stride)
    A.ltot[i] = A.radiance[i];
}

template <class K>
int occupancy_grid(K kernel, int device) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess ||
      per_sm <= 0)
    per_sm = 4;
  return per_sm * sm_count(device);
}

constexpr int64_t kBytesPerPath = 3 * sizeof(float4) + sizeof(uint32_t) +  // beta, radiance, hits, misc
                                  2 * (2 * sizeof(float4) + sizeof(int32_t)) +  // extension queues
                                  3 * sizeof(float4) + sizeof(int32_t) +         // shadow queue
                                  sizeof(float) + sizeof(int32_t);               // spectral fsn, slot
constexpr int64_t kMaxDefaultWave = int64_t{1} << 26;

// Wave buffers are shared by every scene on a device: the largest wave asked
// for so far stays allocated, and renders on different streams are ordered by
// an event so that they never use the buffers at the same time.
struct SharedWaves {
  std::mutex mu;
  RenderWorkspace ws;  // only the wave buffers (beta .. counts) are used
  cudaEvent_t done = nullptr;
  cudaStream_t last = nullptr;
};

SharedWaves &shared_waves(int device) {
  static SharedWaves pool[64];
  return pool[device & 63];
}

void free_wave_buffers(RenderWorkspace &w) {
  cudaFree(w.beta);
  cudaFree(w.misc);
  cudaFree(w.radiance);
  for (int q = 0; q < 2; ++q) {
    cudaFree(w.q_o[q]);
    cudaFree(w.q_d[q]);
    cudaFree(w.q_slot[q]);
  }
  cudaFree(w.hits);
  cudaFree(w.s_o);
  cudaFree(w.s_d);
  cudaFree(w.s_pb);
  cudaFree(w.s_target);
  cudaFree(w.fsn);
  cudaFree(w.s_slot);
  cudaFree(w.counts);
  w.fsn = nullptr;
  w.s_slot = nullptr;
  w.beta = w.radiance = w.hits = w.s_o = w.s_d = w.s_pb = nullptr;
  w.misc = nullptr;
  w.q_o[0] = w.q_o[1] = w.q_d[0] = w.q_d[1] = nullptr;
  w.q_slot[0] = w.q_slot[1] = w.s_target = w.counts = nullptr;
  w.capacity = 0;
  w.max_iters = 0;
}

int ensure_wave_buffers(RenderWorkspace &w, int64_t capacity, int iters) {
  if (w.capacity >= capacity && w.max_iters >= iters) return XYZGPU_OK;
  capacity = std::max(capacity, w.capacity);
  iters = std::max(iters, w.max_iters);
  free_wave_buffers(w);
  size_t const c = static_cast<size_t>(capacity);
#define XYZ_ALLOC(ptr, bytes)                                                         \
  do {                                                                                \
    cudaError_t const e_ = cudaMalloc(reinterpret_cast<void **>(&(ptr)), (bytes));    \
    if (e_ != cudaSuccess) {                                                          \
      free_wave_buffers(w);                                                           \
      return set_error(e_ == cudaErrorMemoryAllocation ? XYZGPU_E_NOMEM : XYZGPU_E_CUDA, \
                       "render: allocating %zu bytes of wave buffers failed: %s",     \
                       static_cast<size_t>(bytes), cudaGetErrorString(e_));           \
    }                                                                                 \
  } while (0)
  XYZ_ALLOC(w.beta, c * sizeof(float4));
  XYZ_ALLOC(w.misc, c * sizeof(uint32_t));
  XYZ_ALLOC(w.radiance, c * sizeof(float4));
  for (int q = 0; q < 2; ++q) {
    XYZ_ALLOC(w.q_o[q], c * sizeof(float4));
    XYZ_ALLOC(w.q_d[q], c * sizeof(float4));
    XYZ_ALLOC(w.q_slot[q], c * sizeof(int32_t));
  }
  XYZ_ALLOC(w.hits, c * sizeof(float4));
  XYZ_ALLOC(w.s_o, c * sizeof(float4));
  XYZ_ALLOC(w.s_d, c * sizeof(float4));
  XYZ_ALLOC(w.s_pb, c * sizeof(float4));
  XYZ_ALLOC(w.s_target, c * sizeof(int32_t));
  XYZ_ALLOC(w.fsn, c * sizeof(float));
  XYZ_ALLOC(w.s_slot, c * sizeof(int32_t));
  XYZ_ALLOC(w.counts, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t));
#undef XYZ_ALLOC
  w.capacity = capacity;
  w.max_iters = iters;
  return XYZGPU_OK;
}

}  // namespace

// Frees a scene's own render state (profiling tally and events, host-film
// staging); the wave buffers belong to the device.
void render_workspace_free(RenderWorkspace &w) {
  cudaFree(w.tally);
  for (cudaEvent_t e : w.events) cudaEventDestroy(e);
  cudaFree(w.film_dev);
  cudaFreeHost(w.film_pinned);
  w = RenderWorkspace{};
}

int render_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp, float *film,
                  cudaStream_t st, const AdjointArgs *adj) {
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  int64_t const npix_total = static_cast<int64_t>(rp.width) * rp.height;
  int64_t const film_elems = 3 * npix_total;
  int const iters = rp.max_depth;

  // Camera set-up as ThinLensCamera::Reset (thinlenscamera.cpp:71-90) and
  // Scene::SetDimension (scene.hpp:226-230), in float on the host.
  CamDev C;
  C.eye = mk3(cam.eye[0], cam.eye[1], cam.eye[2]);
  f3 const at = mk3(cam.at[0], cam.at[1], cam.at[2]);
  f3 const view = sub3(C.eye, at);
  C.L = std::sqrt(dot3(view, view));
  C.V = C.L * cam.focal_length / (C.L - cam.focal_length);
  C.R = cam.focal_length / (2 * cam.f_number);
  {
    float const r = 1.0f / std::sqrt(dot3(view, view));
    C.back = scl3(view, r);
    f3 const rr = cross3(mk3(0.0f, 1.0f, 0.0f), C.back);
    float const r2 = 1.0f / std::sqrt(dot3(rr, rr));
    C.right = scl3(rr, r2);
    C.up = cross3(C.back, C.right);
  }
  C.film = cam.film_size;
  C.aspect = static_cast<float>(rp.width) / static_cast<float>(rp.height);
  C.pinhole = cam.pinhole ? 1 : 0;

  float *film_dev = film;
  RenderWorkspace &w = s.ws;
  if (!w.tally) XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&w.tally), kTallyWords * sizeof(unsigned long long)));
  SharedWaves &sw = shared_waves(s.device);
  std::lock_guard<std::mutex> lock(sw.mu);
  // Wave size: the caller's, else every path of the call (at most 2^26),
  // bounded by half of the free device memory.
  int64_t cap = rp.wave_paths;
  if (cap <= 0) {
    cap = std::min<int64_t>(kMaxDefaultWave, std::max<int64_t>(1, npix_total * rp.spp));
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
      int64_t const afford = static_cast<int64_t>((free_b / 2 + sw.ws.capacity * kBytesPerPath) / kBytesPerPath);
      cap = std::min(cap, std::max<int64_t>(afford, int64_t{1} << 20));
    }
    cap = std::max(cap, sw.ws.capacity);
  }
  if (sw.done && sw.last != st) XYZ_CUDA_TRY(cudaStreamWaitEvent(st, sw.done, 0));
  int rc = ensure_wave_buffers(sw.ws, cap, iters);
  if (rc) return rc;
  if (!sw.done) XYZ_CUDA_TRY(cudaEventCreateWithFlags(&sw.done, cudaEventDisableTiming));
  RenderWorkspace const &wv = sw.ws;
  if (!adj && rp.film_location == XYZGPU_FILM_HOST) {
    if (w.film_elems < film_elems) {
      cudaFree(w.film_dev);
      cudaFreeHost(w.film_pinned);
      w.film_dev = nullptr;
      w.film_pinned = nullptr;
      w.film_elems = 0;
      XYZ_CUDA_TRY(cudaMalloc(reinterpret_cast<void **>(&w.film_dev), film_elems * sizeof(float)));
      XYZ_CUDA_TRY(cudaMallocHost(reinterpret_cast<void **>(&w.film_pinned), film_elems * sizeof(float)));
      w.film_elems = film_elems;
    }
    film_dev = w.film_dev;
    if (rp.accumulate) {
      std::memcpy(w.film_pinned, film, film_elems * sizeof(float));
      XYZ_CUDA_TRY(cudaMemcpyAsync(film_dev, w.film_pinned, film_elems * sizeof(float),
                                   cudaMemcpyHostToDevice, st));
    }
  }
  if (!adj && !rp.accumulate) XYZ_CUDA_TRY(cudaMemsetAsync(film_dev, 0, film_elems * sizeof(float), st));
  float4 *ltot = nullptr;
  if (adj) {
    cudaError_t const e = cudaMallocAsync(reinterpret_cast<void **>(&ltot), static_cast<size_t>(cap) * sizeof(float4), st);
    if (e != cudaSuccess)
      return set_error(e == cudaErrorMemoryAllocation ? XYZGPU_E_NOMEM : XYZGPU_E_CUDA,
                       "adjoint: allocating the primal radiance of %lld paths failed: %s",
                       static_cast<long long>(cap), cudaGetErrorString(e));
  }
  // frees the adjoint's buffer on every return below
  struct FreeAsync {
    float4 *p;
    cudaStream_t st;
    ~FreeAsync() {
      if (p) cudaFreeAsync(p, st);
    }
  } ltot_guard{ltot, st};

  static int g_raygen = 0, g_trace_e = 0, g_trace_s = 0, g_shade = 0, g_film = 0, g_shade_sp = 0;
  if (!g_raygen) {
    g_raygen = occupancy_grid(k_raygen, s.device);
    g_trace_e = occupancy_grid(k_trace_queue<false, false>, s.device);
    g_trace_s = occupancy_grid(k_trace_queue<true, false>, s.device);
    g_shade = occupancy_grid(k_shade<false>, s.device);
    g_shade_sp = occupancy_grid(k_shade_spectral, s.device);
    g_film = occupancy_grid(k_film, s.device);
  }
  int const prof = rp.profile;
  bool const spectral = rp.spectral != XYZGPU_SPECTRAL_OFF;
  bool const timing = prof == XYZGPU_PROFILE_TIMING;
  bool const counting = prof == XYZGPU_PROFILE_COUNTERS;
  XYZ_CUDA_TRY(cudaMemsetAsync(w.tally, 0, kTallyWords * sizeof(unsigned long long), st));
  w.profile_iters = iters;
  s.event_class.clear();
  size_t n_ev = 0;
  // Records the start or end event of a launch of `cls` (TIMING renders).
  auto mark = [&](int cls, bool start) -> int {
    if (!timing) return XYZGPU_OK;
    if (n_ev == w.events.size()) {
      cudaEvent_t e;
      XYZ_CUDA_TRY(cudaEventCreate(&e));
      w.events.push_back(e);
    }
    XYZ_CUDA_TRY(cudaEventRecord(w.events[n_ev++], st));
    if (start) s.event_class.push_back(cls);
    return XYZGPU_OK;
  };
  unsigned long long *const pc = w.tally + 8;

  WaveArgs A;
  std::memset(&A, 0, sizeof(A));
  A.S = s.dev;
  A.cam = C;
  A.W = rp.width;
  A.H = rp.height;
  A.kmax = rp.max_depth + 1;
  A.rr_start = rp.rr_start_depth;
  A.rr_threshold = rp.rr_threshold;
  A.seed = rp.seed;
  A.beta = wv.beta;
  A.misc = wv.misc;
  A.radiance = wv.radiance;
  for (int q = 0; q < 2; ++q) {
    A.q_o[q] = wv.q_o[q];
    A.q_d[q] = wv.q_d[q];
    A.q_slot[q] = wv.q_slot[q];
  }
  A.hits = wv.hits;
  A.s_o = wv.s_o;
  A.s_d = wv.s_d;
  A.s_pb = wv.s_pb;
  A.s_target = wv.s_target;
  A.counts = wv.counts;
  A.spectral = rp.spectral;
  A.hero = spectral ? rp.hero_wavelengths : 1;
  A.wl_dim = cam.pinhole ? 4u : 6u;
  A.fsn = wv.fsn;
  A.s_slot = wv.s_slot;
  if (adj) {
    A.ltot = ltot;
    A.dfilm = adj->d_film;
    A.g_alb = adj->g_albedo;
    A.g_em = adj->g_emission;
  }

  xyzgpu_render_counters rc_out{};
  uint64_t launches = 0;
  // Wave shape: whole samples of as many pixels as fit, else pixel blocks.
  int64_t const spp_per_wave = std::max<int64_t>(1, std::min<int64_t>(rp.spp, cap / std::max<int64_t>(1, npix_total)));
  int64_t const pix_per_wave = std::min<int64_t>(npix_total, cap);
  for (int64_t s0 = 0; s0 < rp.spp; s0 += spp_per_wave) {
    int const ns = static_cast<int>(std::min<int64_t>(spp_per_wave, rp.spp - s0));
    for (int64_t p0 = 0; p0 < npix_total; p0 += pix_per_wave) {
      A.p0 = p0;
      A.npix = std::min<int64_t>(pix_per_wave, npix_total - p0);
      A.s0 = static_cast<uint32_t>(rp.spp_offset + s0);
      A.nsamp = ns;
      A.npaths = A.npix * ns;
      XYZ_CUDA_TRY(cudaMemsetAsync(wv.counts, 0, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t), st));
      int const gr = static_cast<int>(std::min<int64_t>(g_raygen, (A.npaths + kThreads - 1) / kThreads));
#define XYZ_MARK(cls, start)              \
  do {                                    \
    int const m_ = mark((cls), (start));  \
    if (m_) return m_;                    \
  } while (0)
      // One pass over the wave: camera rays, then per bounce closest hit,
      // shading and shadow rays.  The adjoint runs it twice (primal, replay).
      auto pass = [&](bool replay) -> int {
        XYZ_MARK(0, true);
        k_raygen<<<gr, kThreads, 0, st>>>(A);
        XYZ_MARK(0, false);
        ++launches;
        for (int b = 0; b < iters; ++b) {
          XYZ_MARK(1, true);
          if (counting)
            k_trace_queue<false, true><<<g_trace_e, kThreads, 0, st>>>(A, b, pc);
          else
            k_trace_queue<false, false><<<g_trace_e, kThreads, 0, st>>>(A, b, pc);
          XYZ_MARK(1, false);
          XYZ_MARK(2, true);
          if (spectral)
            k_shade_spectral<<<g_shade_sp, kThreads, 0, st>>>(A, b);
          else if (replay)
            k_shade<true><<<g_shade, kThreads, 0, st>>>(A, b);
          else
            k_shade<false><<<g_shade, kThreads, 0, st>>>(A, b);
          XYZ_MARK(2, false);
          XYZ_MARK(3, true);
          if (counting)
            k_trace_queue<true, true><<<g_trace_s, kThreads, 0, st>>>(A, b, pc);
          else if (replay)
            k_trace_queue<true, false, true><<<g_trace_s, kThreads, 0, st>>>(A, b, pc);
          else
            k_trace_queue<true, false><<<g_trace_s, kThreads, 0, st>>>(A, b, pc);
          XYZ_MARK(3, false);
          launches += 3;
        }
        return XYZGPU_OK;
      };
      int const pr = pass(false);
      if (pr) return pr;
      int const gf = static_cast<int>(std::min<int64_t>(g_film, (A.npix + kThreads - 1) / kThreads));
      if (adj) {
        int const gs = static_cast<int>(std::min<int64_t>(g_film, (A.npaths + kThreads - 1) / kThreads));
        k_adj_stash<<<gs, kThreads, 0, st>>>(A);
        ++launches;
        XYZ_CUDA_TRY(cudaMemsetAsync(wv.counts, 0, static_cast<size_t>(iters + 2) * kCountStride * sizeof(int32_t), st));
        int const rr = pass(true);
        if (rr) return rr;
      } else {
        XYZ_MARK(4, true);
        if (spectral)
          k_film_spectral<<<gf, kThreads, 0, st>>>(A, film_dev);
        else
          k_film<<<gf, kThreads, 0, st>>>(A, film_dev);
        XYZ_MARK(4, false);
        ++launches;
      }
#undef XYZ_MARK
      k_tally<<<1, 32, 0, st>>>(A, iters, w.tally);
      ++launches;
      XYZ_CUDA_TRY(cudaGetLastError());
      rc_out.paths += static_cast<uint64_t>(A.npaths);
      rc_out.waves += 1;
    }
  }
  XYZ_CUDA_TRY(cudaEventRecord(sw.done, st));
  sw.last = st;
  if (!adj && rp.film_location == XYZGPU_FILM_HOST) {
    XYZ_CUDA_TRY(cudaMemcpyAsync(w.film_pinned, film_dev, film_elems * sizeof(float), cudaMemcpyDeviceToHost, st));
    XYZ_CUDA_TRY(cudaStreamSynchronize(st));
    std::memcpy(film, w.film_pinned, film_elems * sizeof(float));
  }
  rc_out.kernel_launches = launches;
  s.counters = rc_out;
  s.profile_mode = prof;
  s.profile_pending = true;
  return XYZGPU_OK;
}

// Reads back the device tallies (and event times) of the last render.
int render_collect(SceneImpl &s) {
  if (!s.profile_pending) return XYZGPU_OK;
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  RenderWorkspace &w = s.ws;
  XYZ_CUDA_TRY(cudaDeviceSynchronize());
  unsigned long long t[kTallyWords];
  XYZ_CUDA_TRY(cudaMemcpy(t, w.tally, sizeof(t), cudaMemcpyDeviceToHost));
  s.counters.extension_rays = t[0];
  s.counters.shadow_rays = t[1];
  s.counters.shadow_hits_visible = t[2];
  if (s.profile_mode != XYZGPU_PROFILE_OFF) {
    xyzgpu_render_profile &p = s.profile;
    p = xyzgpu_render_profile{};
    p.ext_rays = t[0];
    p.shadow_rays = t[1];
    p.shadow_visible = t[2];
    p.iterations = static_cast<uint32_t>(std::min(w.profile_iters, XYZGPU_PROFILE_MAX_ITERS));
    for (int b = 0; b < XYZGPU_PROFILE_MAX_ITERS; ++b) {
      p.ext_rays_by_iter[b] = t[kTallyIterBase + b];
      p.shadow_rays_by_iter[b] = t[kTallyIterBase + XYZGPU_PROFILE_MAX_ITERS + b];
    }
    if (s.profile_mode == XYZGPU_PROFILE_COUNTERS) {
      p.ext_nodes = t[8];
      p.ext_leaves = t[9];
      p.ext_tri_tests = t[10];
      p.shadow_nodes = t[11];
      p.shadow_leaves = t[12];
      p.shadow_tri_tests = t[13];
    }
    if (s.profile_mode == XYZGPU_PROFILE_TIMING) {
      for (size_t i = 0; i < s.event_class.size(); ++i) {
        float ms = 0.0f;
        XYZ_CUDA_TRY(cudaEventElapsedTime(&ms, w.events[2 * i], w.events[2 * i + 1]));
        int const c = s.event_class[i];
        p.launches[c] += 1;
        p.ms[c] += ms;
      }
    }
  }
  s.profile_pending = false;
  return XYZGPU_OK;
}

// ---------------------------------------------------------------------------
// xyzgpu_render_noalloc: rendering for callers that cannot allocate.
//
// Some hosts must not allocate device memory once they are running: a
// renderer embedded in an application that hands all GPU memory to its own
// pool at start-up, a real-time loop that may not enter the driver's allocator
// (and its implicit synchronisation) in the middle of a frame, or a process
// whose memory budget is fixed when it starts.  xyzgpu_render allocates the
// per-scene path state and queues on its first call and again whenever a
// larger wave is asked for; this entry point instead keeps them in one
// file-scope device array of fixed size, so it performs no allocation at all.
// The scene (created beforehand) and the device film are the caller's.
//
// The array is XYZGPU_NOALLOC_SCRATCH_BYTES on every device that loads the
// library, held until the process exits.  It holds the state of at most
// XYZGPU_NOALLOC_MAX_WAVE_PATHS paths in flight, so large images render in
// more, smaller waves than xyzgpu_render uses (same image, lower throughput).
// Every call on a device shares the array and it keeps the previous call's
// contents: calls that overlap on the GPU (different streams, threads or
// scenes) race and must be serialised by the caller.
namespace {

constexpr int64_t kNoAllocPaths = XYZGPU_NOALLOC_MAX_WAVE_PATHS;
constexpr int kNoAllocDepth = XYZGPU_NOALLOC_MAX_DEPTH;
constexpr size_t kSeg = 256;
constexpr size_t seg(size_t bytes) { return (bytes + kSeg - 1) / kSeg * kSeg; }
constexpr size_t kNoAllocF4 = seg(kNoAllocPaths * sizeof(float4));
constexpr size_t kNoAllocI4 = seg(kNoAllocPaths * sizeof(int32_t));
constexpr size_t kNoAllocCounts = seg((kNoAllocDepth + 2) * kCountStride * sizeof(int32_t));
constexpr size_t kNoAllocTally = seg(16 * sizeof(unsigned long long));
// beta, radiance, q_o[2], q_d[2], hits, s_o, s_d, s_pb: 10 float4 arrays;
// misc, q_slot[2], s_target: 4 int arrays.
constexpr size_t kNoAllocBytes = 10 * kNoAllocF4 + 4 * kNoAllocI4 + kNoAllocCounts + kNoAllocTally;
static_assert(kNoAllocBytes == XYZGPU_NOALLOC_SCRATCH_BYTES,
              "XYZGPU_NOALLOC_SCRATCH_BYTES must match the scratch layout");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocBytes];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_base[64] = {nullptr};

// Device address of g_noalloc_scratch on `device` (which must be current).
// The first call on a device looks the symbol up; later calls reuse it.
int noalloc_scratch(int device, unsigned char **out) {
  if (device < 0 || device >= 64)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: device ordinal %d is beyond 63", device);
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_base[device]) {
    void *p = nullptr;
    cudaError_t const e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr)
      return set_error(XYZGPU_E_CUDA, "render_noalloc: cudaGetSymbolAddress failed: %s",
                       cudaGetErrorString(e));
    g_noalloc_base[device] = p;
  }
  *out = static_cast<unsigned char *>(g_noalloc_base[device]);
  return XYZGPU_OK;
}

CamDev noalloc_camera(const xyzgpu_camera &cam, int width, int height) {
  // ThinLensCamera::Reset (thinlenscamera.cpp:71-90), as in render_launch.
  CamDev C;
  C.eye = mk3(cam.eye[0], cam.eye[1], cam.eye[2]);
  f3 const at = mk3(cam.at[0], cam.at[1], cam.at[2]);
  f3 const view = sub3(C.eye, at);
  C.L = std::sqrt(dot3(view, view));
  C.V = C.L * cam.focal_length / (C.L - cam.focal_length);
  C.R = cam.focal_length / (2 * cam.f_number);
  float const r = 1.0f / std::sqrt(dot3(view, view));
  C.back = scl3(view, r);
  f3 const rr = cross3(mk3(0.0f, 1.0f, 0.0f), C.back);
  float const r2 = 1.0f / std::sqrt(dot3(rr, rr));
  C.right = scl3(rr, r2);
  C.up = cross3(C.back, C.right);
  C.film = cam.film_size;
  C.aspect = static_cast<float>(width) / static_cast<float>(height);
  C.pinhole = cam.pinhole ? 1 : 0;
  return C;
}

}  // namespace

int render_noalloc_launch(SceneImpl &s, const xyzgpu_camera &cam, const xyzgpu_render_params &rp,
                          float *film, cudaStream_t st) {
  if (rp.film_location != XYZGPU_FILM_DEVICE)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: the film must be device memory");
  if (rp.profile != XYZGPU_PROFILE_OFF)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: profiling is not available");
  if (rp.spectral != XYZGPU_SPECTRAL_OFF)
    return set_error(XYZGPU_E_INVALID, "render_noalloc: only the XYZ film mode is available");
  if (rp.wave_paths > kNoAllocPaths)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: wave_paths %d exceeds the maximum of %lld",
                     rp.wave_paths, static_cast<long long>(kNoAllocPaths));
  if (rp.max_depth > kNoAllocDepth)
    return set_error(XYZGPU_E_LIMIT, "render_noalloc: max_depth %d exceeds the maximum of %d",
                     rp.max_depth, kNoAllocDepth);
  XYZ_CUDA_TRY(cudaSetDevice(s.device));
  unsigned char *base = nullptr;
  int rc = noalloc_scratch(s.device, &base);
  if (rc) return rc;

  WaveArgs A;
  std::memset(&A, 0, sizeof(A));
  unsigned char *p = base;
  auto take = [&p](size_t bytes) {
    unsigned char *q = p;
    p += bytes;
    return q;
  };
  A.beta = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.radiance = reinterpret_cast<float4 *>(take(kNoAllocF4));
  for (int q = 0; q < 2; ++q) {
    A.q_o[q] = reinterpret_cast<float4 *>(take(kNoAllocF4));
    A.q_d[q] = reinterpret_cast<float4 *>(take(kNoAllocF4));
  }
  A.hits = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_o = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_d = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.s_pb = reinterpret_cast<float4 *>(take(kNoAllocF4));
  A.misc = reinterpret_cast<uint32_t *>(take(kNoAllocI4));
  for (int q = 0; q < 2; ++q) A.q_slot[q] = reinterpret_cast<int32_t *>(take(kNoAllocI4));
  A.s_target = reinterpret_cast<int32_t *>(take(kNoAllocI4));
  A.counts = reinterpret_cast<int32_t *>(take(kNoAllocCounts));
  unsigned long long *tally = reinterpret_cast<unsigned long long *>(take(kNoAllocTally));

  A.S = s.dev;
  A.cam = noalloc_camera(cam, rp.width, rp.height);
  A.W = rp.width;
  A.H = rp.height;
  A.kmax = rp.max_depth + 1;
  A.rr_start = rp.rr_start_depth;
  A.rr_threshold = rp.rr_threshold;
  A.seed = rp.seed;

  static int g_raygen = 0, g_trace_e = 0, g_trace_s = 0, g_shade = 0, g_film = 0;
  if (!g_raygen) {
    g_raygen = occupancy_grid(k_raygen, s.device);
    g_trace_e = occupancy_grid(k_trace_queue<false, false>, s.device);
    g_trace_s = occupancy_grid(k_trace_queue<true, false>, s.device);
    g_shade = occupancy_grid(k_shade<false>, s.device);
    g_film = occupancy_grid(k_film, s.device);
  }
  int64_t const npix_total = static_cast<int64_t>(rp.width) * rp.height;
  int64_t const cap = rp.wave_paths > 0 ? rp.wave_paths : kNoAllocPaths;
  int const iters = rp.max_depth;
  if (!rp.accumulate) XYZ_CUDA_TRY(cudaMemsetAsync(film, 0, 3 * npix_total * sizeof(float), st));
  XYZ_CUDA_TRY(cudaMemsetAsync(tally, 0, kNoAllocTally, st));
  int64_t const spp_per_wave =
      std::max<int64_t>(1, std::min<int64_t>(rp.spp, cap / std::max<int64_t>(1, npix_total)));
  int64_t const pix_per_wave = std::min<int64_t>(npix_total, cap);
  for (int64_t s0 = 0; s0 < rp.spp; s0 += spp_per_wave) {
    int const ns = static_cast<int>(std::min<int64_t>(spp_per_wave, rp.spp - s0));
    for (int64_t p0 = 0; p0 < npix_total; p0 += pix_per_wave) {
      A.p0 = p0;
      A.npix = std::min<int64_t>(pix_per_wave, npix_total - p0);
      A.s0 = static_cast<uint32_t>(rp.spp_offset + s0);
      A.nsamp = ns;
      A.npaths = A.npix * ns;
      // queue lengths and work counters from the previous wave or call
      XYZ_CUDA_TRY(cudaMemsetAsync(A.counts, 0, kNoAllocCounts, st));
      int const gr = static_cast<int>(std::min<int64_t>(g_raygen, (A.npaths + kThreads - 1) / kThreads));
      k_raygen<<<gr, kThreads, 0, st>>>(A);
      for (int b = 0; b < iters; ++b) {
        k_trace_queue<false, false><<<g_trace_e, kThreads, 0, st>>>(A, b, tally + 8);
        k_shade<false><<<g_shade, kThreads, 0, st>>>(A, b);
        k_trace_queue<true, false><<<g_trace_s, kThreads, 0, st>>>(A, b, tally + 8);
      }
      int const gf = static_cast<int>(std::min<int64_t>(g_film, (A.npix + kThreads - 1) / kThreads));
      k_film<<<gf, kThreads, 0, st>>>(A, film);
      XYZ_CUDA_TRY(cudaGetLastError());
    }
  }
  return XYZGPU_OK;
}

}  // namespace xyzgpu
