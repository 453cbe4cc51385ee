// Wavefront path tracer: the kernels of xyzgpu_render, xyzgpu_adjoint and the
// batched renders (xyzgpu_batch_*).
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
#pragma once

#include <algorithm>
#include <cmath>
#include <cstring>

#include <cuda_fp16.h>

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

// Batched renders (xyzgpu_batch_*): one wave holds paths of many scenes.
// Per render ("job") constants live in a device table; a wave is a list of
// blocks, each a run of consecutive samples of one job over all its pixels.
// The block of a path travels in its queue records (the w of the origin
// float4, whose value is a constant in single-scene renders).
struct BatchJob {
  DevScene S;
  CamDev cam;
  int W, H;
  int kmax, rr_start;
  float rr_threshold;
  int tile;             // slot order: pixel tiles of tile x tile (1 = scanlines)
  uint64_t seed;
  uint32_t spp_offset;  // first sample index of the job's render
  float *film;          // W * H * 3 sums, device
  int clear;            // the launch zeroes the film first (the job does not accumulate)
};

struct WaveBlock {
  int job;
  int ns;            // samples of the job in this wave
  uint32_t s0;       // first sample, relative to the job's spp_offset
  int64_t npix;      // the job's pixels
  int64_t slot_off;  // first path slot of the block: slot = slot_off + s * npix + p
  int64_t pix_off;   // first film thread of the block (film kernel)
};

// A wave of a batch: its blocks are blocks[first_block .. first_block + n_blocks).
struct BatchWave {
  int first_block, n_blocks;
  int64_t npaths, film_threads;  // path slots; pixels of all its blocks (film threads)
  int iters;                     // bounces: the largest max_depth of its jobs
};

// Where a batch launch is, in device memory: the wave and bounce the batched
// kernels work on and a copy of that wave's entry.  The batch's control
// kernels advance it, so the same kernels serve every wave and bounce.
struct BatchCursor {
  int wave, bounce;
  BatchWave w;
};

// Variants of the shading and shadow kernels: the plain render, the replay
// pass of the adjoint, batched renders and guided renders.
enum WaveMode : int { kModePlain = 0, kModeAdjoint = 1, kModeBatch = 2, kModeGuided = 3, kModeImporton = 4 };

struct WaveArgs {
  DevScene S;
  CamDev cam;
  int W, H;
  int kmax;         // the reference's kMax = max_depth + 1
  int rr_start;
  float rr_threshold;
  uint64_t seed;
  int64_t p0;       // first pixel of the wave, counted over the rendered rows
  int64_t npix;     // pixels in the wave
  const float *imp_cdf;  // importance-driven: 16 cumulative histogram counts per extension-queue
                         // entry of this bounce, or null (Lambert sampling)
  int64_t row0;     // first rendered image row
  int row_step;     // rendered rows are row0, row0 + row_step, ... (0 or 1: consecutive)
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
  float4 *s_m;      // metal vertices: nk2, nk3, lobe pdf, pdf / max(nk1, nk2) * Fresnel
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
  // adjoint with cached intersections: the primal pass records every path's
  // extension hit and its shadow ray's target distance (NaN: not visible) per
  // bounce, at slot * cache_stride + bounce; the replay reads them instead of
  // tracing (both null otherwise)
  float4 *hit_cache;
  float *vis_cache;
  int cache_stride;
  // batched renders
  const BatchJob *jobs;
  const WaveBlock *blocks;    // all blocks of the batch; a record's block indexes it
  const BatchCursor *cursor;  // the current wave and bounce
  // guided renders: the guide's mixture per extension-queue entry (40 fp16:
  // per lobe weight, concentration, mean xyz), the one-sample MIS probability
  // of the guide, and training records (16 floats x train_bounces per path:
  // position, normal, direction, pdf, throughput after the vertex, radiance
  // before the next vertex)
  const __half *mix;
  float guide_alpha;
  float *records;
  int train_bounces;
};

// ------------------------------------------------------- guide mixture
// von Mises-Fisher lobes: vMF(d; mu, k) = k / (2 pi (1 - e^{-2k})) exp(k (mu.d - 1)).
// A vertex's mixture stays in its 40 raw fp16 values (8 lobes of weight,
// kappa, mean xyz; 20 registers) and every use decodes a lobe the same way:
// weight max(w, 0) / sum (uniform if the sum is 0), kappa max(k, 1e-3), mean
// normalised ((0, 0, 1) if zero).  Sampling and the pdf therefore describe
// the same mixture whatever the fp16 rounding.  The decode and the density use
// the fast intrinsics (rsqrt, fast divide, exp2-based exp): both sides read the
// same decoded lobes, and the density's relative error (~1e-6) is far below
// the Monte Carlo noise.
struct GuideMix {
  uint4 q[5];
  float ws;  // sum of the clamped weights
};

XYZ_DEV float mix_half(const GuideMix &M, int t) {
  uint4 const v = M.q[t >> 3];
  int const c = (t >> 1) & 3;
  uint32_t const w = c == 0 ? v.x : c == 1 ? v.y : c == 2 ? v.z : v.w;
  return __half2float(__ushort_as_half(static_cast<unsigned short>((t & 1) ? (w >> 16) : (w & 0xffffu))));
}

// The raw values (issued early: they do not depend on the hit) ...
XYZ_DEV void load_mix(const __half *src, GuideMix &M) {
  const uint4 *q = reinterpret_cast<const uint4 *>(src);
#pragma unroll
  for (int t = 0; t < 5; ++t) M.q[t] = q[t];
}
// ... and the weight sum, once they are needed.
XYZ_DEV void finish_mix(GuideMix &M) {
  float ws = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) ws += fmaxf(mix_half(M, 5 * i), 0.0f);
  M.ws = ws;
}

XYZ_DEV float mix_weight(const GuideMix &M, int i) {
  return M.ws > 0.0f ? fmaxf(mix_half(M, 5 * i), 0.0f) : 1.0f;
}
XYZ_DEV float mix_kappa(const GuideMix &M, int i) { return fmaxf(mix_half(M, 5 * i + 1), 1e-3f); }
XYZ_DEV f3 mix_mean(f3 m) {
  float const l2 = dot3(m, m);
  return l2 > 0.0f ? scl3(m, rsqrtf(l2)) : mk3(0.0f, 0.0f, 1.0f);
}
XYZ_DEV f3 mix_mean(const GuideMix &M, int i) {
  return mix_mean(mk3(mix_half(M, 5 * i + 2), mix_half(M, 5 * i + 3), mix_half(M, 5 * i + 4)));
}

// vMF normaliser k / (2 pi (1 - e^{-2k})); below k = 0.05 the series
// 1 - e^{-2k} = 2k (1 - k + 2k^2/3 - k^3/3) avoids the cancellation.
XYZ_DEV float vmf_norm(float k) {
  float const den = k < 0.05f ? 2.0f * k * (1.0f - k * (1.0f - k * (2.0f / 3.0f - k * (1.0f / 3.0f))))
                              : 1.0f - __expf(-2.0f * k);
  return __fdividef(k, static_cast<float>(2.0 * kPi) * den);
}

// Mixture density at two directions in one pass over the lobes.
XYZ_DEV void mix_pdf2(const GuideMix &M, f3 d1, f3 d2, float *p1, float *p2) {
  float a1 = 0.0f, a2 = 0.0f;
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    float const k = mix_kappa(M, i);
    float const wc = mix_weight(M, i) * vmf_norm(k);
    f3 const mu = mix_mean(M, i);
    a1 += wc * __expf(k * (dot3(mu, d1) - 1.0f));
    a2 += wc * __expf(k * (dot3(mu, d2) - 1.0f));
  }
  float const inv = M.ws > 0.0f ? 1.0f / M.ws : 0.125f;
  *p1 = a1 * inv;
  *p2 = a2 * inv;
}

// Lobe by weight, then the lobe's cosine w = 1 + log(u1 + (1 - u1) e^{-2k}) / k
// (Jakob, "Numerically stable sampling of the von Mises-Fisher distribution
// on S^2", 2012) around its mean, in the orthonormal basis of Duff et al.,
// "Building an Orthonormal Basis, Revisited" (JCGT 2017).  The lobe's raw
// values are picked with selects (no indexed access to the registers); the
// inversion uses the fast intrinsics (the density above is that of the
// exact inversion, ~1e-6 relative away).
XYZ_DEV f3 mix_sample(const GuideMix &M, float ul, float u1, float u2) {
  float const target = ul * (M.ws > 0.0f ? M.ws : 8.0f);
  float acc = 0.0f;
  bool found = false;
  float kr = mix_half(M, 36), mx = mix_half(M, 37), my = mix_half(M, 38), mz = mix_half(M, 39);
#pragma unroll
  for (int i = 0; i < 7; ++i) {
    acc += mix_weight(M, i);
    bool const take = !found && target < acc;
    kr = take ? mix_half(M, 5 * i + 1) : kr;
    mx = take ? mix_half(M, 5 * i + 2) : mx;
    my = take ? mix_half(M, 5 * i + 3) : my;
    mz = take ? mix_half(M, 5 * i + 4) : mz;
    found = found || take;
  }
  float const k = fmaxf(kr, 1e-3f);
  f3 const n = mix_mean(mk3(mx, my, mz));
  float w = 1.0f + __fdividef(__logf(u1 + (1.0f - u1) * __expf(-2.0f * k)), k);
  w = fminf(fmaxf(w, -1.0f), 1.0f);
  float const sw = sqrtf(fmaxf(0.0f, 1.0f - w * w));
  float sp, cp;
  __sincosf(static_cast<float>(2.0 * kPi) * u2, &sp, &cp);
  float const sign = copysignf(1.0f, n.z);
  float const a = __fdividef(-1.0f, sign + n.z);
  float const bb = n.x * n.y * a;
  f3 const t = mk3(1.0f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
  f3 const bt = mk3(bb, sign + n.y * n.y * a, -n.y);
  return add3(add3(scl3(t, sw * cp), scl3(bt, sw * sp)), scl3(n, w));
}

XYZ_DEV uint32_t pack_misc(uint32_t dim, uint32_t k, uint32_t specular) {
  return (dim & 0xffffu) | ((k & 0x7fffu) << 16) | (specular << 31);
}

// Image pixel (y * W + x) of pixel `lp` counted over the rendered rows.
XYZ_DEV int64_t film_pixel(const WaveArgs &A, int64_t lp) {
  if (A.row_step <= 1) return A.row0 * A.W + lp;
  int64_t const r = lp / A.W;
  return (A.row0 + r * A.row_step) * A.W + (lp - r * A.W);
}

XYZ_DEV void slot_to_pixel_sample(const WaveArgs &A, int64_t slot, uint32_t *pixel,
                                  uint32_t *sample) {
  int64_t const sl = slot / A.npix;
  int64_t const pl = slot - sl * A.npix;
  *pixel = static_cast<uint32_t>(film_pixel(A, A.p0 + pl));
  *sample = A.s0 + static_cast<uint32_t>(sl);
}

// Block of a path slot in a batched wave (the wave's blocks are in slot order).
XYZ_DEV int block_of_slot(const WaveArgs &A, const BatchWave &w, int64_t slot) {
  int lo = w.first_block, hi = w.first_block + w.n_blocks - 1;
  while (lo < hi) {
    int const mid = (lo + hi + 1) >> 1;
    if (A.blocks[mid].slot_off <= slot)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Pixel index of the pl-th pixel of a job in tile order: tiles of
// tile x tile pixels, row-major, pixels row-major inside a tile (the image
// dimensions are multiples of tile).
XYZ_DEV uint32_t tile_pixel(int64_t pl, int W, int tile) {
  if (tile <= 1) return static_cast<uint32_t>(pl);
  int64_t const tt = static_cast<int64_t>(tile) * tile;
  int64_t const t = pl / tt;
  int const r = static_cast<int>(pl - t * tt);
  int const tiles_x = W / tile;
  int const tx = static_cast<int>(t % tiles_x), ty = static_cast<int>(t / tiles_x);
  int const x = tx * tile + r % tile, y = ty * tile + r / tile;
  return static_cast<uint32_t>(y) * static_cast<uint32_t>(W) + static_cast<uint32_t>(x);
}

// The scene, estimator parameters and (pixel, sample) of a path.  kBatch:
// from the job table through the path's block; else the single render's.
template <bool kBatch>
XYZ_DEV const DevScene &scene_of(const WaveArgs &A, int block) {
  if constexpr (kBatch)
    return A.jobs[A.blocks[block].job].S;
  else
    return A.S;
}

struct PathParams {
  int kmax, rr_start;
  float rr_threshold;
  uint64_t seed;
};

template <bool kBatch>
XYZ_DEV PathParams params_of(const WaveArgs &A, int block) {
  if constexpr (kBatch) {
    const BatchJob &J = A.jobs[A.blocks[block].job];
    return PathParams{J.kmax, J.rr_start, J.rr_threshold, J.seed};
  } else {
    return PathParams{A.kmax, A.rr_start, A.rr_threshold, A.seed};
  }
}

template <bool kBatch>
XYZ_DEV void path_pixel_sample(const WaveArgs &A, int block, int64_t slot, uint32_t *pixel,
                               uint32_t *sample) {
  if constexpr (kBatch) {
    const WaveBlock &B = A.blocks[block];
    const BatchJob &J = A.jobs[B.job];
    int64_t const l = slot - B.slot_off;
    int64_t const sl = l / B.npix;
    int64_t const pl = l - sl * B.npix;
    *pixel = tile_pixel(pl, J.W, J.tile);
    *sample = J.spp_offset + B.s0 + static_cast<uint32_t>(sl);
  } else {
    slot_to_pixel_sample(A, slot, pixel, sample);
  }
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
template <bool kBatch>
__global__ void __launch_bounds__(kThreads) k_raygen(WaveArgs A) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  BatchWave wv{};
  if constexpr (kBatch) wv = A.cursor->w;
  int64_t const npaths = kBatch ? wv.npaths : A.npaths;
  for (int64_t slot = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; slot < npaths;
       slot += stride) {
    int const block = kBatch ? block_of_slot(A, wv, slot) : 0;
    uint32_t pixel, sample;
    path_pixel_sample<kBatch>(A, block, slot, &pixel, &sample);
    uint64_t const seed = params_of<kBatch>(A, block).seed;
    int const W = kBatch ? A.jobs[A.blocks[block].job].W : A.W;
    int const H = kBatch ? A.jobs[A.blocks[block].job].H : A.H;
    uint32_t w[4];
    philox4x32_10(pixel, sample, 0u, 0u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), w);
    float const jx = u01_from_bits(w[0]);
    float const jy = u01_from_bits(w[1]);
    int const px = static_cast<int>(pixel % static_cast<uint32_t>(W));
    int const py = static_cast<int>(pixel / static_cast<uint32_t>(W));
    float const x = (static_cast<float>(px) + jx) / static_cast<float>(W);
    float const y = (static_cast<float>(py) + jy) / static_cast<float>(H);
    CamDev const &C = kBatch ? A.jobs[A.blocks[block].job].cam : A.cam;
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
      philox4x32_10(pixel, sample, 1u, 0u, static_cast<uint32_t>(seed), static_cast<uint32_t>(seed >> 32), w2);
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
    A.q_o[0][slot] = make_float4(o.x, o.y, o.z, kBatch ? __int_as_float(block) : kRayTMin);
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
  if (blockIdx.x == 0 && threadIdx.x == 0) A.counts[kCExt] = static_cast<int32_t>(npaths);
}

// ------------------------------------------------------------------ trace
// Persistent warps with per-lane refill over a device-sized queue
// (trace_persistent).  kShadow: the ray starts at a light point and the
// vertex's NEE term is added when the closest hit is the vertex's own triangle.
// Queue records are read and written once: streaming (evict-first) accesses
// keep them from displacing tree nodes and triangles in L1.
template <bool kBatch>
struct ExtSink {
  const float4 *__restrict__ qo;
  const float4 *__restrict__ qd;
  float4 *__restrict__ hits;
  const WaveArgs *A;
  XYZ_DEV void load(int i, f3 &o, f3 &d, float &tmin, float &tmax) const {
    float4 const a = __ldcs(&qo[i]), b = __ldcs(&qd[i]);
    o = xyz3(a);
    d = xyz3(b);
    tmin = kBatch ? kRayTMin : a.w;  // batched: w holds the path's block
    tmax = b.w;
  }
  XYZ_DEV const DevScene *scene(int i) const {
    return &scene_of<true>(*A, __float_as_int(qo[i].w));
  }
  XYZ_DEV void store(int i, const RayHit &h) {
    int32_t const code = h.id >= 0 ? ((h.id << 1) | h.back) : -1;
    __stcs(&hits[i], make_float4(h.t, h.f, h.g, __int_as_float(code)));
  }
};

template <bool kSpec, int kMode = kModePlain>
struct ShadowSink {
  static constexpr bool kAdj = kMode == kModeAdjoint;
  static constexpr bool kBatch = kMode == kModeBatch;
  static constexpr bool kGuide = kMode == kModeGuided;
  static constexpr bool kImp = kMode == kModeImporton;
  static constexpr bool kTarget = true;  // only "is the target the closest hit?" matters
  const WaveArgs *A;
  uint32_t visible;
  int bounce;
  XYZ_DEV int32_t target(int i) const { return __ldg(&A->s_target[i]); }
  XYZ_DEV void load(int i, f3 &o, f3 &d, float &tmin, float &tmax) const {
    float4 const a = __ldcs(&A->s_o[i]), b = __ldcs(&A->s_d[i]);
    o = xyz3(a);
    d = xyz3(b);
    tmin = kRayTMin;
    tmax = kBatch ? __int_as_float(0x7f800000) : a.w;  // batched: w holds the block
  }
  XYZ_DEV const DevScene *scene(int i) const {
    return &scene_of<true>(*A, __float_as_int(A->s_o[i].w));
  }
  XYZ_DEV void store(int i, const RayHit &h) {
    if (h.id < 0 || h.id != A->s_target[i]) return;
    float const light_area = kBatch ? scene(i)->light_area : A->S.light_area;
    const DevScene &SV = kBatch ? *scene(i) : A->S;
    double wgt;
    if (!kSpec && SV.has_metal && __ldg(&SV.mat[__float_as_int(__ldg(&SV.tri_ng[h.id]).w)]).w == 3.0f) {
      // Metal::CalculateWeightedDirectLighting (xyz/bsdf/metal.cpp:68-119):
      // w = nk3 / t^2, G = nk2 w, the MIS density of the lobe's pdf against
      // the light's area density; the lobe pdf / max(nk1, nk2) * Fresnel
      // factor comes with the record
      float4 const sm = A->s_m[i];
      float const w = sm.y / (h.t * h.t);
      float const Gm = sm.x * w;
      float const fd = sm.z * w * light_area;
      wgt = (static_cast<double>(Gm) * kInvPi) * static_cast<double>(sm.w) *
            static_cast<double>(1.0f / (1.0f + fd * fd));
    } else {
      // Lambert::CalculateWeightedDirectLighting, lambert.cpp:157-172
      float const G = A->s_d[i].w / (h.t * h.t);  // nk2 * nk3 / t^2
      // importance-driven: M_1_PI * G * the histogram's density of the light
      // direction, in double as Lambert::CalculateWeightedDirectLighting with
      // importons computes it (xyz/bsdf/lambert.cpp:210-212)
      float dimp = kImp ? static_cast<float>(kInvPi * static_cast<double>(G) *
                                             static_cast<double>(__int_as_float(A->s_slot[i])))
                        : static_cast<float>(kInvPi * static_cast<double>(G));
      // guided: the sampling density is the guide / Lambert mixture, rho times Lambert's
      if (kGuide) dimp *= __int_as_float(A->s_slot[i]);
      float const dexp = 1.0f / light_area;
      float const dens = dimp / dexp;
      wgt = (static_cast<double>(G) * (kInvPi * kInvPi)) * static_cast<double>(1.0f / (1.0f + dens * dens));
    }
    float4 pb = A->s_pb[i];
    int32_t const slot = kSpec ? A->s_slot[i] : __float_as_int(pb.w);
    if (kMode == kModePlain && !kSpec && A->vis_cache)
      A->vis_cache[static_cast<int64_t>(slot) * A->cache_stride + bounce] = h.t;
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

// CTAs per SM: extension rays run at 9 (56 registers, no spills: 5 % faster
// than 10 CTAs at 48 registers with ~50 bytes of spills), shadow rays at 10
// (measured on B200, 1M-triangle scene).
template <bool kShadow, bool kCount, int kMode = kModePlain>
__global__ void __launch_bounds__(kThreads, kShadow ? 10 : 9) k_trace_queue(WaveArgs A, int b,
                                                          unsigned long long *prof) {
  constexpr bool kBatch = kMode == kModeBatch;
  if constexpr (kBatch) b = A.cursor->bounce;
  int32_t *const cnt = A.counts + b * kCountStride;
  int const n = kShadow ? cnt[kCShadow] : cnt[kCExt];
  int const lane = threadIdx.x & 31;
  int const qi = b & 1;
  TraceCount tc{0u, 0u, 0u};
  uint32_t visible = 0;
  if (kShadow && kMode != kModePlain) {
    ShadowSink<false, kMode> sink{&A, 0u, b};
    trace_persistent<kCount, kBatch>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else if (kBatch) {
    ExtSink<true> sink{A.q_o[qi], A.q_d[qi], A.hits, &A};
    trace_persistent<kCount, true>(A.S, n, &cnt[kCFetchExt], sink, tc);
  } else if (kShadow && A.spectral) {
    ShadowSink<true> sink{&A, 0u, b};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else if (kShadow) {
    ShadowSink<false> sink{&A, 0u, b};
    trace_persistent<kCount>(A.S, n, &cnt[kCFetchSh], sink, tc);
    visible = sink.visible;
  } else {
    ExtSink<false> sink{A.q_o[qi], A.q_d[qi], A.hits, &A};
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

// Batched waves (A.cursor set) take their bounce count from the cursor.
__global__ void k_tally(WaveArgs A, int iters, unsigned long long *tally) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  if (A.cursor) iters = A.cursor->w.iters;
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

// ImportanceQuery::GetDensity (xyz/core/photonmap.cpp:375-401): the density,
// relative to cosine sampling, of direction `dir` (towards the surface) under
// the histogram c (cumulative counts, c[0] = 0): bins of cos^2 theta (2) and
// phi / 2 (8) about the shading frame.
XYZ_DEV int importon_bin(f3 dir, f3 sn, f3 tan, f3 bin, bool *above) {
  float const cs = -dot3(dir, sn);
  *above = cs > 0.0f;
  int u = static_cast<int>(cs * cs * 2.0f);
  if (u >= 2) u = 1;
  float phi = 0.5f * atan2f(-dot3(dir, bin), -dot3(dir, tan));
  if (phi < 0.0f) phi = static_cast<float>(static_cast<double>(phi) + kPi);
  int v = static_cast<int>(static_cast<double>(phi) * (8.0 * kInvPi));
  if (v >= 8) v = 7;
  return u * 8 + v;
}

XYZ_DEV float importon_density(const float *c, f3 dir, f3 sn, f3 tan, f3 bin) {
  bool above;
  int const n = importon_bin(dir, sn, tan, bin, &above);
  if (!above) return 0.0f;
  return 16.0f * (c[n + 1] - c[n]) / c[16];
}

// FakeFresnelTerm (xyz/stdafx.hpp:44-47): F0 + (1 - F0) (1 - hk)^5, F0 = 0.9,
// the fifth power as hi::fifth_power_of forms it (x * ((x x) (x x))).
XYZ_DEV float fake_fresnel(float hk) {
  float const f0 = 0.9f;
  float const x = 1.0f - hk;
  float const x2 = x * x;
  return f0 + (1.0f - f0) * (x * (x2 * x2));
}

// Triangle::ShadingBasis (triangle.cpp:194-219) at barycentrics (f, g):
// geometric and interpolated shading normals (flipped on the back side) and
// the tangent frame about the shading normal; returns the material id.
XYZ_DEV int32_t shading_frame(const DevScene &S, int32_t tri, int back, float f, float g, f3 *gn_out, f3 *sn_out,
                              f3 *tan_out, f3 *bin_out) {
  float4 const g4 = __ldg(&S.tri_ng[tri]);
  f3 gn = xyz3(g4);
  f3 sn;
  if (S.tri_sn) {
    f3 const n0 = xyz3(__ldg(&S.tri_sn[3 * tri])), s1 = xyz3(__ldg(&S.tri_sn[3 * tri + 1])),
             s2 = xyz3(__ldg(&S.tri_sn[3 * tri + 2]));
    sn = normalize3(add3(add3(n0, scl3(s1, f)), scl3(s2, g)));
  } else {
    f3 const z = mk3(0.0f, 0.0f, 0.0f);
    sn = normalize3(add3(add3(gn, scl3(z, f)), scl3(z, g)));
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
  *gn_out = gn;
  *sn_out = sn;
  *tan_out = tan;
  *bin_out = bin;
  return __float_as_int(g4.w);
}

// kModeAdjoint: the replay pass of xyzgpu_adjoint (same path, plus gradients).
// kModeBatch: paths of many scenes (xyzgpu_batch_*).
// kModeGuided: directions from the learned guide mixed with Lambert sampling.
// kModeImporton: directions from the light-importance histogram of the vertex
// (the reference's importance-driven tracer).
template <int kMode>
__global__ void __launch_bounds__(kThreads, kMode == kModeGuided ? 5 : 0) k_shade(WaveArgs A, int b) {
  constexpr bool kAdj = kMode == kModeAdjoint;
  constexpr bool kBatch = kMode == kModeBatch;
  constexpr bool kGuide = kMode == kModeGuided;
  constexpr bool kImp = kMode == kModeImporton;
  // mirror and metal materials exist in plain and batched renders only (the
  // other modes refuse such scenes), so the other variants carry no code for them
  constexpr bool kSpecMat = kMode == kModePlain || kMode == kModeBatch;
  if constexpr (kBatch) b = A.cursor->bounce;
  int32_t *const cnt = A.counts + b * kCountStride;
  int32_t *const cnt_next = A.counts + (b + 1) * kCountStride;
  int const n = cnt[kCExt];
  int const lane = threadIdx.x & 31;
  int const qi = b & 1, qo = qi ^ 1;
  int const warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int const nwarps = (gridDim.x * blockDim.x) >> 5;
  for (int base = warp * 32; base < n; base += nwarps * 32) {
    int const i = base + lane;
    bool push_ext = false, push_sh = false;
    int32_t slot = 0, tri = 0;
    f3 pos{}, dir{}, lpos{}, vin{}, pbv{};
    float nk2nk3 = 0.0f;
    float4 beta4{};
    uint32_t misc = 0;
    int32_t light_mat = 0;
    float rho = 1.0f;
    float4 sm4{};           // metal vertex: next-event terms for the shadow ray
    bool sh_metal = false;
    int block = 0;
    // guide_alpha is 0 at bounces without inference: Lambert sampling
    // alone, and the mixture buffer is not read
    bool const use_guide = kGuide && A.guide_alpha > 0.0f;
    GuideMix M;
    if (use_guide && i < n) load_mix(A.mix + 40 * static_cast<int64_t>(i), M);
    if (i < n) {
      slot = A.q_slot[qi][i];
      int64_t const cache_at = static_cast<int64_t>(slot) * A.cache_stride + b;
      float4 const h = (kAdj && A.hit_cache) ? A.hit_cache[cache_at] : A.hits[i];
      if (kMode == kModePlain && A.hit_cache) A.hit_cache[cache_at] = h;
      int32_t const code = __float_as_int(h.w);
      if (code >= 0) {
        tri = code >> 1;
        int const back = code & 1;
        float4 const o4 = A.q_o[qi][i], d4 = A.q_d[qi][i];
        if (kBatch) block = __float_as_int(o4.w);
        DevScene const &S = scene_of<kBatch>(A, block);
        PathParams const P = params_of<kBatch>(A, block);
        f3 const d = xyz3(d4);
        if (kGuide && b >= 1 && b - 1 < A.train_bounces) {
          // radiance gathered before this vertex: closes the previous vertex's record
          float4 const L = A.radiance[slot];
          float *rec = A.records + (static_cast<int64_t>(slot) * A.train_bounces + (b - 1)) * 16;
          rec[13] = L.x;
          rec[14] = L.y;
          rec[15] = L.z;
        }
        f3 gn, sn, tan, bin;
        int32_t const m = shading_frame(S, tri, back, h.y, h.z, &gn, &sn, &tan, &bin);
        if (!(-dot3(d, sn) <= 0.0f)) {
          pos = add3(xyz3(o4), scl3(d, h.x));
          float4 const m4 = __ldg(&S.mat[m]);
          int const kind = static_cast<int>(m4.w);  // 0 Lambert, 1 light, 2 mirror, 3 metal
          bool const is_light = kind == 1;
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
              path_pixel_sample<kBatch>(A, block, slot, &px, &smp);
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
            if (static_cast<int>(k) >= P.kmax) alive = false;
          }
          uint32_t pixel = 0, sample = 0;
          if (use_guide && alive && !is_light) finish_mix(M);
          // importance-driven: this vertex's histogram (cumulative counts
          // c[1..16], c[0] = 0), filled by k_importon_query; none beyond the
          // guided bounces
          bool const use_imp = kImp && A.imp_cdf != nullptr && alive && !is_light;
          float ic[17];
          if (use_imp) {
            ic[0] = 0.0f;
            const float4 *c4 = reinterpret_cast<const float4 *>(A.imp_cdf + 16 * static_cast<int64_t>(i));
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              float4 const v4 = c4[q];
              ic[1 + 4 * q] = v4.x;
              ic[2 + 4 * q] = v4.y;
              ic[3 + 4 * q] = v4.z;
              ic[4 + 4 * q] = v4.w;
            }
          }
          float nee_pl = 0.0f;  // guided: Lambert density of the light direction (0: no shadow ray)
          if (alive) {
            path_pixel_sample<kBatch>(A, block, slot, &pixel, &sample);
            // a mirror has no next-event estimation and leaves the throughput
            // alone (Mirror::CalculateWeightedDirectLighting, xyz/bsdf/mirror.cpp:47-51)
            if (!is_light && !(kSpecMat && kind == 2)) {
              // next-event estimation (lambert.cpp:125-156; a metal's albedo
              // enters the throughput the same way, metal.cpp:68-71)
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
                LightSample const ls = sample_light(S, P.seed, pixel, sample);
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
                    if (kAdj && A.vis_cache) {
                      // replay with cached intersections: the primal's shadow
                      // ray gave the target's distance (NaN if it was not
                      // visible); the shadow kernel's term, computed here
                      push_sh = false;
                      float const ts = A.vis_cache[static_cast<int64_t>(slot) * A.cache_stride + b];
                      if (ts > 0.0f) {
                        float const G = nk2nk3 / (ts * ts);
                        float const dimp = static_cast<float>(kInvPi * static_cast<double>(G));
                        float const dexp = 1.0f / S.light_area;
                        float const dens = dimp / dexp;
                        double const wgt = (static_cast<double>(G) * (kInvPi * kInvPi)) *
                                           static_cast<double>(1.0f / (1.0f + dens * dens));
                        float const *df = A.dfilm + 3 * static_cast<int64_t>(pixel);
                        float const gl = df[0] * static_cast<float>(static_cast<double>(pbv.x) * wgt) +
                                         df[1] * static_cast<float>(static_cast<double>(pbv.y) * wgt) +
                                         df[2] * static_cast<float>(static_cast<double>(pbv.z) * wgt);
                        if (gl != 0.0f) atomicAdd(&A.g_em[light_mat], gl);
                        f3 const pe = scl3(pbv, __ldg(&S.emission[light_mat]));
                        float4 L = A.radiance[slot];
                        L.x += static_cast<float>(static_cast<double>(pe.x) * wgt);
                        L.y += static_cast<float>(static_cast<double>(pe.y) * wgt);
                        L.z += static_cast<float>(static_cast<double>(pe.z) * wgt);
                        A.radiance[slot] = L;
                      }
                    }
                    if (use_guide) nee_pl = nk2 * static_cast<float>(kInvPi);
                    if (kImp) rho = use_imp ? importon_density(ic, v, sn, tan, bin) : 1.0f;
                    if (kSpecMat && kind == 3) {
                      // Metal::CalculateWeightedDirectLighting (metal.cpp:92-113):
                      // the Phong-lobe pdf of the light direction about the
                      // half vector, its Fresnel term and the max(nk1, nk2)
                      // normalisation travel with the shadow ray
                      float const shin = __ldg(&S.shininess[m]);
                      f3 const hv = neg3(normalize3(add3(v, d)));
                      float const hk = -dot3(hv, v);
                      float const nh = dot3(sn, hv);
                      float const nk1 = -dot3(sn, d);
                      float const fsn_m = static_cast<float>(static_cast<double>(shin + 1.0f) * (kInvPi / 8.0) *
                                                             static_cast<double>(powf(nh, shin)) /
                                                             static_cast<double>(hk));
                      float const kf = static_cast<float>(static_cast<double>(fsn_m) /
                                                          static_cast<double>(fmaxf(nk1, nk2)) *
                                                          static_cast<double>(fake_fresnel(hk)));
                      sm4 = make_float4(nk2, nk3, fsn_m, kf);
                      sh_metal = true;
                    }
                  }
                }
              }
            }
            PathRng rng;
            rng.init(P.seed, pixel, sample, dim);
            // guided: the product of the guide / Lambert density ratios so far
            // (radiance.w), so that Russian roulette sees the throughput the
            // path would have with Lambert sampling and does not end paths
            // for being sent towards bright regions
            float rr_scale = 1.0f;
            if (kGuide) {
              float const w = reinterpret_cast<const float *>(A.radiance + slot)[3];
              rr_scale = w > 0.0f ? w : 1.0f;
            }
            // Russian roulette (scene_pathtracing.cpp:128-137)
            if (static_cast<int>(k) - 1 >= P.rr_start) {
              float const ty = kGuide ? beta.y * rr_scale : beta.y;
              if (ty < P.rr_threshold) {
                float const q = ty / P.rr_threshold;
                if (rng.next() >= q) {
                  alive = false;
                } else {
                  beta = scl3(beta, 1.0f / q);
                }
              }
            }
            if (alive && is_light) alive = false;  // Light::NextScatteringDirection
            if (kGuide) {
              // one-sample MIS of the guide (probability alpha) and Lambert
              // sampling: the path weight uses the mixture density; one pass
              // over the lobes gives it for the sampled and the light direction
              f3 wd = mk3(0.0f, 0.0f, 1.0f);
              bool cont = false;
              float cs = 0.0f;
              if (alive) {
                if (use_guide && rng.next() < A.guide_alpha) {
                  float const ul = rng.next();
                  float const u1 = rng.next();
                  float const u2 = rng.next();
                  wd = mix_sample(M, ul, u1, u2);
                } else {
                  // cosine-weighted (the density below is evaluated at the
                  // direction produced, so the fast sincos is exact enough)
                  float const mu_phi = rng.next();
                  float const mu_theta = rng.next();
                  float sp, cp;
                  __sincosf(static_cast<float>(2.0 * kPi) * mu_phi, &sp, &cp);
                  float const sin_t = sqrtf(1.0f - mu_theta);
                  wd = add3(add3(scl3(tan, sin_t * cp), scl3(bin, sin_t * sp)), scl3(sn, sqrtf(mu_theta)));
                }
                cs = dot3(wd, sn);
                cont = cs > 0.0f && dot3(wd, gn) > 0.0f;
              }
              float pm_light = 0.0f, pm_wd = 0.0f;
              if (use_guide && (cont || nee_pl > 0.0f)) mix_pdf2(M, neg3(vin), wd, &pm_light, &pm_wd);
              if (nee_pl > 0.0f) rho = (A.guide_alpha * pm_light + (1.0f - A.guide_alpha) * nee_pl) / nee_pl;
              if (cont) {
                float const pdf = use_guide ? A.guide_alpha * pm_wd +
                                                  (1.0f - A.guide_alpha) * cs * static_cast<float>(kInvPi)
                                            : cs * static_cast<float>(kInvPi);
                float const lambert = cs * static_cast<float>(kInvPi);
                beta = scl3(beta, lambert / pdf);
                reinterpret_cast<float *>(A.radiance + slot)[3] = rr_scale * (pdf / lambert);
                dir = wd;
                push_ext = true;
                beta4 = make_float4(beta.x, beta.y, beta.z, pdf);
                misc = pack_misc(rng.dim, k, 0u);
                if (b < A.train_bounces) {
                  float *rec = A.records + (static_cast<int64_t>(slot) * A.train_bounces + b) * 16;
                  float const r[13] = {pos.x, pos.y, pos.z, sn.x, sn.y, sn.z, wd.x, wd.y, wd.z, pdf,
                                       beta.x, beta.y, beta.z};
                  for (int t = 0; t < 13; ++t) rec[t] = r[t];
                  // the next vertex (if the ray hits one) replaces these
                  rec[13] = rec[14] = rec[15] = __int_as_float(0x7fc00000);
                }
              }
            } else if (kImp && use_imp && alive) {
              // Lambert::NextScatteringDirection with importons
              // (lambert.cpp:243-257) -> ImportanceQuery::SetDiffusedVector
              // (photonmap.cpp:403-439): a bin by the cumulative counts, then
              // (cos^2 theta, phi) uniform in it; the throughput is divided by
              // the bin's density and the sampling density is density cos / pi
              float const value = ic[16] * rng.next();
              int lo = 0, hi = 17;  // upper_bound over c[0..16]
              while (lo < hi) {
                int const mid = (lo + hi) >> 1;
                if (!(value < ic[mid]))
                  lo = mid + 1;
                else
                  hi = mid;
              }
              int const nb = lo - 1;
              int const bu = nb / 8, bv = nb % 8;
              float const mu_u = (static_cast<float>(bu) + rng.next()) / 2.0f;
              float const mu_v = (static_cast<float>(bv) + rng.next()) / 8.0f;
              float const cos_t = sqrtf(mu_u);
              float const sin_t = sqrtf(1.0f - mu_u);
              float const phi = static_cast<float>(2.0 * kPi) * mu_v;
              dir = add3(add3(scl3(tan, sin_t * cosf(phi)), scl3(bin, sin_t * sinf(phi))), scl3(sn, cos_t));
              float const dens = 16.0f * (ic[nb + 1] - ic[nb]) / ic[16];
              float const fsn = static_cast<float>(static_cast<double>(dens * cos_t) * kInvPi);
              beta = scl3(beta, 1.0f / dens);
              if (dot3(dir, gn) > 0.0f) {
                push_ext = true;
                beta4 = make_float4(beta.x, beta.y, beta.z, fsn);
                misc = pack_misc(rng.dim, k, 0u);
              }
            } else if (kSpecMat && alive && kind == 2) {
              // Mirror::NextScatteringDirection (mirror.cpp:53-71): the
              // reflection about the shading normal, a specular bounce
              float const ct = -dot3(d, sn);
              dir = add3(d, scl3(sn, 2.0f * ct));
              if (dot3(dir, gn) > 0.0f) {
                push_ext = true;
                beta4 = make_float4(beta.x, beta.y, beta.z, 1.0f);
                misc = pack_misc(rng.dim, k, 1u);
              }
            } else if (kSpecMat && alive && kind == 3) {
              // Metal::NextScatteringDirection (metal.cpp:122-159) with
              // ComputeGlossyHalfwayVector (xyz/stdafx.hpp:154-168): a half
              // vector from the Phong lobe (g++ passes the first draw to rMuPhi),
              // the mirror direction about it; throughput times
              // Fresnel / max(nk1, nk2) * nk2; not specular (CONFIG_EXPLICIT_GLOSSY)
              float const mu_phi = rng.next();
              float const mu_theta = rng.next();
              float const shin = __ldg(&S.shininess[m]);
              float const rphi = static_cast<float>(2.0 * kPi) * mu_phi;
              float const cos_t = powf(mu_theta, 1.0f / shin);
              float const sin_t = sqrtf(1.0f - cos_t * cos_t);
              f3 const hv = add3(add3(scl3(tan, sin_t * cosf(rphi)), scl3(bin, sin_t * sinf(rphi))), scl3(sn, cos_t));
              float const nk1 = -dot3(sn, d);
              float const hk = -dot3(hv, d);
              dir = add3(d, scl3(hv, 2.0f * hk));
              float const nk2 = dot3(sn, dir);
              if (!((nk2 <= 0.0f) || (dot3(gn, dir) <= 0.0f))) {
                beta = scl3(beta, fake_fresnel(hk) / fmaxf(nk1, nk2) * nk2);
                float const fsn = static_cast<float>(static_cast<double>(shin + 1.0f) * (kInvPi / 8.0) *
                                                     static_cast<double>(powf(cos_t, shin)) / static_cast<double>(hk));
                push_ext = true;
                beta4 = make_float4(beta.x, beta.y, beta.z, fsn);
                misc = pack_misc(rng.dim, k, 0u);
              }
            } else if (alive) {
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
      A.s_o[js] = make_float4(lpos.x, lpos.y, lpos.z, kBatch ? __int_as_float(block) : __int_as_float(0x7f800000));
      A.s_d[js] = make_float4(vin.x, vin.y, vin.z, nk2nk3);
      A.s_pb[js] = make_float4(pbv.x, pbv.y, pbv.z, __int_as_float(slot));
      A.s_target[js] = tri;
      if (kAdj) A.s_slot[js] = light_mat;
      if (kGuide || kImp) A.s_slot[js] = __float_as_int(rho);
      if (sh_metal) A.s_m[js] = sm4;
    }
    int32_t const je = warp_append(&cnt_next[kCExt], push_ext);
    if (push_ext) {
      A.q_o[qo][je] = make_float4(pos.x, pos.y, pos.z, kBatch ? __int_as_float(block) : kRayTMin);
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
          bool const is_light = __ldg(&S.mat[m]).w == 1.0f;
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
    float *f = film + 3 * film_pixel(A, A.p0 + p);
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
    float *f = film + 3 * film_pixel(A, A.p0 + p);
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

// Batched film: one thread per pixel of each block of the wave; the block's
// samples are added in sample order into the job's film.
__global__ void __launch_bounds__(kThreads) k_film_batch(WaveArgs A) {
  int64_t const stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
  BatchWave const wv = A.cursor->w;
  for (int64_t q = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; q < wv.film_threads; q += stride) {
    int lo = wv.first_block, hi = wv.first_block + wv.n_blocks - 1;
    while (lo < hi) {
      int const mid = (lo + hi + 1) >> 1;
      if (A.blocks[mid].pix_off <= q)
        lo = mid;
      else
        hi = mid - 1;
    }
    const WaveBlock &B = A.blocks[lo];
    const BatchJob &J = A.jobs[B.job];
    int64_t const pl = q - B.pix_off;
    float *f = J.film + 3 * static_cast<int64_t>(tile_pixel(pl, J.W, J.tile));
    float fx = f[0], fy = f[1], fz = f[2];
    for (int s = 0; s < B.ns; ++s) {
      float4 const L = A.radiance[B.slot_off + static_cast<int64_t>(s) * B.npix + pl];
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


// Camera set-up as ThinLensCamera::Reset (thinlenscamera.cpp:71-90) and
// Scene::SetDimension (scene.hpp:226-230), in float on the host.
inline CamDev camera_setup(const xyzgpu_camera &cam, int width, int height) {
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

template <class K>
int occupancy_grid(K kernel, int device) {
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess ||
      per_sm <= 0)
    per_sm = 4;
  return per_sm * sm_count(device);
}

}  // namespace
}  // namespace xyzgpu
