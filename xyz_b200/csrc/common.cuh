// Device-side building blocks shared by the traversal and render kernels.
//
// Arithmetic that decides which triangle a ray hits, where a path goes and
// what it carries is written in the reference's operation order
// (hi::dot = a0*b0 + a1*b1 + a2*b2, hi::cross, hi::normalize = a * (1/sqrt),
// libhi/hi/math/vector3.hpp:120-131, math.hpp:155-157) and these translation
// units are compiled with --fmad=false and IEEE division / square root, so a
// path computed here rounds like the reference's float code.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kdtree.h"

namespace xyzgpu {

#define XYZ_DEV __device__ __forceinline__
#define XYZ_HD __host__ __device__ __forceinline__

constexpr float kEpsilon = 1e-6f;   // xyz/stdafx.hpp:36
constexpr float kRayTMin = 1e-5f;   // xyz/geom/intersection.hpp:12
constexpr double kInvPi = 0.318309886183790671538;  // M_1_PI
constexpr double kPi = 3.14159265358979323846;

struct f3 {
  float x, y, z;
};

XYZ_HD f3 mk3(float x, float y, float z) { return f3{x, y, z}; }
XYZ_HD f3 add3(f3 a, f3 b) { return f3{a.x + b.x, a.y + b.y, a.z + b.z}; }
XYZ_HD f3 sub3(f3 a, f3 b) { return f3{a.x - b.x, a.y - b.y, a.z - b.z}; }
XYZ_HD f3 mul3(f3 a, f3 b) { return f3{a.x * b.x, a.y * b.y, a.z * b.z}; }
XYZ_HD f3 scl3(f3 a, float s) { return f3{a.x * s, a.y * s, a.z * s}; }
XYZ_HD f3 neg3(f3 a) { return f3{-a.x, -a.y, -a.z}; }
XYZ_HD float dot3(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
XYZ_HD f3 cross3(f3 a, f3 b) {
  return f3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
XYZ_HD float comp3(f3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
XYZ_DEV f3 normalize3(f3 a) {
  float const r = 1.0f / sqrtf(dot3(a, a));
  return scl3(a, r);
}
XYZ_HD f3 xyz3(float4 v) { return f3{v.x, v.y, v.z}; }

// ---------------------------------------------------------------- random
// Philox4x32-10 (Salmon et al., SC'11).  Stream layout in include/xyzgpu.h.
XYZ_HD void philox4x32_10(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0,
                          uint32_t k1, uint32_t out[4]) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
#ifdef __CUDA_ARCH__
    uint32_t const hi0 = __umulhi(0xD2511F53u, c0), lo0 = 0xD2511F53u * c0;
    uint32_t const hi1 = __umulhi(0xCD9E8D57u, c2), lo1 = 0xCD9E8D57u * c2;
#else
    uint64_t const p0 = static_cast<uint64_t>(0xD2511F53u) * c0;
    uint64_t const p1 = static_cast<uint64_t>(0xCD9E8D57u) * c2;
    uint32_t const hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    uint32_t const hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
#endif
    uint32_t const n0 = hi1 ^ c1 ^ k0;
    uint32_t const n2 = hi0 ^ c3 ^ k1;
    c0 = n0;
    c1 = lo1;
    c2 = n2;
    c3 = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  out[0] = c0;
  out[1] = c1;
  out[2] = c2;
  out[3] = c3;
}

XYZ_HD float u01_from_bits(uint32_t w) {
  return static_cast<float>(w >> 8) * (1.0f / 16777216.0f);
}

// Sequential reader of one path's dimensions with a one-block cache.
struct PathRng {
  uint32_t k0, k1, pixel, sample, dim, blk;
  uint32_t w[4];
  XYZ_DEV void init(uint64_t seed, uint32_t p, uint32_t s, uint32_t d) {
    k0 = static_cast<uint32_t>(seed);
    k1 = static_cast<uint32_t>(seed >> 32);
    pixel = p;
    sample = s;
    dim = d;
    blk = 0xffffffffu;
  }
  XYZ_DEV float next() {
    uint32_t const b = dim >> 2;
    if (b != blk) {
      philox4x32_10(pixel, sample, b, 0u, k0, k1, w);
      blk = b;
    }
    uint32_t const j = dim & 3u;
    uint32_t const bits = j == 0 ? w[0] : (j == 1 ? w[1] : (j == 2 ? w[2] : w[3]));
    ++dim;
    return u01_from_bits(bits);
  }
};

// ------------------------------------------------------------ scene view
// Device pointers of one scene (owned by the host-side Scene object).
struct DevScene {
  const float4 *tri;      // 3 per triangle: (v0, n.x) (e1, n.y) (e2, n.z), n = cross(e2, e1)
  const float4 *tri_ng;   // (normalize(n), material id bits)
  const float4 *tri_sn;   // 3 per triangle: shading n0, s1 = n1 - n0, s2 = n2 - n0 (or null)
  const float4 *mat;      // (albedo xyz, kind: 0 Lambert, 1 light, 2 mirror, 3 metal)
  const float *shininess; // per material (metal lobe exponent)
  int has_metal;          // a metal material exists (shadow rays check their vertex's kind)
  const float *emission;  // per-material scale of the light's emitted power (1 by default)
  const int32_t *lights;  // light triangle ids, triangle order
  const float *cdf;       // n_lights + 1 prefix sums of light areas, cdf[0] = 0
  const uint2 *nodes;
  const int32_t *refs;
  int n_lights;
  float light_area;
  f3 power;
  f3 bmin, bmax;
  const float *spd_albedo;  // 31 bins per material, or null (spectral modes need it)
  float spd_light[31];      // light power spectrum (spectral modes)
};

}  // namespace xyzgpu
