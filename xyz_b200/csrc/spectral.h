// Spectral tables and wavelength sampling for the hero-wavelength film
// modes (host and device).
//
// The reference's spectra are 31 bins at 400, 410, ..., 700 nm
// (libhi/hi/image/spectrum.hpp:14).  Its spectral renderer draws one bin per
// path uniformly and writes XYZ = L * 31 * CMF[bin]
// (renderer/core/SceneStrategy.cpp:17-20, 148; libhi/hi/image/spectrum.cpp:
// 561-567).  Here a path carries H hero wavelengths u_j = frac(u_h + j / H)
// (j < H), each an equally weighted stratified sample:
//   binned      bin_j = floor(31 u_j) over 400..700 nm (H = 1 is the reference's
//               own estimator), XYZ = sum_j L_j * 31 * CMF[bin_j] / H
//   continuous  lambda_j = 380 + 340 u_j nm; spectra and CMF interpolated
//               linearly between bin centres and clamped to the end bins
//               (basic_spectrum::Sample, spectrum.cpp:148-165),
//               XYZ = sum_j L_j * 34 * CMF(lambda_j) / H (34 = 340 nm / 10 nm bins).
#pragma once

#include "common.cuh"

namespace xyzgpu {

constexpr int kSpecBins = 31;
constexpr int kMaxHero = 4;

// CIE 1931 colour-matching functions, Glassner's 10 nm table divided by
// 9.80328 (libhi/hi/image/spectrum.cpp:505-533): each entry is the double
// quotient rounded to float, as the reference's float constructor stores it.
#define XYZGPU_D(v) static_cast<float>((v) / 9.80328)
__constant__ static float c_cmf[3][kSpecBins] = {
    {XYZGPU_D(0.014), XYZGPU_D(0.044), XYZGPU_D(0.134), XYZGPU_D(0.284), XYZGPU_D(0.348),
     XYZGPU_D(0.336), XYZGPU_D(0.291), XYZGPU_D(0.195), XYZGPU_D(0.096), XYZGPU_D(0.032),
     XYZGPU_D(0.005), XYZGPU_D(0.009), XYZGPU_D(0.063), XYZGPU_D(0.166), XYZGPU_D(0.290),
     XYZGPU_D(0.433), XYZGPU_D(0.595), XYZGPU_D(0.762), XYZGPU_D(0.916), XYZGPU_D(1.026),
     XYZGPU_D(1.062), XYZGPU_D(1.003), XYZGPU_D(0.854), XYZGPU_D(0.642), XYZGPU_D(0.448),
     XYZGPU_D(0.284), XYZGPU_D(0.165), XYZGPU_D(0.087), XYZGPU_D(0.047), XYZGPU_D(0.023),
     XYZGPU_D(0.011)},
    {XYZGPU_D(0.000), XYZGPU_D(0.001), XYZGPU_D(0.004), XYZGPU_D(0.012), XYZGPU_D(0.023),
     XYZGPU_D(0.038), XYZGPU_D(0.060), XYZGPU_D(0.091), XYZGPU_D(0.139), XYZGPU_D(0.208),
     XYZGPU_D(0.323), XYZGPU_D(0.503), XYZGPU_D(0.710), XYZGPU_D(0.862), XYZGPU_D(0.954),
     XYZGPU_D(0.995), XYZGPU_D(0.995), XYZGPU_D(0.952), XYZGPU_D(0.870), XYZGPU_D(0.757),
     XYZGPU_D(0.631), XYZGPU_D(0.503), XYZGPU_D(0.381), XYZGPU_D(0.265), XYZGPU_D(0.175),
     XYZGPU_D(0.107), XYZGPU_D(0.061), XYZGPU_D(0.032), XYZGPU_D(0.017), XYZGPU_D(0.008),
     XYZGPU_D(0.004)},
    {XYZGPU_D(0.068), XYZGPU_D(0.207), XYZGPU_D(0.646), XYZGPU_D(1.386), XYZGPU_D(1.747),
     XYZGPU_D(1.772), XYZGPU_D(1.669), XYZGPU_D(1.288), XYZGPU_D(0.813), XYZGPU_D(0.465),
     XYZGPU_D(0.272), XYZGPU_D(0.158), XYZGPU_D(0.078), XYZGPU_D(0.042), XYZGPU_D(0.020),
     XYZGPU_D(0.009), XYZGPU_D(0.004), XYZGPU_D(0.002), XYZGPU_D(0.002), XYZGPU_D(0.001),
     XYZGPU_D(0.001), XYZGPU_D(0.000), XYZGPU_D(0.000), XYZGPU_D(0.000), XYZGPU_D(0.000),
     XYZGPU_D(0.000), XYZGPU_D(0.000), XYZGPU_D(0.000), XYZGPU_D(0.000), XYZGPU_D(0.000),
     XYZGPU_D(0.000)},
};
#undef XYZGPU_D

// u_j = frac(u_h + j / H)
XYZ_HD float hero_u(float uh, int j, int H) {
  float u = uh + static_cast<float>(j) / static_cast<float>(H);
  if (u >= 1.0f) u -= 1.0f;
  return u;
}

XYZ_HD int hero_bin(float u) {
  int b = static_cast<int>(u * static_cast<float>(kSpecBins));
  return b > kSpecBins - 1 ? kSpecBins - 1 : b;
}

// basic_spectrum::Sample parameter of wavelength 380 + 340 u (bin centres at
// 400 + 10 i nm sit at (i + 0.5) / 31).
XYZ_HD float hero_sample_param(float u) {
  float const lambda = 380.0f + 340.0f * u;
  return (lambda - 395.0f) / 310.0f;
}

// basic_spectrum::Sample (spectrum.cpp:148-165) of a 31-entry table.
template <class Get>
XYZ_HD float spectrum_sample(float p, Get get) {
  p *= static_cast<float>(kSpecBins);
  p -= 0.5f;
  if (p <= 0.0f) return get(0);
  if (p >= static_cast<float>(kSpecBins - 1)) return get(kSpecBins - 1);
  int const k = static_cast<int>(p);
  p -= static_cast<float>(k);
  float const a = get(k), b = get(k + 1);
  return a + (b - a) * p;
}

}  // namespace xyzgpu
