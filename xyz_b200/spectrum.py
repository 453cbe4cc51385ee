"""Spectral tables and conversions used by the tracer's film.

The renderer's colour space is CIE XYZ over 31 bins at 400, 410, ..., 700 nm.
The colour-matching functions are the CIE 1931 2-degree observer as tabulated
by Glassner ("Principles of Digital Image Synthesis", 1995), normalised by
9.80328 exactly as the reference renderer stores them
(libhi/hi/image/spectrum.cpp:505-533); `spd_to_xyz` is the full dot product of
libhi/hi/image/spectrum.cpp:554-559 and `bin_to_xyz` the single-bin form of
spectrum.cpp:561-567 (value * 31 * CMF[i]).
"""

from __future__ import annotations

import numpy as np

N_BINS = 31
LAMBDA_MIN_NM = 400.0
LAMBDA_STEP_NM = 10.0
CMF_NORMALISER = 9.80328

_CMF_RAW = np.array(
    [
        [0.014, 0.044, 0.134, 0.284, 0.348, 0.336, 0.291, 0.195, 0.096, 0.032,
         0.005, 0.009, 0.063, 0.166, 0.290, 0.433, 0.595, 0.762, 0.916, 1.026,
         1.062, 1.003, 0.854, 0.642, 0.448, 0.284, 0.165, 0.087, 0.047, 0.023,
         0.011],
        [0.000, 0.001, 0.004, 0.012, 0.023, 0.038, 0.060, 0.091, 0.139, 0.208,
         0.323, 0.503, 0.710, 0.862, 0.954, 0.995, 0.995, 0.952, 0.870, 0.757,
         0.631, 0.503, 0.381, 0.265, 0.175, 0.107, 0.061, 0.032, 0.017, 0.008,
         0.004],
        [0.068, 0.207, 0.646, 1.386, 1.747, 1.772, 1.669, 1.288, 0.813, 0.465,
         0.272, 0.158, 0.078, 0.042, 0.020, 0.009, 0.004, 0.002, 0.002, 0.001,
         0.001, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000, 0.000,
         0.000],
    ],
    dtype=np.float64,
)

# float32 table, each entry the double quotient rounded once (as the reference's
# `basic_spectrum(0.014 / 9.80328, ...)` float constructor does).
XYZ_CMF = (_CMF_RAW / CMF_NORMALISER).astype(np.float32)


def spd_to_xyz(spd) -> np.ndarray:
    """Full 31-bin dot product with the CMF, in float32 (bin order)."""
    spd = np.asarray(spd, dtype=np.float32)
    out = np.zeros(3, dtype=np.float32)
    for c in range(3):
        acc = np.float32(0.0)
        for i in range(N_BINS):
            acc = np.float32(acc + np.float32(spd[i] * XYZ_CMF[c, i]))
        out[c] = acc
    return out


def bin_to_xyz(i: int, value: float) -> np.ndarray:
    """XYZ of a single-bin sample: value * 31 * CMF[:, i]."""
    v = np.float32(np.float32(value) * np.float32(N_BINS))
    return (v * XYZ_CMF[:, i]).astype(np.float32)


def flat_spd_xyz(radiance: float = 1.0) -> np.ndarray:
    """XYZ of a spectrally flat source of the given per-bin value."""
    return spd_to_xyz(np.full(N_BINS, radiance, dtype=np.float32))


def ccir601_rgb_to_xyz(rgb) -> np.ndarray:
    """Linear RGB -> XYZ with the CCIR 601-1 primaries the reference's MQO
    loader uses for material colours (libhi/hi/image/color_space.hpp:58-67),
    clamped to [0, 1] per channel as xyz/core/scene_mqo.cpp clamps albedos."""
    r, g, b = (np.float32(c) for c in rgb)
    x = np.float32(np.float32(0.6069) * r + np.float32(0.1735) * g + np.float32(0.2003) * b)
    y = np.float32(np.float32(0.2989) * r + np.float32(0.5866) * g + np.float32(0.1145) * b)
    z = np.float32(np.float32(0.0000) * r + np.float32(0.0661) * g + np.float32(1.1162) * b)
    return np.clip(np.array([x, y, z], dtype=np.float32), 0.0, 1.0)


def rgb_to_spd(rgb) -> np.ndarray:
    """31-bin spectrum of a linear RGB colour by the reference's Gaussian-basis
    fit (libhi/hi/image/spectrum.cpp:574-626): three Gaussians centred at
    641, 508 and 426 nm whose widths narrow from 150 to 80 nm with the colour's
    saturation, weighted so that the spectrum's XYZ (through the CMF) equals
    the colour's CCIR 601-1 XYZ (float32 arithmetic)."""
    f32 = np.float32
    r, g, b = (f32(c) for c in rgb)
    lam_c = np.array([641, 508, 426], dtype=np.float32)
    smin, smax = f32(80), f32(150)
    int12 = f32(0) if (r + g) == 0 else f32(abs(r - g) / (r + g))
    int23 = f32(0) if (b + g) == 0 else f32(abs(b - g) / (b + g))
    sigma = np.zeros(3, np.float32)
    sigma[0] = smax + (smin - smax) * int12
    sigma[1] = smax + (smin - smax) * int23
    sigma[2] = min(sigma[0], sigma[1])
    inv_sigma = (f32(1) / np.sqrt(f32(2 * np.pi) * sigma)).astype(np.float32)
    lam = (400 + 10 * np.arange(N_BINS)).astype(np.float32)
    f = np.zeros((3, N_BINS), np.float32)
    for i in range(3):
        x = ((lam - lam_c[i]) / sigma[i]).astype(np.float32)
        f[i] = (np.exp((x * x) / f32(-2)) * inv_sigma[i]).astype(np.float32)
    a = np.array([[float(np.dot(f[i].astype(np.float64), XYZ_CMF[c].astype(np.float64))) for c in range(3)]
                  for i in range(3)])
    xyz = np.array([0.6069 * r + 0.1735 * g + 0.2003 * b,
                    0.2989 * r + 0.5866 * g + 0.1145 * b,
                    0.0000 * r + 0.0661 * g + 1.1162 * b], dtype=np.float64)
    # SolveLinearSystem (libhi/hi/math/vector3.hpp:221-240): xyz = sum_i w_i a_i
    w = np.linalg.solve(a.T, xyz)
    return (w[:, None] * f.astype(np.float64)).sum(axis=0).astype(np.float32)
