"""Generates guide_reference_fp64.npz: the converged reference image of the
path-guiding benchmark's scene from the CPU oracle (the C restatement of the
reference's PathTracer::run estimator, oracle/xyz_oracle.c, itself pinned to
the reference's own renderer), with per-pixel sums in double.  Run from the
repository root (a few minutes on 8 cores):

    python tests/golden/make_guide_reference.py

Scene: the occluded room (196,146 triangles, light only through a 0.1 m gap),
1024 x 1024 pinhole camera of the benchmark, max depth 10, Russian roulette
0.2.  Pixels: the 32 x 32 grid x, y = 16, 48, ..., 1008, which lies on the
benchmark's measured rows.  65,536 samples per pixel, Philox seed 77.  Stored:
the pixel list, per pixel (sum X, sum Y, sum Z, sum Y^2) in float64, and a
SHA-256 of the scene arrays so a changed scene generator is detected.
"""

from __future__ import annotations

import hashlib
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refbind import PortLib  # noqa: E402
from xyz_b200 import scenes  # noqa: E402

OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "guide_reference_fp64.npz")
W = H = 1024
SPP = 65536
SEED = 77
DEPTH = 10
CAMERA = ((0.0, 1.5, 1.2), (0.0, 1.1, -2.0), 60.0)   # eye, gaze point, vertical fov (degrees)


def scene_digest(sd) -> str:
    h = hashlib.sha256()
    for a in (sd.positions, sd.tris, sd.tri_mat, sd.albedo_xyz, sd.is_light, sd.light_power_xyz):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def pixel_grid():
    xs = np.arange(16, W, 32, dtype=np.int32)
    px, py = np.meshgrid(xs, xs)
    return px.ravel(), py.ravel()


def main():
    sd = scenes.occluded_room()
    cam = scenes.Camera.with_fov(*CAMERA, pinhole=True)
    P = PortLib()
    P.set_spectral(0, 1)
    P.scene_create(sd)
    P.set_camera(cam, W, H)
    P.set_path_params(max_depth=DEPTH)
    px, py = pixel_grid()
    acc = np.zeros((px.size, 4), np.float64)
    t0 = time.time()
    chunk = 4096
    for s0 in range(0, SPP, chunk):
        P.render_pixels(px, py, chunk, seed=SEED, s0=s0, acc=acc)
        print(f"{s0 + chunk} spp, {time.time() - t0:.0f} s", flush=True)
    np.savez_compressed(OUT, px=px, py=py, acc=acc, spp=SPP, seed=SEED, max_depth=DEPTH, width=W, height=H,
                        camera=np.array(CAMERA[0] + CAMERA[1] + (CAMERA[2],), np.float64),
                        scene_sha256=scene_digest(sd))
    print("wrote", OUT)


if __name__ == "__main__":
    main()
