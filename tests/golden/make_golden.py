"""Generates the golden fixtures in this directory from the reference renderer's
own path tracer (oracle/_ref, built from the reference sources by
`make -C oracle`).  Run from the repository root:

    python tests/golden/make_golden.py

Each .npz holds the scene arrays it was made from, so the tests do not depend
on the scene generators staying unchanged.  Light power: the reference lights
every scene with its Mercury-arc power (xyz/core/config.hpp:81-95); the
fixtures record that power and the films are the reference's raw output.
"""

from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle.refbind import RefLib  # noqa: E402
from xyz_b200 import scenes  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def scene_arrays(sd):
    d = dict(positions=sd.positions, tris=sd.tris, tri_mat=sd.tri_mat, albedo_xyz=sd.albedo_xyz,
             is_light=sd.is_light,
             cam=np.array(list(sd.camera.eye) + list(sd.camera.at) +
                          [sd.camera.film_size, sd.camera.focal_length, sd.camera.f_number,
                           float(sd.camera.pinhole)], np.float32))
    if sd.normals is not None:
        d["normals"] = sd.normals
    return d


def make_trace(name, sd, n_rays, seed):
    R = RefLib(pinhole=True)
    R.scene_create(sd)
    org, d = scenes.random_rays(sd, n_rays, seed=seed)
    tri, t, f, g, back = R.trace(org, d, nthreads=1)
    np.savez_compressed(os.path.join(OUT, name), org=org, dir=d, tri=tri, t=t, f=f, g=g, back=back,
                        **scene_arrays(sd))
    print(name, "hit fraction", (tri >= 0).mean())


def make_film(name, sd, W, H, spp, seed, max_depth, pts):
    R = RefLib(pinhole=sd.camera.pinhole)
    R.scene_create(sd)
    R.set_camera(sd.camera, W, H)
    R.set_path_params(max_depth=max_depth)
    film = R.render(spp, seed=seed, nthreads=1)
    paths = []
    for (px, py, s) in pts:
        v, dims = R.eval_path(px, py, s, seed)
        paths.append([px, py, s, dims, v[0], v[1], v[2]])
    np.savez_compressed(os.path.join(OUT, name), film=film, W=W, H=H, spp=spp, seed=seed,
                        max_depth=max_depth, power_ref=R.light_power_xyz(),
                        paths=np.array(paths, np.float64), **scene_arrays(sd))
    print(name, "mean", film.mean(axis=(0, 1)) / spp)


def main():
    rng = np.random.default_rng(0)
    make_trace("cornell_trace.npz", scenes.cornell_box(), 4096, seed=1)
    make_trace("spheres_l3_trace.npz", scenes.spheres_scene(level=3, n_spheres=2), 4096, seed=2)
    pts = [(int(rng.integers(32)), int(rng.integers(24)), int(rng.integers(8))) for _ in range(32)]
    make_film("cornell_pinhole_film.npz", scenes.cornell_box(pinhole=True), 32, 24, 8, 5, 8, pts)
    make_film("cornell_thinlens_film.npz", scenes.cornell_box(pinhole=False), 32, 24, 8, 6, 15, pts)
    make_film("spheres_l2_film.npz", scenes.spheres_scene(level=2, n_spheres=2), 32, 24, 4, 7, 10, pts)


if __name__ == "__main__":
    main()
