"""Shared test helpers: oracle loading and fixture-to-scene conversion."""

import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def ensure_port():
    """Builds oracle/_port/libxyzport.so if missing (plain C, gcc only)."""
    from oracle import refbind
    if not refbind.port_available():
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "port"], check=True,
                       stdout=subprocess.DEVNULL)
    return refbind.PortLib()


def ref_lib(pinhole):
    from oracle import refbind
    if not refbind.ref_available(pinhole):
        return None
    return refbind.RefLib(pinhole=pinhole)


def load_fixture(name):
    from xyz_b200.scenes import Camera, SceneData
    z = np.load(os.path.join(GOLDEN, name))
    cam = z["cam"]
    sd = SceneData(z["positions"], z["tris"], z["tri_mat"], z["albedo_xyz"], z["is_light"],
                   np.zeros(3, np.float32), normals=z["normals"] if "normals" in z else None,
                   camera=Camera(tuple(cam[0:3]), tuple(cam[3:6]), float(cam[6]), float(cam[7]),
                                 float(cam[8]), bool(cam[9] > 0.5)))
    if "power_ref" in z:
        sd.light_power_xyz = z["power_ref"].astype(np.float32)
    return sd, z


def grazing_mask(sd, org, d, tri, f, g, eps=1e-4):
    """Rays whose hit is within `eps` of a triangle edge (barycentrics) or at a
    near-tangent angle: there, the closest triangle depends on rounding."""
    m = np.zeros(tri.shape[0], bool)
    hit = tri >= 0
    m[hit] |= (f[hit] < eps) | (g[hit] < eps) | (f[hit] + g[hit] > 1 - eps)
    p = sd.positions.astype(np.float64)
    t = sd.tris[np.maximum(tri, 0)]
    n = np.cross(p[t[:, 2]] - p[t[:, 0]], p[t[:, 1]] - p[t[:, 0]])
    n /= np.maximum(np.linalg.norm(n, axis=1, keepdims=True), 1e-30)
    cosang = np.abs((n * d).sum(axis=1))
    m[hit] |= cosang[hit] < 1e-3
    return m
