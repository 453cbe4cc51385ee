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


def read_hdr(path):
    """Radiance .hdr reader (header, then flat or run-length scanlines):
    returns (header lines, (rows, W, 4) uint8 in file order)."""
    data = open(path, "rb").read()
    end = data.index(b"\n\n")
    head = data[:end].decode().split("\n")
    nl = data.index(b"\n", end + 2)
    res = data[end + 2:nl].decode().split()
    H, W = int(res[1]), int(res[3])
    pos = nl + 1
    img = np.zeros((H, W, 4), np.uint8)
    for r in range(H):
        if 8 <= W <= 0x7FFF:
            assert data[pos] == 2 and data[pos + 1] == 2 and (data[pos + 2] << 8 | data[pos + 3]) == W
            pos += 4
            for c in range(4):
                x = 0
                while x < W:
                    code = data[pos]
                    pos += 1
                    if code > 128:
                        n = code - 128
                        img[r, x:x + n, c] = data[pos]
                        pos += 1
                    else:
                        n = code
                        assert n > 0
                        img[r, x:x + n, c] = np.frombuffer(data[pos:pos + n], np.uint8)
                        pos += n
                    x += n
                assert x == W
        else:
            img[r] = np.frombuffer(data[pos:pos + 4 * W], np.uint8).reshape(W, 4)
            pos += 4 * W
    assert pos == len(data)
    return head + [" ".join(res)], img


def sample_films(seed=0):
    """Films (H, W, 3) of XYZ sums for the output formats: smooth, saturated
    (negative RGB components), dark, very bright, with zeros and a NaN."""
    rng = np.random.default_rng(seed)
    H, W = 19, 37
    base = rng.uniform(0.0, 2.0, (H, W, 3)).astype(np.float32)
    base[0] = 0.0
    base[1, :, 0] = rng.uniform(0.0, 0.05, W)         # saturated: X small, Y large
    base[1, :, 1] = rng.uniform(1.0, 3.0, W)
    base[2] *= np.float32(1e-6)
    base[3] *= np.float32(1e4)
    base[4, :5] = [0.7, 0.7, 0.7]                      # a run of equal pixels
    base[5, 3] = np.nan
    base[6, 7] = [-1.0, 0.5, 0.2]
    return base
