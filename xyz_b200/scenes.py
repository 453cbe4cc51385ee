"""Seeded synthetic scenes for the path tracer.

The reference renderer loads Metasequoia (.mqo) scenes that are not part of its
tree, so every workload here is generated from a seed.  Triangle ids are the
generator's order (the reference's loader would Morton-sort them,
xyz/core/scene_mqo.cpp:676-692).

Conventions shared with the reference (xyz/geom/triangle.cpp:10-33):
  * a triangle (v0, v1, v2) has geometric normal normalize(cross(v2-v0, v1-v0));
    its *front* side is the side that normal points to, and an emitter radiates
    only from its front side (xyz/core/scene_pathtracing.cpp:84);
  * lights share one power Phi (XYZ), spread as radiance Phi / (pi * A_lights)
    (xyz/core/scene_pathtracing.cpp:87-109).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field
from typing import Optional

import numpy as np

from .spectrum import N_BINS, ccir601_rgb_to_xyz, flat_spd_xyz, named_spectrum, rgb_to_spd, spd_to_xyz


@dataclass
class Camera:
    """Reference camera model (xyz/core/thinlenscamera.cpp:20-28, 71-90).

    `pinhole` selects the CONFIG_PINHOLE_CAMERA_MODEL ray generation
    (thinlenscamera.cpp:111-124); otherwise the thin lens of :188-205."""

    eye: tuple = (0.0, 1.0, 4.0)
    at: tuple = (0.0, 1.0, 0.0)
    film_size: float = 0.025
    focal_length: float = 0.035
    f_number: float = 1.4
    pinhole: bool = False

    @staticmethod
    def with_fov(eye, at, fov_y_deg: float, pinhole: bool = True,
                 focal_length: float = 0.035, f_number: float = 1.4) -> "Camera":
        """Film size that gives vertical field of view `fov_y_deg` with the
        reference's lens-film distance V = L f / (L - f)."""
        L = math.dist(eye, at)
        V = L * focal_length / (L - focal_length)
        film = 2.0 * V * math.tan(math.radians(fov_y_deg) / 2.0)
        return Camera(tuple(map(float, eye)), tuple(map(float, at)), float(film),
                      float(focal_length), float(f_number), pinhole)


@dataclass
class SceneData:
    positions: np.ndarray              # (nv, 3) float32
    tris: np.ndarray                   # (nt, 3) int32
    tri_mat: np.ndarray                # (nt,) int32
    albedo_xyz: np.ndarray             # (nm, 3) float32
    is_light: np.ndarray               # (nm,) int32
    light_power_xyz: np.ndarray        # (3,) float32, Phi shared by all lights
    normals: Optional[np.ndarray] = None  # (nv, 3) float32 shading normals
    camera: Camera = field(default_factory=Camera)
    name: str = ""
    albedo_spd: Optional[np.ndarray] = None       # (nm, 31) float32 spectra (spectral modes)
    light_power_spd: Optional[np.ndarray] = None  # (31,) float32, Phi per bin
    material_kind: Optional[np.ndarray] = None    # (nm,) int32: 0 Lambert, 2 mirror, 3 metal
    shininess: Optional[np.ndarray] = None        # (nm,) float32 metal lobe exponents

    @property
    def n_tris(self) -> int:
        return int(self.tris.shape[0])

    def light_area(self) -> float:
        """Total emitter area in float32, accumulated in triangle order."""
        lit = self.is_light[self.tri_mat] != 0
        acc = np.float32(0.0)
        for a in triangle_areas(self.positions, self.tris[lit]):
            acc = np.float32(acc + a)
        return float(acc)


def triangle_areas(pos: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """|cross(e2, e1)| * 0.5 in float32 (xyz/geom/triangle.hpp:57-59)."""
    p = pos.astype(np.float32)
    v0 = p[tris[:, 0]]
    e1 = (p[tris[:, 1]] - v0).astype(np.float32)
    e2 = (p[tris[:, 2]] - v0).astype(np.float32)
    c = np.cross(e2, e1).astype(np.float32)
    return (np.sqrt((c * c).sum(axis=1, dtype=np.float32)) * np.float32(0.5)).astype(np.float32)


def flat_emitter_power_spd(radiance: float, light_area: float) -> np.ndarray:
    """Phi per 10 nm bin of a flat emitter of `radiance` W/m^2/sr: pi * A * L."""
    return np.full(N_BINS, np.float32(math.pi * light_area) * np.float32(radiance), np.float32)


def flat_emitter_power(radiance: float, light_area: float) -> np.ndarray:
    """Phi (XYZ) for a spectrally flat emitter of `radiance` W/m^2/sr per bin:
    the reference spreads Phi as Phi / (pi * A), so Phi = pi * A * L_xyz."""
    return (flat_spd_xyz(radiance) * np.float32(math.pi * light_area)).astype(np.float32)


# --------------------------------------------------------------------------
# geometry helpers
# --------------------------------------------------------------------------

class _Builder:
    def __init__(self):
        self.pos: list = []
        self.tris: list = []
        self.mat: list = []

    def add_tri(self, a, b, c, m, front=None):
        """Adds (a, b, c); if `front` is given, orders the vertices so that the
        reference's geometric normal cross(v2-v0, v1-v0) points along it."""
        a, b, c = (np.asarray(v, dtype=np.float64) for v in (a, b, c))
        if front is not None:
            n = np.cross(c - a, b - a)
            if np.dot(n, np.asarray(front, dtype=np.float64)) < 0:
                b, c = c, b
        base = len(self.pos)
        self.pos.extend([a, b, c])
        self.tris.append((base, base + 1, base + 2))
        self.mat.append(m)

    def add_quad(self, p0, p1, p2, p3, m, front):
        self.add_tri(p0, p1, p2, m, front)
        self.add_tri(p0, p2, p3, m, front)

    def add_box(self, lo, hi, m):
        """Axis-aligned box, faces pointing outwards (12 triangles)."""
        x0, y0, z0 = lo
        x1, y1, z1 = hi
        c = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0),
             (x0, y0, z1), (x1, y0, z1), (x1, y1, z1), (x0, y1, z1)]
        faces = [((0, 1, 2, 3), (0, 0, -1)), ((4, 5, 6, 7), (0, 0, 1)),
                 ((0, 1, 5, 4), (0, -1, 0)), ((3, 2, 6, 7), (0, 1, 0)),
                 ((0, 3, 7, 4), (-1, 0, 0)), ((1, 2, 6, 5), (1, 0, 0))]
        for (i, j, k, l), n in faces:
            self.add_quad(c[i], c[j], c[k], c[l], m, n)

    def arrays(self):
        return (np.asarray(self.pos, dtype=np.float32).reshape(-1, 3),
                np.asarray(self.tris, dtype=np.int32).reshape(-1, 3),
                np.asarray(self.mat, dtype=np.int32))


def cornell_box(res_fov: float = 40.0, pinhole: bool = True,
                radiance: float = 15.0) -> SceneData:
    """Cornell-style closed room: 2x2x2 m (x in [-1,1], y in [0,2], z in [-1,1]),
    10 wall triangles (floor, ceiling, back, red left, green right; the front is
    open towards the camera), two axis-aligned boxes (24 triangles) and a
    0.5 x 0.5 m ceiling light 1 mm below the ceiling facing down (2 triangles).
    Albedos (linear RGB -> XYZ): white 0.8, red (0.63, 0.06, 0.05),
    green (0.14, 0.45, 0.09).  Spectrally flat emission of `radiance`
    W/m^2/sr.  Pinhole camera, vertical fov `res_fov` degrees."""
    WHITE, RED, GREEN, LIGHT = 0, 1, 2, 3
    b = _Builder()
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), WHITE, (0, 1, 0))     # floor
    b.add_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1), WHITE, (0, -1, 0))    # ceiling
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), WHITE, (0, 0, 1))   # back
    b.add_quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1), RED, (1, 0, 0))     # left
    b.add_quad((1, 0, -1), (1, 2, -1), (1, 2, 1), (1, 0, 1), GREEN, (-1, 0, 0))      # right
    b.add_box((-0.70, 0.0, -0.70), (-0.10, 1.2, -0.10), WHITE)                     # tall box
    b.add_box((0.10, 0.0, -0.20), (0.70, 0.6, 0.40), WHITE)                        # short box
    y = 2.0 - 0.001
    b.add_quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25),
               LIGHT, (0, -1, 0))
    pos, tris, mat = b.arrays()
    albedo = np.stack([ccir601_rgb_to_xyz((0.8, 0.8, 0.8)),
                       ccir601_rgb_to_xyz((0.63, 0.06, 0.05)),
                       ccir601_rgb_to_xyz((0.14, 0.45, 0.09)),
                       np.zeros(3, np.float32)]).astype(np.float32)
    is_light = np.array([0, 0, 0, 1], dtype=np.int32)
    sd = SceneData(pos, tris, mat, albedo, is_light, np.zeros(3, np.float32),
                   camera=Camera.with_fov((0.0, 1.0, 3.75), (0.0, 1.0, 0.0), res_fov,
                                          pinhole=pinhole),
                   name="cornell")
    sd.light_power_xyz = flat_emitter_power(radiance, sd.light_area())
    sd.albedo_spd = np.stack([rgb_to_spd((0.8, 0.8, 0.8)), rgb_to_spd((0.63, 0.06, 0.05)),
                              rgb_to_spd((0.14, 0.45, 0.09)), np.zeros(N_BINS, np.float32)])
    sd.light_power_spd = flat_emitter_power_spd(radiance, sd.light_area())
    return sd


def cornell_specular(shininess: float = 40.0, pinhole: bool = True, radiance: float = 15.0) -> SceneData:
    """The Cornell room with the tall box a perfect mirror (the reference's
    Mirror, xyz/bsdf/mirror.cpp) and the short box a glossy metal (its Metal,
    xyz/bsdf/metal.cpp: Phong lobe of exponent `shininess`, albedo of a
    gold-like RGB (1.0, 0.78, 0.34) in XYZ)."""
    sd = cornell_box(pinhole=pinhole, radiance=radiance)
    # materials 0..3 are white, red, green, light; 4 mirror, 5 metal
    tall = slice(10, 22)     # triangles of the tall box (after 10 wall triangles)
    short = slice(22, 34)
    tri_mat = sd.tri_mat.copy()
    tri_mat[tall] = 4
    tri_mat[short] = 5
    albedo = np.concatenate([sd.albedo_xyz, np.ones((1, 3), np.float32),
                             ccir601_rgb_to_xyz((1.0, 0.78, 0.34))[None]]).astype(np.float32)
    sd.tri_mat = tri_mat
    sd.albedo_xyz = albedo
    sd.is_light = np.array([0, 0, 0, 1, 0, 0], np.int32)
    sd.material_kind = np.array([0, 0, 0, 0, 2, 3], np.int32)
    sd.shininess = np.array([1, 1, 1, 1, 1, shininess], np.float32)
    sd.albedo_spd = None
    sd.name = "cornell-specular"
    return sd


def color_checker_room(illuminant: str = "light_d65", radiance: float = 15.0, pinhole: bool = True) -> SceneData:
    """The Cornell room with spectral materials from the reference's tables
    (libhi/hi/image/spectrum.cpp:170-476): walls of Macbeth ColorChecker
    patches (floor and ceiling neutral 8, back wall white, left red, right
    green, boxes blue sky and foliage), the 24 patches as a 6 x 4 chart of
    0.2 m squares 1 mm in front of the back wall, and the ceiling light
    emitting the named illuminant's spectrum scaled to a mean radiance of
    `radiance` W/m^2/sr per bin.  XYZ albedos are the spectra's XYZ (clamped to
    [0, 1]) for the XYZ film mode."""
    from .spectrum import COLOR_CHECKER
    WALL = ["mcc_neutral80", "mcc_white", "mcc_red", "mcc_green", "mcc_blue_sky", "mcc_foliage"]
    b = _Builder()
    N80, WHITE, RED, GREEN, SKY, FOL, LIGHT = range(7)
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 0, 1), (-1, 0, 1), N80, (0, 1, 0))
    b.add_quad((-1, 2, -1), (1, 2, -1), (1, 2, 1), (-1, 2, 1), N80, (0, -1, 0))
    b.add_quad((-1, 0, -1), (1, 0, -1), (1, 2, -1), (-1, 2, -1), WHITE, (0, 0, 1))
    b.add_quad((-1, 0, -1), (-1, 2, -1), (-1, 2, 1), (-1, 0, 1), RED, (1, 0, 0))
    b.add_quad((1, 0, -1), (1, 2, -1), (1, 2, 1), (1, 0, 1), GREEN, (-1, 0, 0))
    b.add_box((-0.70, 0.0, -0.70), (-0.10, 1.2, -0.10), SKY)
    b.add_box((0.10, 0.0, -0.20), (0.70, 0.6, 0.40), FOL)
    y = 2.0 - 0.001
    b.add_quad((-0.25, y, -0.25), (0.25, y, -0.25), (0.25, y, 0.25), (-0.25, y, 0.25), LIGHT, (0, -1, 0))
    z = -1.0 + 0.001
    for k, _ in enumerate(COLOR_CHECKER):
        r, c = divmod(k, 6)
        x0, y0 = -0.6 + 0.2 * c, 1.95 - 0.2 * (r + 1)
        b.add_quad((x0, y0, z), (x0 + 0.19, y0, z), (x0 + 0.19, y0 + 0.19, z), (x0, y0 + 0.19, z), 7 + k, (0, 0, 1))
    pos, tris, mat = b.arrays()
    names = WALL + [None] + list(COLOR_CHECKER)
    spd = np.stack([named_spectrum(n) if n else np.zeros(N_BINS, np.float32) for n in names]).astype(np.float32)
    albedo = np.stack([np.clip(spd_to_xyz(v), 0.0, 1.0) for v in spd]).astype(np.float32)
    is_light = np.zeros(len(names), np.int32)
    is_light[LIGHT] = 1
    sd = SceneData(pos, tris, mat, albedo, is_light, np.zeros(3, np.float32),
                   camera=Camera.with_fov((0.0, 1.0, 3.75), (0.0, 1.0, 0.0), 40.0, pinhole=pinhole),
                   name="color-checker-room")
    illum = named_spectrum(illuminant).astype(np.float64)
    L = (illum / illum.mean() * radiance).astype(np.float32)
    area = sd.light_area()
    sd.light_power_spd = (np.float32(math.pi * area) * L).astype(np.float32)
    sd.light_power_xyz = spd_to_xyz(sd.light_power_spd)
    sd.albedo_spd = spd
    return sd


# --------------------------------------------------------------------------
# icospheres and value noise
# --------------------------------------------------------------------------

def icosphere(level: int):
    """Unit icosphere subdivided `level` times: 20 * 4**level faces.  Face
    winding makes cross(v2-v0, v1-v0) point outwards (front side outside)."""
    t = (1.0 + 5.0 ** 0.5) / 2.0
    v = np.array([(-1, t, 0), (1, t, 0), (-1, -t, 0), (1, -t, 0),
                  (0, -1, t), (0, 1, t), (0, -1, -t), (0, 1, -t),
                  (t, 0, -1), (t, 0, 1), (-t, 0, -1), (-t, 0, 1)], dtype=np.float64)
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    f = np.array([(0, 11, 5), (0, 5, 1), (0, 1, 7), (0, 7, 10), (0, 10, 11),
                  (1, 5, 9), (5, 11, 4), (11, 10, 2), (10, 7, 6), (7, 1, 8),
                  (3, 9, 4), (3, 4, 2), (3, 2, 6), (3, 6, 8), (3, 8, 9),
                  (4, 9, 5), (2, 4, 11), (6, 2, 10), (8, 6, 7), (9, 8, 1)], dtype=np.int64)
    for _ in range(level):
        nv = v.shape[0]
        e = np.concatenate([f[:, [0, 1]], f[:, [1, 2]], f[:, [2, 0]]])
        e.sort(axis=1)
        key = e[:, 0] * (nv + 1) + e[:, 1]
        uniq, inv = np.unique(key, return_inverse=True)
        a, bb = uniq // (nv + 1), uniq % (nv + 1)
        mid = v[a] + v[bb]
        mid /= np.linalg.norm(mid, axis=1, keepdims=True)
        v = np.concatenate([v, mid])
        m = inv.reshape(3, -1).T + nv          # midpoints of edges 01, 12, 20
        f0, f1, f2 = f[:, 0], f[:, 1], f[:, 2]
        m01, m12, m20 = m[:, 0], m[:, 1], m[:, 2]
        f = np.concatenate([np.stack([f0, m01, m20], 1), np.stack([f1, m12, m01], 1),
                            np.stack([f2, m20, m12], 1), np.stack([m01, m12, m20], 1)])
    # The 20 seed faces are counter-clockwise seen from outside; the reference's
    # front normal is cross(v2-v0, v1-v0), so flip the winding.
    f = f[:, [0, 2, 1]]
    return v, f


def _hash3(ix, iy, iz, seed):
    h = (ix.astype(np.uint32) * np.uint32(0x8DA6B343)) ^ \
        (iy.astype(np.uint32) * np.uint32(0xD8163841)) ^ \
        (iz.astype(np.uint32) * np.uint32(0xCB1AB31F)) ^ np.uint32(seed * 0x9E3779B1 & 0xFFFFFFFF)
    h ^= h >> np.uint32(16)
    h *= np.uint32(0x7FEB352D)
    h ^= h >> np.uint32(15)
    h *= np.uint32(0x846CA68B)
    h ^= h >> np.uint32(16)
    return h.astype(np.float64) / 4294967295.0 * 2.0 - 1.0


def value_noise(p: np.ndarray, seed: int, octaves: int = 4, base_freq: float = 2.0) -> np.ndarray:
    """Seeded lattice value noise in [-1, 1]: per-octave trilinear
    interpolation of hashed lattice values with smoothstep weights; octave o
    has frequency base_freq * 2**o and weight 0.5**o (weights normalised)."""
    total = np.zeros(p.shape[0])
    norm = 0.0
    with np.errstate(over="ignore"):
        for o in range(octaves):
            q = p * (base_freq * 2 ** o)
            i0 = np.floor(q).astype(np.int64)
            fr = q - i0
            w = fr * fr * (3.0 - 2.0 * fr)
            acc = np.zeros(p.shape[0])
            for dx in (0, 1):
                for dy in (0, 1):
                    for dz in (0, 1):
                        h = _hash3(i0[:, 0] + dx, i0[:, 1] + dy, i0[:, 2] + dz, seed * 7 + o)
                        wx = w[:, 0] if dx else 1 - w[:, 0]
                        wy = w[:, 1] if dy else 1 - w[:, 1]
                        wz = w[:, 2] if dz else 1 - w[:, 2]
                        acc += h * wx * wy * wz
            total += acc * 0.5 ** o
            norm += 0.5 ** o
    return total / norm


def vertex_normals(pos: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """Area-weighted vertex normals along the reference's front normal
    cross(v2-v0, v1-v0), normalised."""
    p = pos.astype(np.float64)
    n = np.cross(p[tris[:, 2]] - p[tris[:, 0]], p[tris[:, 1]] - p[tris[:, 0]])
    acc = np.zeros_like(p)
    for k in range(3):
        np.add.at(acc, tris[:, k], n)
    acc /= np.maximum(np.linalg.norm(acc, axis=1, keepdims=True), 1e-30)
    return acc.astype(np.float32)


def displaced_icosphere(level: int, seed: int, amplitude: float = 0.15):
    """Unit icosphere radially displaced by 4-octave value noise:
    r = 1 + amplitude * noise(direction)."""
    v, f = icosphere(level)
    r = 1.0 + amplitude * value_noise(v, seed)
    return v * r[:, None], f


def spheres_scene(level: int = 7, n_spheres: int = 3, seed: int = 0,
                  radiance: float = 15.0, smooth: bool = True,
                  fov: float = 40.0, light_level: int = 3) -> SceneData:
    """Large-mesh workload: `n_spheres` displaced level-`level` icospheres
    (radius 0.6, noise amplitude 0.15) over a 40 x 40 m ground plane, lit by one
    tessellated spherical area light of radius 0.3.  Every triangle has its own
    grey Lambert albedo drawn uniformly from [0.2, 0.9] (seeded).  At level 7 and
    three spheres this is 983,040 + 2 + 1,280 = 984,322 triangles."""
    rng = np.random.default_rng(seed)
    pos_l, tri_l, norm_l = [], [], []
    base = 0
    xs = np.linspace(-1.4, 1.4, n_spheres) if n_spheres > 1 else np.zeros(1)
    for s, x in enumerate(xs):
        v, f = displaced_icosphere(level, seed * 101 + s, 0.15)
        v = v * 0.6 + np.array([x, 0.72, 0.0])
        pos_l.append(v)
        tri_l.append(f + base)
        norm_l.append(vertex_normals(v, f) if smooth else None)
        base += v.shape[0]
    # ground (front side up)
    g = np.array([(-20, 0, -20), (20, 0, -20), (20, 0, 20), (-20, 0, 20)], dtype=np.float64)
    gt = np.array([(0, 1, 2), (0, 2, 3)], dtype=np.int64)   # front normal +y
    pos_l.append(g)
    tri_l.append(gt + base)
    norm_l.append(np.tile(np.array([[0, 1, 0]], np.float32), (4, 1)))
    base += 4
    # spherical light, front side outwards
    lv, lf = icosphere(light_level)
    lv = lv * 0.3 + np.array([0.0, 2.6, 1.2])
    pos_l.append(lv)
    tri_l.append(lf + base)
    norm_l.append(vertex_normals(lv, lf))
    pos = np.concatenate(pos_l).astype(np.float32)
    tris = np.concatenate(tri_l).astype(np.int32)
    n_geom = tris.shape[0] - lf.shape[0]
    grey = rng.uniform(0.2, 0.9, size=n_geom)
    white = ccir601_rgb_to_xyz((1.0, 1.0, 1.0))
    albedo = np.concatenate([(grey[:, None] * white[None, :]).astype(np.float32),
                             np.zeros((1, 3), np.float32)])
    is_light = np.zeros(n_geom + 1, dtype=np.int32)
    is_light[-1] = 1
    tri_mat = np.concatenate([np.arange(n_geom, dtype=np.int32),
                              np.full(lf.shape[0], n_geom, dtype=np.int32)])
    normals = np.concatenate(norm_l).astype(np.float32) if smooth else None
    sd = SceneData(pos, tris, tri_mat, albedo, is_light, np.zeros(3, np.float32),
                   normals=normals,
                   camera=Camera.with_fov((0.0, 1.6, 4.8), (0.0, 0.6, 0.0), fov, pinhole=True),
                   name=f"spheres-l{level}x{n_spheres}")
    sd.light_power_xyz = flat_emitter_power(radiance, sd.light_area())
    # grey materials have flat spectra
    sd.albedo_spd = np.concatenate([np.repeat(grey[:, None], N_BINS, axis=1).astype(np.float32),
                                    np.zeros((1, N_BINS), np.float32)])
    sd.light_power_spd = flat_emitter_power_spd(radiance, sd.light_area())
    return sd



def _grid_quad(b: "_Builder", origin, u, v, n: int, m_first: int, front) -> int:
    """n x n grid of quads spanning origin + [0,1] u + [0,1] v, one material per
    triangle starting at m_first; returns the next free material id."""
    o, u, v = (np.asarray(x, dtype=np.float64) for x in (origin, u, v))
    m = m_first
    for i in range(n):
        for j in range(n):
            p00 = o + u * (i / n) + v * (j / n)
            p10 = o + u * ((i + 1) / n) + v * (j / n)
            p11 = o + u * ((i + 1) / n) + v * ((j + 1) / n)
            p01 = o + u * (i / n) + v * ((j + 1) / n)
            b.add_tri(p00, p10, p11, m, front)
            b.add_tri(p00, p11, p01, m + 1, front)
            m += 2
    return m


@dataclass
class DiffScene:
    """A differentiable-rendering workload: the scene (one material per
    triangle), the initial parameters and the target's parameters."""
    scene: SceneData
    albedo: np.ndarray          # (n_materials, 3) float32, initial
    emission: np.ndarray        # (n_materials,) float32, initial (0 for non-lights)
    target_albedo: np.ndarray
    target_emission: np.ndarray
    light_materials: np.ndarray  # ids of the emitting materials


def diff_scene(level: int = 4, wall_n: int = 20, light_n: int = 4, seed: int = 0,
               target_seed: int = 1, perturb: float = 0.2) -> DiffScene:
    """Room + 3 displaced spheres with per-triangle parameters.

    The room is the Cornell box's 2 x 2 x 2 m shell (floor, ceiling, back, left,
    right; open front) with each wall an wall_n x wall_n grid of quads; a
    0.5 x 0.5 m ceiling light (light_n x light_n quads) 1 mm below the
    ceiling; three displaced level-`level` icospheres of radius 0.3 on the
    floor.  Every triangle is its own material.  Albedo: 3 channels (the film's
    XYZ channels) uniform in [0.1, 0.9]; light triangles: emission scale uniform
    in [5, 20] on a base radiance of 1 per channel (Phi = pi * A_light).  The
    target's parameters add uniform noise of +-`perturb` (emission: a relative
    +-`perturb`) drawn from `target_seed`.  At level 4, wall_n 20 and light_n 4
    this is 15,360 + 4,000 + 32 = 19,392 triangles."""
    b = _Builder()
    m = 0
    m = _grid_quad(b, (-1, 0, -1), (2, 0, 0), (0, 0, 2), wall_n, m, (0, 1, 0))    # floor
    m = _grid_quad(b, (-1, 2, -1), (2, 0, 0), (0, 0, 2), wall_n, m, (0, -1, 0))   # ceiling
    m = _grid_quad(b, (-1, 0, -1), (2, 0, 0), (0, 2, 0), wall_n, m, (0, 0, 1))    # back
    m = _grid_quad(b, (-1, 0, -1), (0, 2, 0), (0, 0, 2), wall_n, m, (1, 0, 0))    # left
    m = _grid_quad(b, (1, 0, -1), (0, 2, 0), (0, 0, 2), wall_n, m, (-1, 0, 0))    # right
    n_walls = m
    y = 2.0 - 0.001
    m = _grid_quad(b, (-0.25, y, -0.25), (0.5, 0, 0), (0, 0, 0.5), light_n, m, (0, -1, 0))
    n_light = m - n_walls
    pos_r, tris_r, mat_r = b.arrays()
    nrm_r = np.zeros_like(pos_r)
    for t in range(tris_r.shape[0]):
        a, bb, c = pos_r[tris_r[t]].astype(np.float64)
        n = np.cross(c - a, bb - a)
        nrm_r[tris_r[t]] = (n / np.linalg.norm(n)).astype(np.float32)
    pos_l, tri_l, nrm_l, mat_l = [pos_r], [tris_r], [nrm_r], [mat_r]
    base = pos_r.shape[0]
    for k, (cx, cz) in enumerate([(-0.45, -0.35), (0.15, 0.35), (0.55, -0.45)]):
        v, f = displaced_icosphere(level, seed * 31 + k, 0.15)
        v = v * 0.3 + np.array([cx, 0.36, cz])
        pos_l.append(v)
        tri_l.append(f + base)
        nrm_l.append(vertex_normals(v, f))
        mat_l.append(np.arange(m, m + f.shape[0], dtype=np.int32))
        m += f.shape[0]
        base += v.shape[0]
    pos = np.concatenate(pos_l).astype(np.float32)
    tris = np.concatenate(tri_l).astype(np.int32)
    tri_mat = np.concatenate(mat_l).astype(np.int32)
    normals = np.concatenate(nrm_l).astype(np.float32)
    nm = m
    is_light = np.zeros(nm, np.int32)
    light_mats = np.arange(n_walls, n_walls + n_light, dtype=np.int32)
    is_light[light_mats] = 1
    rng = np.random.default_rng(seed)
    albedo = rng.uniform(0.1, 0.9, size=(nm, 3)).astype(np.float32)
    albedo[light_mats] = 0.0
    emission = np.zeros(nm, np.float32)
    emission[light_mats] = rng.uniform(5.0, 20.0, size=n_light).astype(np.float32)
    sd = SceneData(pos, tris, tri_mat, albedo, is_light, np.zeros(3, np.float32), normals=normals,
                   camera=Camera.with_fov((0.0, 1.0, 3.75), (0.0, 1.0, 0.0), 40.0, pinhole=True),
                   name=f"diff-room-l{level}")
    sd.light_power_xyz = np.full(3, np.float32(math.pi * sd.light_area()), np.float32)
    rt = np.random.default_rng(target_seed)
    t_alb = np.clip(albedo + rt.uniform(-perturb, perturb, size=albedo.shape), 0.0, 1.0).astype(np.float32)
    t_alb[light_mats] = 0.0
    t_em = (emission * (1.0 + rt.uniform(-perturb, perturb, size=nm))).astype(np.float32)
    return DiffScene(sd, albedo, emission, t_alb, t_em, light_mats)


_ICO_CACHE: dict = {}


def _icosphere_cached(level: int):
    if level not in _ICO_CACHE:
        _ICO_CACHE[level] = icosphere(level)
    return _ICO_CACHE[level]


def _box_tris(lo: np.ndarray, hi: np.ndarray):
    """Axis-aligned boxes (n, 3) lo / hi -> (n * 8, 3) vertices, (n * 12, 3)
    triangles with outward front normals (cross(v2-v0, v1-v0))."""
    n = lo.shape[0]
    corners = np.array([(0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0),
                        (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1)], dtype=np.float64)
    v = lo[:, None, :] + corners[None, :, :] * (hi - lo)[:, None, :]
    # quads (i, j, k, l) with outward normals; split (i, j, k), (i, k, l)
    quads = [((0, 3, 2, 1)), ((4, 5, 6, 7)), ((0, 1, 5, 4)), ((3, 7, 6, 2)),
             ((0, 4, 7, 3)), ((1, 2, 6, 5))]
    t = []
    for (i, j, k, l) in quads:
        t.append((i, k, j))
        t.append((i, l, k))
    t = np.array(t, dtype=np.int64)
    tris = (t[None, :, :] + 8 * np.arange(n)[:, None, None]).reshape(-1, 3)
    return v.reshape(-1, 3), tris


def batch_scene(seed: int, target_tris: Optional[int] = None, radiance: float = 15.0) -> SceneData:
    """One scene of the batched workload.  Triangle count log-uniform in
    [1,000, 500,000] (from the seed) unless given.  Odd seeds: displaced
    icospheres (the level whose face count fits, as many spheres as make up
    the count); even seeds: random stacks of boxes (12 triangles each).  All on
    a 20 x 20 m ground under a spherical light of radius 0.25 (320 triangles);
    8 grey / coloured Lambert materials; pinhole camera, 40 degree fov."""
    rng = np.random.default_rng(1000 + seed)
    if target_tris is None:
        target_tris = int(round(math.exp(rng.uniform(math.log(1000), math.log(500000)))))
    pos_l, tri_l = [], []
    base = 0
    if seed % 2 == 1:
        level = 3
        while level < 7 and 20 * 4 ** (level + 1) <= target_tris:
            level += 1
        n_sph = max(1, int(round(target_tris / (20 * 4 ** level))))
        xs = np.linspace(-1.2, 1.2, n_sph) if n_sph > 1 else np.zeros(1)
        r = 0.6 if n_sph <= 2 else 1.6 / n_sph
        for k, x in enumerate(xs):
            v, f = _icosphere_cached(level)
            v = v * (1.0 + 0.15 * value_noise(v, seed * 13 + k))[:, None]
            v = v * r + np.array([x, r * 1.2, 0.0])
            pos_l.append(v)
            tri_l.append(f + base)
            base += v.shape[0]
    else:
        n_box = max(1, int(round(target_tris / 12)))
        cols = max(1, int(math.ceil(math.sqrt(n_box / 4.0))))
        per_col = int(math.ceil(n_box / (cols * cols)))
        idx = np.arange(n_box)
        c = idx // per_col
        lvl = idx % per_col
        cx, cz = c % cols, c // cols
        cell = 2.4 / cols
        h = 1.6 / per_col
        jitter = rng.uniform(-0.1, 0.1, size=(n_box, 2)) * cell
        size = rng.uniform(0.4, 0.9, size=(n_box, 2)) * cell
        x0 = -1.2 + (cx + 0.5) * cell + jitter[:, 0] - size[:, 0] / 2
        z0 = -1.2 + (cz + 0.5) * cell + jitter[:, 1] - size[:, 1] / 2
        y0 = lvl * h
        lo = np.stack([x0, y0, z0], 1)
        hi = np.stack([x0 + size[:, 0], y0 + h * rng.uniform(0.6, 1.0, size=n_box), z0 + size[:, 1]], 1)
        v, f = _box_tris(lo, hi)
        pos_l.append(v)
        tri_l.append(f + base)
        base += v.shape[0]
    n_geom = int(sum(t.shape[0] for t in tri_l))
    g = np.array([(-10, 0, -10), (10, 0, -10), (10, 0, 10), (-10, 0, 10)], dtype=np.float64)
    pos_l.append(g)
    tri_l.append(np.array([(0, 1, 2), (0, 2, 3)], dtype=np.int64) + base)
    base += 4
    lv, lf = _icosphere_cached(2)
    lv = lv * 0.25 + np.array([0.4, 2.8, 1.4])
    pos_l.append(lv)
    tri_l.append(lf + base)
    pos = np.concatenate(pos_l).astype(np.float32)
    tris = np.concatenate(tri_l).astype(np.int32)
    n_mat = 8
    tri_mat = np.concatenate([rng.integers(0, n_mat, size=n_geom), np.zeros(2, np.int64),
                              np.full(lf.shape[0], n_mat)]).astype(np.int32)
    rgb = rng.uniform(0.15, 0.85, size=(n_mat, 3))
    albedo = np.concatenate([np.stack([ccir601_rgb_to_xyz(c) for c in rgb]),
                             np.zeros((1, 3), np.float32)]).astype(np.float32)
    is_light = np.zeros(n_mat + 1, np.int32)
    is_light[n_mat] = 1
    sd = SceneData(pos, tris, tri_mat, albedo, is_light, np.zeros(3, np.float32),
                   camera=Camera.with_fov((0.0, 1.5, 4.2), (0.0, 0.7, 0.0), 40.0, pinhole=True),
                   name=f"batch-{seed}")
    sd.light_power_xyz = flat_emitter_power(radiance, sd.light_area())
    return sd


@dataclass
class BatchEntry:
    scene: SceneData
    width: int
    height: int
    spp: int
    max_depth: int = 8


def batch_workload(n: int = 64, first_seed: int = 0) -> list:
    """The batched workload: scenes of seeds first_seed .. first_seed + n - 1
    (batch_scene), resolution drawn from {128, 256, 512, 1024} squared and
    samples per pixel uniform in 4..64 (seeded per scene), max depth 8."""
    out = []
    for k in range(n):
        seed = first_seed + k
        rng = np.random.default_rng(2000 + seed)
        res = int(rng.choice([128, 256, 512, 1024]))
        spp = int(rng.integers(4, 65))
        out.append(BatchEntry(batch_scene(seed), res, res, spp, 8))
    return out


def occluded_room(level: int = 6, wall_n: int = 48, seed: int = 0, radiance: float = 40.0,
                  room_albedo: float = 0.75, compartment_albedo: float = 0.75) -> SceneData:
    """Indirect-lit room for path guiding: a closed 4 x 4 x 3 m room (x, z in
    [-2, 2], y in [0, 3]); a dividing wall at z = 1.5 that stops 0.1 m below
    the ceiling; behind it a 3 x 0.3 m area light on the floor facing up.  The
    main room sees no emitter: light reaches it through the 0.1 m gap after
    bouncing off the compartment's ceiling and walls.  Furniture: two displaced
    level-`level` icospheres and four boxes.  Walls are wall_n x wall_n grids;
    at level 6 and wall_n 48: 2 x 81,920 sphere + 7 x 4,608 wall + 48 box +
    2 light = 196,146 triangles.  Lambert albedos: walls `room_albedo` (the
    wall behind the light `compartment_albedo`), a red and a blue sphere,
    grey boxes.  Pinhole camera in the main room facing the dividing wall,
    60 degree fov."""
    rng = np.random.default_rng(seed)
    WHITE, RED, BLUE, GREY, LIGHT, BRIGHT = 0, 1, 2, 3, 4, 5
    b = _Builder()

    def grid(origin, u, v, front, mat):
        o, u, v = (np.asarray(x, dtype=np.float64) for x in (origin, u, v))
        n = wall_n
        for i in range(n):
            for j in range(n):
                p00 = o + u * (i / n) + v * (j / n)
                p10 = o + u * ((i + 1) / n) + v * (j / n)
                p11 = o + u * ((i + 1) / n) + v * ((j + 1) / n)
                p01 = o + u * (i / n) + v * ((j + 1) / n)
                b.add_tri(p00, p10, p11, mat, front)
                b.add_tri(p00, p11, p01, mat, front)

    grid((-2, 0, -2), (4, 0, 0), (0, 0, 4), (0, 1, 0), WHITE)      # floor
    grid((-2, 3, -2), (4, 0, 0), (0, 0, 4), (0, -1, 0), WHITE)     # ceiling
    grid((-2, 0, -2), (4, 0, 0), (0, 3, 0), (0, 0, 1), WHITE)      # back wall
    grid((-2, 0, 2), (4, 0, 0), (0, 3, 0), (0, 0, -1), BRIGHT)     # wall behind the light
    grid((-2, 0, -2), (0, 3, 0), (0, 0, 4), (1, 0, 0), WHITE)      # left
    grid((2, 0, -2), (0, 3, 0), (0, 0, 4), (-1, 0, 0), WHITE)      # right
    grid((-2, 0, 1.5), (4, 0, 0), (0, 2.9, 0), (0, 0, -1), WHITE)  # dividing wall, gap above
    # boxes in the main room
    for k in range(4):
        x0, z0 = rng.uniform(-1.6, 1.0), rng.uniform(-1.6, 0.8)
        sx, sz, sy = rng.uniform(0.2, 0.5), rng.uniform(0.2, 0.5), rng.uniform(0.2, 0.8)
        b.add_box((x0, 0.0, z0), (x0 + sx, sy, z0 + sz), GREY)
    # the light: on the compartment floor, facing up
    b.add_quad((-1.5, 0.01, 1.6), (1.5, 0.01, 1.6), (1.5, 0.01, 1.9), (-1.5, 0.01, 1.9), LIGHT, (0, 1, 0))
    pos_r, tris_r, mat_r = b.arrays()
    nrm_r = np.zeros_like(pos_r)
    a = pos_r[tris_r[:, 0]].astype(np.float64)
    n = np.cross(pos_r[tris_r[:, 2]] - a, pos_r[tris_r[:, 1]] - a)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    for c in range(3):
        nrm_r[tris_r[:, c]] = n.astype(np.float32)
    pos_l, tri_l, nrm_l, mat_l = [pos_r], [tris_r], [nrm_r], [mat_r]
    base = pos_r.shape[0]
    for k, (cx, cz, mat) in enumerate([(-0.7, 0.3, RED), (0.8, -0.4, BLUE)]):
        v, f = displaced_icosphere(level, seed * 17 + k, 0.15)
        v = v * 0.45 + np.array([cx, 0.52, cz])
        pos_l.append(v)
        tri_l.append(f + base)
        nrm_l.append(vertex_normals(v, f))
        mat_l.append(np.full(f.shape[0], mat, np.int32))
        base += v.shape[0]
    pos = np.concatenate(pos_l).astype(np.float32)
    tris = np.concatenate(tri_l).astype(np.int32)
    tri_mat = np.concatenate(mat_l).astype(np.int32)
    normals = np.concatenate(nrm_l).astype(np.float32)
    ra, ca = room_albedo, compartment_albedo
    albedo = np.stack([ccir601_rgb_to_xyz((ra, ra, ra)), ccir601_rgb_to_xyz((0.7, 0.15, 0.1)),
                       ccir601_rgb_to_xyz((0.1, 0.2, 0.7)), ccir601_rgb_to_xyz((0.5, 0.5, 0.5)),
                       np.zeros(3, np.float32), ccir601_rgb_to_xyz((ca, ca, ca))]).astype(np.float32)
    is_light = np.array([0, 0, 0, 0, 1, 0], np.int32)
    sd = SceneData(pos, tris, tri_mat, albedo, is_light, np.zeros(3, np.float32), normals=normals,
                   camera=Camera.with_fov((0.0, 1.5, -1.9), (0.0, 1.3, 1.5), 60.0, pinhole=True),
                   name=f"occluded-room-l{level}")
    sd.light_power_xyz = flat_emitter_power(radiance, sd.light_area())
    return sd

def random_rays(scene: SceneData, n: int, seed: int = 0):
    """Seeded test rays: origins uniform in the scene box grown by 20 %,
    directions uniform on the sphere.  Returns (org, dir) float32 (n, 3)."""
    rng = np.random.default_rng(seed)
    lo = scene.positions.min(axis=0)
    hi = scene.positions.max(axis=0)
    c, h = (lo + hi) / 2, (hi - lo) / 2 * 1.2
    org = (c + h * rng.uniform(-1, 1, size=(n, 3))).astype(np.float32)
    d = rng.normal(size=(n, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return org, d.astype(np.float32)
