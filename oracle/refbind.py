"""ctypes bindings to the oracle libraries.  TEST INFRASTRUCTURE: imported only
by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg.

* `RefLib`  - the reference renderer's own path tracer compiled from its
  sources (oracle/_ref/libxyzref_{thinlens,pinhole}.so, see oracle/Makefile).
* `PortLib` - the plain-C restatement of the same algorithm
  (oracle/_port/libxyzport.so built from oracle/xyz_oracle.c).

Both take the same scene arrays as the CUDA library and read the same Philox
stream per (pixel, sample), so results can be compared path by path.
"""

from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
PORT_DIR = os.path.join(HERE, "_port")

_f32p = np.ctypeslib.ndpointer(dtype=np.float32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def ref_available(pinhole: bool = True) -> bool:
    return os.path.exists(_ref_path(pinhole))


def _ref_path(pinhole: bool) -> str:
    return os.path.join(REF_DIR, "libxyzref_pinhole.so" if pinhole else "libxyzref_thinlens.so")


FAST_REF_PATH = os.path.join(REF_DIR, "libxyzref_pinhole_o3.so")


def host_has_x86_64_v3() -> bool:
    """True when this host's CPU runs x86-64-v3 code (AVX2, FMA, BMI2), which
    the -O3 timing build of the reference (libxyzref_pinhole_o3.so) needs."""
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    fl = set(line.split(":", 1)[1].split())
                    return {"avx2", "fma", "bmi2", "movbe"} <= fl
    except OSError:
        pass
    return False


def fast_ref_available() -> bool:
    return os.path.exists(FAST_REF_PATH) and host_has_x86_64_v3()


def port_available() -> bool:
    return os.path.exists(os.path.join(PORT_DIR, "libxyzport.so"))


class _Common:
    """Shared scene/camera/render plumbing of the two oracle libraries."""

    prefix = ""

    def _sym(self, name):
        return getattr(self.lib, self.prefix + name)

    def set_path_params(self, max_depth: int, rr_threshold: float = 0.2, rr_start: int = 1):
        """max_depth = maximum number of path segments (the reference's kMax - 1)."""
        self._set_path(max_depth + 1, rr_threshold, rr_start)

    def light_power_xyz(self):
        out = np.zeros(3, np.float32)
        self._sym("light_power_xyz")(out.ctypes.data_as(C.POINTER(C.c_float)))
        return out

    def set_camera(self, cam, width: int, height: int):
        eye = _f(cam.eye)
        at = _f(cam.at)
        self._sym("set_camera")(eye.ctypes.data_as(C.c_void_p), at.ctypes.data_as(C.c_void_p),
                                C.c_float(cam.film_size), C.c_float(cam.focal_length),
                                C.c_float(cam.f_number), width, height)
        self.width, self.height = width, height

    def trace(self, org, dirs, nthreads: int = 0):
        org, dirs = _f(org), _f(dirs)
        n = org.shape[0]
        tri = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        f = np.empty(n, np.float32)
        g = np.empty(n, np.float32)
        back = np.empty(n, np.int32)
        self._sym("trace")(n, org.ctypes.data_as(C.c_void_p), dirs.ctypes.data_as(C.c_void_p),
                           tri.ctypes.data_as(C.c_void_p), t.ctypes.data_as(C.c_void_p),
                           f.ctypes.data_as(C.c_void_p), g.ctypes.data_as(C.c_void_p),
                           back.ctypes.data_as(C.c_void_p), nthreads)
        return tri, t, f, g, back

    def eval_path(self, px: int, py: int, s: int, seed: int):
        out = np.zeros(3, np.float32)
        dims = self._sym("eval_path")(px, py, s, C.c_uint64(seed), out.ctypes.data_as(C.c_void_p))
        return out, dims

    def render(self, spp: int, seed: int, s0: int = 0, y0: int = 0, y1=None,
               film=None, nthreads: int = 0):
        """Sum (not mean) of `spp` samples per pixel, film (H, W, 3) float32."""
        if y1 is None:
            y1 = self.height
        if film is None:
            film = np.zeros((self.height, self.width, 3), np.float32)
        self._sym("render")(s0, spp, C.c_uint64(seed), y0, y1,
                            film.ctypes.data_as(C.c_void_p), nthreads)
        return film


class RefLib(_Common):
    prefix = "xyzref_"

    def __init__(self, pinhole: bool = True, fast: bool = False):
        """fast: the -O3 x86-64-v3 timing build (pinhole only; same IEEE
        arithmetic as the parity build)."""
        if fast and not pinhole:
            raise ValueError("the timing build of the reference is the pinhole one")
        path = FAST_REF_PATH if fast else _ref_path(pinhole)
        if not os.path.exists(path):
            raise FileNotFoundError(f"reference oracle not built: {path} (run make -C oracle)")
        self.lib = C.CDLL(path)
        L = self.lib
        L.xyzref_scene_create.restype = C.c_int
        L.xyzref_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int]
        L.xyzref_set_camera.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                        C.c_int, C.c_int]
        L.xyzref_set_path_params.argtypes = [C.c_int, C.c_float]
        L.xyzref_trace.argtypes = [C.c_int] + [C.c_void_p] * 7 + [C.c_int]
        L.xyzref_eval_path.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_void_p]
        L.xyzref_eval_path.restype = C.c_int
        L.xyzref_render.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.xyzref_light_area.restype = C.c_float
        L.xyzref_max_threads.restype = C.c_int
        self.pinhole = bool(L.xyzref_is_pinhole())
        self.kind = "reference"
        self.build = "-O3 -march=x86-64-v3" if fast else "-O2"

    def _set_path(self, kmax, rr_threshold, rr_start):
        if rr_start != 1:
            raise ValueError("the reference applies Russian roulette from the first vertex")
        self.lib.xyzref_set_path_params(kmax, rr_threshold)

    def scene_create(self, sd, kd_max_bucket: int = 16, kd_max_depth: int = 16):
        """Loads a SceneData.  The reference scales every light by one global
        Mercury-arc power (xyz/core/config.hpp:81-95); `light_scale` maps its
        per-channel output to the scene's own Phi (the estimator is linear in
        Phi per channel)."""
        pos, tris, mat = _f(sd.positions), _i(sd.tris), _i(sd.tri_mat)
        alb, lit = _f(sd.albedo_xyz), _i(sd.is_light)
        nrm = _f(sd.normals) if sd.normals is not None else None
        if getattr(sd, "material_kind", None) is not None:
            # Mirror (2) / Metal (3) materials of the next scene
            kind = _i(sd.material_kind)
            shin = _f(sd.shininess if sd.shininess is not None else np.ones(kind.shape[0]))
            self.lib.xyzref_material_kinds.argtypes = [C.c_int, C.c_void_p, C.c_void_p]
            self.lib.xyzref_material_kinds(kind.shape[0], kind.ctypes.data_as(C.c_void_p),
                                           shin.ctypes.data_as(C.c_void_p))
            self._kinds = (kind, shin)
        r = self.lib.xyzref_scene_create(pos.shape[0], pos.ctypes.data_as(C.c_void_p),
                                         None if nrm is None else nrm.ctypes.data_as(C.c_void_p),
                                         tris.shape[0], tris.ctypes.data_as(C.c_void_p),
                                         mat.ctypes.data_as(C.c_void_p), alb.shape[0],
                                         alb.ctypes.data_as(C.c_void_p), lit.ctypes.data_as(C.c_void_p),
                                         kd_max_bucket, kd_max_depth)
        if r < 0:
            raise ValueError("reference rejected the scene")
        self.light_scale = (np.asarray(sd.light_power_xyz, np.float64) /
                            self.light_power_xyz().astype(np.float64))
        self._keep = (pos, tris, mat, alb, lit, nrm)
        return r

    def max_threads(self):
        return self.lib.xyzref_max_threads()

    def load_mqo(self, path: str):
        """The reference's Scene::Load on an .mqo file (run by the program
        oracle/_ref/xyzref_mqo in a process of its own): per triangle (in its
        order) the stored geometry (n, 21: v0, e1, e2, ng, n0, s1, s2) and
        material; per material (kind = Bsdf::What, albedo XYZ, shininess);
        the camera (eye, at)."""
        import subprocess
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            pre = os.path.join(d, "ref")
            subprocess.run([os.path.join(REF_DIR, "xyzref_mqo"), path, pre], check=True,
                           stdout=subprocess.DEVNULL, stderr=subprocess.DEVNULL)
            cam = np.fromfile(pre + ".cam", np.float32)
            return {"geo": np.fromfile(pre + ".geo", np.float32).reshape(-1, 21),
                    "mat": np.fromfile(pre + ".mat", np.int32),
                    "kind": np.fromfile(pre + ".kind", np.int32),
                    "albedo": np.fromfile(pre + ".alb", np.float32).reshape(-1, 3),
                    "shininess": np.fromfile(pre + ".shin", np.float32),
                    "eye": cam[:3], "at": cam[3:]}

    def named_spectra(self):
        """The reference library's named spectra {CamelCaseName: 31 float32}
        (libhi/hi/image/spectrum.cpp:170-476)."""
        self.lib.xyzref_spectrum_names.restype = C.c_char_p
        self.lib.xyzref_named_spectrum.argtypes = [C.c_int, C.c_void_p]
        names = self.lib.xyzref_spectrum_names().decode().split()
        out = {}
        for i, n in enumerate(names):
            v = np.zeros(31, np.float32)
            if self.lib.xyzref_named_spectrum(i, v.ctypes.data_as(C.c_void_p)) != 0:
                raise ValueError(n)
            out[n] = v
        return out


class PortLib(_Common):
    prefix = "xyzo_"

    def __init__(self):
        path = os.path.join(PORT_DIR, "libxyzport.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle port not built: {path} (run make -C oracle port)")
        self.lib = C.CDLL(path)
        L = self.lib
        L.xyzo_scene_create.restype = C.c_int
        L.xyzo_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                        C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                        C.c_int, C.c_int]
        L.xyzo_set_camera_full.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                           C.c_int, C.c_int, C.c_int]
        L.xyzo_set_path_params.argtypes = [C.c_int, C.c_float, C.c_int]
        L.xyzo_trace.argtypes = [C.c_int] + [C.c_void_p] * 7 + [C.c_int]
        L.xyzo_eval_path.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_void_p]
        L.xyzo_eval_path.restype = C.c_int
        L.xyzo_render.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_void_p, C.c_int]
        L.xyzo_render_pixels.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_uint64,
                                         C.c_void_p, C.c_int]
        L.xyzo_light_area.restype = C.c_float
        L.xyzo_max_threads.restype = C.c_int
        L.xyzo_philox_u01.restype = C.c_float
        L.xyzo_philox_u01.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
        L.xyzo_kdtree_stats.argtypes = [C.c_void_p]
        L.xyzo_scene_set_spectra.argtypes = [C.c_void_p, C.c_void_p]
        L.xyzo_set_spectral.argtypes = [C.c_int, C.c_int]
        L.xyzo_set_materials.argtypes = [C.c_void_p, C.c_void_p]
        L.xyzo_importons_emit.argtypes = [C.c_int, C.c_int, C.c_int, C.c_uint64, C.c_void_p, C.c_int]
        L.xyzo_importons_emit.restype = C.c_int
        L.xyzo_importons_set.argtypes = [C.c_void_p, C.c_int, C.c_float, C.c_int, C.c_int]
        L.xyzo_importons_query.argtypes = [C.c_void_p, C.c_int, C.c_void_p]
        L.xyzo_encode_rgbe.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_void_p]
        L.xyzo_tonemap.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_float, C.c_float,
                                   C.c_float, C.c_float, C.c_int, C.c_void_p]
        L.xyzo_adjoint.argtypes = [C.c_int, C.c_int, C.c_uint64, C.c_void_p, C.c_void_p, C.c_void_p,
                                   C.c_int]
        self.kind = "port"
        self.light_scale = np.ones(3)


    def render_pixels(self, px, py, spp: int, seed: int, s0: int = 0, acc=None, nthreads: int = 0):
        """Per-pixel double sums over samples [s0, s0 + spp) of the listed
        pixels: (n, 4) float64 rows (sum X, sum Y, sum Z, sum Y^2), added to
        `acc` when given."""
        px = np.ascontiguousarray(px, np.int32)
        py = np.ascontiguousarray(py, np.int32)
        if acc is None:
            acc = np.zeros((px.shape[0], 4), np.float64)
        self.lib.xyzo_render_pixels(px.shape[0], px.ctypes.data, py.ctypes.data, s0, spp, C.c_uint64(seed),
                                    acc.ctypes.data, nthreads)
        return acc
    def _set_path(self, kmax, rr_threshold, rr_start):
        self.lib.xyzo_set_path_params(kmax, rr_threshold, rr_start)

    def importons_emit(self, particles: int, max_depth: int = 16, min_depth: int = 1, seed: int = 0):
        """Light-importance map of the importance-driven tracer: (n, 6)
        float32 importons (position, incoming direction) in particle order."""
        n = self.lib.xyzo_importons_emit(particles, max_depth, min_depth, C.c_uint64(seed), None, 0)
        out = np.zeros((max(n, 1), 6), np.float32)
        self.lib.xyzo_importons_emit(particles, max_depth, min_depth, C.c_uint64(seed),
                                     out.ctypes.data_as(C.c_void_p), n)
        return out[:n]

    def importons_set(self, importons, radius: float = 0.1, enable: bool = True, guide_bounces: int = 1 << 30):
        """Loads a map; with enable the estimator samples Lambert vertices of
        the first guide_bounces from its histograms."""
        imp = _f(importons).reshape(-1, 6)
        self._imp = imp
        self.lib.xyzo_importons_set(imp.ctypes.data_as(C.c_void_p), imp.shape[0], C.c_float(radius), int(enable),
                                    int(guide_bounces))

    def importons_query(self, frames):
        """Cumulative histograms (n, 16) for frames (n, 12): position, tangent,
        binormal, shading normal."""
        fr = _f(frames).reshape(-1, 12)
        out = np.zeros((fr.shape[0], 16), np.float32)
        self.lib.xyzo_importons_query(fr.ctypes.data_as(C.c_void_p), fr.shape[0], out.ctypes.data_as(C.c_void_p))
        return out

    def encode_rgbe(self, film, scale: float, xyze: bool = False):
        """Pixels of the reference's .hdr writer, (H, W, 4) uint8 in file order."""
        film = _f(film)
        H, W = film.shape[:2]
        out = np.zeros((H, W, 4), np.uint8)
        self.lib.xyzo_encode_rgbe(film.ctypes.data_as(C.c_void_p), W, H, C.c_float(scale), int(xyze),
                                  out.ctypes.data_as(C.c_void_p))
        return out

    def tonemap(self, film, scale: float = 1.0, op: int = 0, exposure: float = 1.0, white: float = 0.0,
                dst_gamma: float = 2.2, src_gamma: float = 1.0, rgb: bool = False):
        """float2bmp's tone operators: BMP rows (H, stride) uint8, rows from the bottom."""
        film = _f(film)
        H, W = film.shape[:2]
        stride = (3 * W + 3) & ~3
        out = np.zeros((H, stride), np.uint8)
        self.lib.xyzo_tonemap(film.ctypes.data_as(C.c_void_p), W, H, C.c_float(scale), op, C.c_float(exposure),
                              C.c_float(white), C.c_float(dst_gamma), C.c_float(src_gamma), int(rgb),
                              out.ctypes.data_as(C.c_void_p))
        return out

    def set_camera(self, cam, width: int, height: int):
        eye = _f(cam.eye)
        at = _f(cam.at)
        self.lib.xyzo_set_camera_full(eye.ctypes.data_as(C.c_void_p), at.ctypes.data_as(C.c_void_p),
                                      C.c_float(cam.film_size), C.c_float(cam.focal_length),
                                      C.c_float(cam.f_number), width, height, int(cam.pinhole))
        self.width, self.height = width, height

    def scene_create(self, sd, kd_max_bucket: int = 16, kd_max_depth: int = 16):
        pos, tris, mat = _f(sd.positions), _i(sd.tris), _i(sd.tri_mat)
        alb, lit = _f(sd.albedo_xyz), _i(sd.is_light)
        nrm = _f(sd.normals) if sd.normals is not None else None
        pw = _f(sd.light_power_xyz)
        r = self.lib.xyzo_scene_create(pos.shape[0], pos.ctypes.data_as(C.c_void_p),
                                       None if nrm is None else nrm.ctypes.data_as(C.c_void_p),
                                       tris.shape[0], tris.ctypes.data_as(C.c_void_p),
                                       mat.ctypes.data_as(C.c_void_p), alb.shape[0],
                                       alb.ctypes.data_as(C.c_void_p), lit.ctypes.data_as(C.c_void_p),
                                       pw.ctypes.data_as(C.c_void_p), kd_max_bucket, kd_max_depth)
        if r < 0:
            raise ValueError("oracle port rejected the scene")
        self._keep = (pos, tris, mat, alb, lit, nrm, pw)
        return r

    def eval_path_record(self, px: int, py: int, s: int, seed: int, cap: int = 64):
        """One path with its traced segments: (xyz, dims, rays (n,6), tri, t, kind)."""
        out = np.zeros(3, np.float32)
        rays = np.zeros((cap, 6), np.float32)
        tri = np.zeros(cap, np.int32)
        t = np.zeros(cap, np.float32)
        kind = np.zeros(cap, np.int32)
        n = C.c_int(0)
        f = self.lib.xyzo_eval_path_record
        f.restype = C.c_int
        dims = f(px, py, s, C.c_uint64(seed), out.ctypes.data_as(C.c_void_p), cap,
                 rays.ctypes.data_as(C.c_void_p), tri.ctypes.data_as(C.c_void_p),
                 t.ctypes.data_as(C.c_void_p), kind.ctypes.data_as(C.c_void_p), C.byref(n))
        k = n.value
        return out, dims, rays[:k], tri[:k], t[:k], kind[:k]

    def set_spectra(self, albedo_spd, light_spd):
        a, l = _f(albedo_spd), _f(light_spd)
        self.lib.xyzo_scene_set_spectra(a.ctypes.data_as(C.c_void_p), l.ctypes.data_as(C.c_void_p))
        self._spectra = (a, l)

    def set_spectral(self, mode: int, hero: int = 1):
        """0: XYZ estimator; 1: binned (the reference's spectral estimator);
        2: continuous 380..720 nm; `hero` wavelengths per path."""
        self.lib.xyzo_set_spectral(int(mode), int(hero))

    def set_materials(self, albedo_xyz=None, emission=None):
        """Replaces the albedos (n_materials, 3) and / or sets the per-material
        emission scale (n_materials,); None leaves a table unchanged."""
        a = None if albedo_xyz is None else _f(albedo_xyz)
        e = None if emission is None else _f(emission)
        self.lib.xyzo_set_materials(None if a is None else a.ctypes.data_as(C.c_void_p),
                                    None if e is None else e.ctypes.data_as(C.c_void_p))

    def adjoint(self, dfilm, spp: int, seed: int, n_materials: int, s0: int = 0, nthreads: int = 0):
        """Gradient of sum(dfilm * film) over samples [s0, s0 + spp) with
        respect to albedo (n_materials, 3) and emission scale (n_materials,),
        float64 (per-contribution derivatives, XYZ estimator)."""
        df = _f(dfilm)
        assert df.shape == (self.height, self.width, 3)
        ga = np.zeros((n_materials, 3), np.float64)
        ge = np.zeros(n_materials, np.float64)
        self.lib.xyzo_adjoint(s0, spp, C.c_uint64(seed), df.ctypes.data_as(C.c_void_p),
                              ga.ctypes.data_as(C.c_void_p), ge.ctypes.data_as(C.c_void_p), nthreads)
        return ga, ge

    def philox_u01(self, seed, pixel, sample, dim):
        return self.lib.xyzo_philox_u01(C.c_uint64(seed), pixel, sample, dim)

    def kdtree_stats(self):
        out = np.zeros(8, np.int64)
        self.lib.xyzo_kdtree_stats(out.ctypes.data_as(C.c_void_p))
        return dict(zip(["nodes", "leaves", "empty_leaves", "refs", "max_depth", "tris", "_6", "_7"],
                        out.tolist()))

    def max_threads(self):
        return self.lib.xyzo_max_threads()


def twin_available() -> bool:
    return os.path.exists(os.path.join(REF_DIR, "libxyztwin_thinlens.so"))


class TwinLib:
    """The reference's spectral renderer (renderer/, tgir) built from its
    sources (thin-lens camera; its pinhole branch does not compile).  Each row
    of a sample pass uses its own std::mt19937_64, so comparisons with it are
    statistical."""

    def __init__(self):
        path = os.path.join(REF_DIR, "libxyztwin_thinlens.so")
        if not os.path.exists(path):
            raise FileNotFoundError(f"spectral reference oracle not built: {path}")
        self.lib = C.CDLL(path)
        L = self.lib
        L.xyztwin_scene_create.restype = C.c_int
        L.xyztwin_scene_create.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p,
                                           C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
        L.xyztwin_set_camera.argtypes = [C.c_void_p, C.c_void_p, C.c_float, C.c_float, C.c_float,
                                         C.c_int, C.c_int]
        L.xyztwin_set_path_params.argtypes = [C.c_int, C.c_double]
        L.xyztwin_render.argtypes = [C.c_int, C.c_int, C.c_ulonglong, C.c_void_p, C.c_int]
        L.xyztwin_light_spd.argtypes = [C.c_void_p]

    def light_spd(self):
        out = np.zeros(31, np.float32)
        self.lib.xyztwin_light_spd(out.ctypes.data_as(C.c_void_p))
        return out

    def scene_create(self, sd):
        pos, tris, mat = _f(sd.positions), _i(sd.tris), _i(sd.tri_mat)
        spd, lit = _f(sd.albedo_spd), _i(sd.is_light)
        nrm = _f(sd.normals) if sd.normals is not None else None
        r = self.lib.xyztwin_scene_create(pos.shape[0], pos.ctypes.data_as(C.c_void_p),
                                          None if nrm is None else nrm.ctypes.data_as(C.c_void_p),
                                          tris.shape[0], tris.ctypes.data_as(C.c_void_p),
                                          mat.ctypes.data_as(C.c_void_p), spd.shape[0],
                                          spd.ctypes.data_as(C.c_void_p), lit.ctypes.data_as(C.c_void_p))
        if r < 0:
            raise ValueError("spectral reference rejected the scene")
        self._keep = (pos, tris, mat, spd, lit, nrm)
        return r

    def set_camera(self, cam, width, height):
        eye, at = _f(cam.eye), _f(cam.at)
        self.lib.xyztwin_set_camera(eye.ctypes.data_as(C.c_void_p), at.ctypes.data_as(C.c_void_p),
                                    C.c_float(cam.film_size), C.c_float(cam.focal_length),
                                    C.c_float(cam.f_number), width, height)
        self.width, self.height = width, height

    def set_path_params(self, max_depth: int, rr_threshold: float = 0.2):
        self.lib.xyztwin_set_path_params(max_depth + 1, rr_threshold)

    def render(self, spp, seed, s0=0, nthreads=0):
        film = np.zeros((self.height, self.width, 3), np.float32)
        self.lib.xyztwin_render(s0, spp, C.c_ulonglong(seed), film.ctypes.data_as(C.c_void_p), nthreads)
        return film


FILM_REF_PATH = os.path.join(REF_DIR, "xyzref_hdr")


def ref_film_available() -> bool:
    return os.path.exists(FILM_REF_PATH)


class RefFilmLib:
    """The reference's Radiance writer, ImageFilm::SaveAsHdr, built from its
    sources into the program oracle/_ref/xyzref_hdr (run in its own process)."""

    def save_hdr(self, path: str, film, spp: float):
        import subprocess
        film = _f(film)
        H, W = film.shape[:2]
        raw = path + ".film.f32"
        film.tofile(raw)
        try:
            subprocess.run([FILM_REF_PATH, raw, str(W), str(H), repr(float(spp)), path], check=True)
        finally:
            os.remove(raw)
