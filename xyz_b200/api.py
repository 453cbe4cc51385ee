"""ctypes binding of libxyzgpu.so (the C ABI declared in include/xyzgpu.h).

This module is plumbing for Python callers (tests, benchmarks): every call goes
through the C ABI to the CUDA kernels.  There is no CPU code path; if the shared
library is missing or no sm_100 device is present, calls raise.
Device buffers are torch CUDA tensors (torch provides memory and streams only).
"""

from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libxyzgpu.so")

XYZGPU_BUILD_DEVICE = 0
XYZGPU_BUILD_HOST = 1
XYZGPU_FILM_DEVICE = 0
XYZGPU_FILM_HOST = 1

ERRORS = {0: "OK", -1: "XYZGPU_E_INVALID", -2: "XYZGPU_E_CUDA", -3: "XYZGPU_E_NOMEM",
          -4: "XYZGPU_E_LIMIT", -5: "XYZGPU_E_NODEVICE"}

# every symbol declared in include/xyzgpu.h
EXPORTED = [
    "xyzgpu_build_params_default", "xyzgpu_scene_create", "xyzgpu_scene_destroy",
    "xyzgpu_scene_stats_get", "xyzgpu_scene_copy_tree", "xyzgpu_trace_closest",
    "xyzgpu_trace_closest_counted", "xyzgpu_render_params_default", "xyzgpu_render",
    "xyzgpu_render_counters_get", "xyzgpu_render_profile_get", "xyzgpu_render_noalloc",
    "xyzgpu_philox_u01", "xyzgpu_last_error", "xyzgpu_abi_version", "xyzgpu_adjoint",
    "xyzgpu_scene_set_materials", "xyzgpu_scene_get_materials",
    "xyzgpu_batch_config_default", "xyzgpu_batch_create", "xyzgpu_batch_launch",
    "xyzgpu_batch_set_sample_offsets", "xyzgpu_batch_autotune", "xyzgpu_batch_stats_get",
    "xyzgpu_batch_config_get", "xyzgpu_batch_destroy", "xyzgpu_render_batch",
    "xyzgpu_guide_config_default", "xyzgpu_guide_create", "xyzgpu_guide_destroy",
    "xyzgpu_guide_get_params", "xyzgpu_guide_set_params", "xyzgpu_guide_forward",
    "xyzgpu_guide_gradient", "xyzgpu_guide_train_step", "xyzgpu_render_guided", "xyzgpu_guide_stats_get",
    "xyzgpu_guide_reserve", "xyzgpu_film_encode_rgbe", "xyzgpu_hdr_write", "xyzgpu_tonemap_params_default",
    "xyzgpu_film_tonemap", "xyzgpu_bmp_write", "xyzgpu_checkpoint_save", "xyzgpu_checkpoint_load",
    "xyzgpu_film_save_hdr", "xyzgpu_film_save_bmp", "xyzgpu_importon_config_default",
    "xyzgpu_importons_create", "xyzgpu_importons_destroy", "xyzgpu_importons_get", "xyzgpu_importons_query",
    "xyzgpu_render_importon", "xyzgpu_named_spectrum", "xyzgpu_spectrum_to_xyz",
]


class XyzGpuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERRORS.get(code, code)}: {msg}")
        self.code = code


class SceneDesc(C.Structure):
    _fields_ = [("positions", C.c_void_p), ("normals", C.c_void_p), ("n_vertices", C.c_int),
                ("triangles", C.c_void_p), ("tri_material", C.c_void_p), ("n_triangles", C.c_int),
                ("albedo_xyz", C.c_void_p), ("is_light", C.c_void_p), ("n_materials", C.c_int),
                ("light_power_xyz", C.c_float * 3), ("albedo_spd", C.c_void_p),
                ("light_power_spd", C.c_float * 31), ("material_kind", C.c_void_p), ("shininess", C.c_void_p)]


MATERIAL_LAMBERT, MATERIAL_MIRROR, MATERIAL_METAL = 0, 2, 3


class BuildParams(C.Structure):
    _fields_ = [("leaf_max_tris", C.c_int), ("max_depth", C.c_int), ("cost_traversal", C.c_float),
                ("cost_intersect", C.c_float), ("empty_bonus", C.c_float), ("bins", C.c_int),
                ("builder", C.c_int), ("max_refs_factor", C.c_int)]


class SceneStats(C.Structure):
    _fields_ = [("n_triangles", C.c_int64), ("n_lights", C.c_int64), ("n_nodes", C.c_int64),
                ("n_leaves", C.c_int64), ("n_empty_leaves", C.c_int64), ("n_leaf_refs", C.c_int64),
                ("max_depth", C.c_int64), ("device_bytes", C.c_int64), ("build_ms", C.c_double),
                ("light_area", C.c_float), ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3)]


class TraceCounters(C.Structure):
    _fields_ = [("rays", C.c_uint64), ("nodes_visited", C.c_uint64), ("leaves_visited", C.c_uint64),
                ("tri_tests", C.c_uint64), ("hits", C.c_uint64)]


class CameraDesc(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("at", C.c_float * 3), ("film_size", C.c_float),
                ("focal_length", C.c_float), ("f_number", C.c_float), ("pinhole", C.c_int)]


class RenderParams(C.Structure):
    _fields_ = [("width", C.c_int), ("height", C.c_int), ("spp", C.c_int), ("spp_offset", C.c_int),
                ("max_depth", C.c_int), ("rr_start_depth", C.c_int), ("rr_threshold", C.c_float),
                ("seed", C.c_uint64), ("film_location", C.c_int), ("accumulate", C.c_int),
                ("wave_paths", C.c_int), ("profile", C.c_int), ("spectral", C.c_int),
                ("hero_wavelengths", C.c_int), ("row_begin", C.c_int), ("row_end", C.c_int),
                ("row_step", C.c_int)]

SPECTRAL_MODES = {"off": 0, "xyz": 0, "binned": 1, "continuous": 2}


GUIDE_PARAMS = 28992
GUIDE_OUTPUTS = 64


class GuideConfig(C.Structure):
    _fields_ = [("alpha", C.c_float), ("learning_rate", C.c_float), ("batch_size", C.c_int),
                ("steps_per_pass", C.c_int), ("train_bounces", C.c_int), ("seed", C.c_uint64),
                ("guide_bounces", C.c_int)]


class GuideStats(C.Structure):
    _fields_ = [("adam_steps", C.c_uint64), ("trained_records", C.c_uint64)]


class ImportonConfig(C.Structure):
    _fields_ = [("particles", C.c_int), ("max_depth", C.c_int), ("min_depth", C.c_int), ("radius", C.c_float),
                ("seed", C.c_uint64), ("guide_bounces", C.c_int)]


class TonemapParams(C.Structure):
    _fields_ = [("scale", C.c_float), ("op", C.c_int), ("exposure", C.c_float), ("white", C.c_float),
                ("dst_gamma", C.c_float), ("src_gamma", C.c_float), ("rgb", C.c_int)]


TONEMAP_OPS = {"film": 0, "linear": 1, "reinhard": 2, "reinhard_white": 3}


class BatchJobDesc(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", CameraDesc), ("params", RenderParams),
                ("film", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("wave_paths", C.c_int), ("tile", C.c_int), ("trace_ctas_per_sm", C.c_int),
                ("use_graph", C.c_int)]


class BatchStats(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("waves", C.c_uint64), ("kernel_launches_per_launch", C.c_uint64),
                ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("device_bytes", C.c_int64),
                ("graph_nodes", C.c_int), ("graph_top_nodes", C.c_int)]


class RenderProfile(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 6), ("ms", C.c_double * 6), ("ext_rays", C.c_uint64),
                ("ext_nodes", C.c_uint64), ("ext_leaves", C.c_uint64), ("ext_tri_tests", C.c_uint64),
                ("shadow_rays", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_leaves", C.c_uint64),
                ("shadow_tri_tests", C.c_uint64), ("shadow_visible", C.c_uint64),
                ("iterations", C.c_uint32), ("ext_rays_by_iter", C.c_uint64 * 64),
                ("shadow_rays_by_iter", C.c_uint64 * 64)]


KERNEL_CLASSES = ["raygen", "trace_extension", "shade", "trace_shadow", "film", "guide"]


class RenderCounters(C.Structure):
    _fields_ = [("paths", C.c_uint64), ("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64),
                ("shadow_hits_visible", C.c_uint64), ("waves", C.c_uint64), ("kernel_launches", C.c_uint64)]


_LIB = None


def load_library(path: str = LIB_PATH) -> C.CDLL:
    """Loads libxyzgpu.so (raises if it has not been built)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `make -C xyz_b200/csrc` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(path)
    L.xyzgpu_last_error.restype = C.c_char_p
    L.xyzgpu_abi_version.restype = C.c_int
    L.xyzgpu_scene_create.argtypes = [C.POINTER(SceneDesc), C.POINTER(BuildParams), C.POINTER(C.c_void_p)]
    L.xyzgpu_scene_destroy.argtypes = [C.c_void_p]
    L.xyzgpu_scene_stats_get.argtypes = [C.c_void_p, C.POINTER(SceneStats)]
    L.xyzgpu_scene_copy_tree.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.xyzgpu_trace_closest.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.xyzgpu_trace_closest_counted.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p,
                                               C.POINTER(TraceCounters)]
    L.xyzgpu_render.argtypes = [C.c_void_p, C.POINTER(CameraDesc), C.POINTER(RenderParams), C.c_void_p,
                                C.c_void_p]
    L.xyzgpu_render_noalloc.argtypes = [C.c_void_p, C.POINTER(CameraDesc), C.POINTER(RenderParams),
                                        C.c_void_p, C.c_void_p]
    L.xyzgpu_render_counters_get.argtypes = [C.c_void_p, C.POINTER(RenderCounters)]
    L.xyzgpu_render_profile_get.argtypes = [C.c_void_p, C.POINTER(RenderProfile)]
    L.xyzgpu_philox_u01.restype = C.c_float
    L.xyzgpu_philox_u01.argtypes = [C.c_uint64, C.c_uint32, C.c_uint32, C.c_uint32]
    L.xyzgpu_adjoint.argtypes = [C.c_void_p, C.POINTER(CameraDesc), C.POINTER(RenderParams), C.c_void_p,
                                 C.c_void_p, C.c_void_p, C.c_void_p]
    L.xyzgpu_scene_set_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.xyzgpu_scene_get_materials.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p]
    L.xyzgpu_batch_config_default.argtypes = [C.POINTER(BatchConfig)]
    L.xyzgpu_batch_create.argtypes = [C.POINTER(BatchJobDesc), C.c_int, C.POINTER(BatchConfig),
                                      C.POINTER(C.c_void_p)]
    L.xyzgpu_batch_launch.argtypes = [C.c_void_p, C.c_void_p]
    L.xyzgpu_batch_set_sample_offsets.argtypes = [C.c_void_p, C.c_void_p]
    L.xyzgpu_batch_autotune.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_void_p, C.POINTER(BatchConfig)]
    L.xyzgpu_batch_stats_get.argtypes = [C.c_void_p, C.POINTER(BatchStats)]
    L.xyzgpu_batch_config_get.argtypes = [C.c_void_p, C.POINTER(BatchConfig)]
    L.xyzgpu_batch_destroy.argtypes = [C.c_void_p]
    L.xyzgpu_render_batch.argtypes = [C.POINTER(BatchJobDesc), C.c_int, C.POINTER(BatchConfig), C.c_void_p]
    L.xyzgpu_guide_config_default.argtypes = [C.POINTER(GuideConfig)]
    L.xyzgpu_guide_create.argtypes = [C.c_void_p, C.POINTER(GuideConfig), C.POINTER(C.c_void_p)]
    L.xyzgpu_guide_destroy.argtypes = [C.c_void_p]
    L.xyzgpu_guide_get_params.argtypes = [C.c_void_p, C.c_void_p]
    L.xyzgpu_guide_set_params.argtypes = [C.c_void_p, C.c_void_p]
    L.xyzgpu_guide_forward.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.xyzgpu_guide_gradient.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_float, C.c_void_p, C.c_void_p]
    L.xyzgpu_guide_train_step.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
    L.xyzgpu_render_guided.argtypes = [C.c_void_p, C.POINTER(CameraDesc), C.POINTER(RenderParams), C.c_int,
                                       C.c_void_p, C.c_void_p]
    L.xyzgpu_guide_stats_get.argtypes = [C.c_void_p, C.POINTER(GuideStats)]
    L.xyzgpu_guide_reserve.argtypes = [C.c_void_p, C.c_int64, C.c_int, C.c_void_p]
    L.xyzgpu_importon_config_default.argtypes = [C.POINTER(ImportonConfig)]
    L.xyzgpu_importons_create.argtypes = [C.c_void_p, C.POINTER(ImportonConfig), C.c_void_p, C.c_int64, C.c_void_p,
                                          C.POINTER(C.c_void_p)]
    L.xyzgpu_importons_destroy.argtypes = [C.c_void_p]
    L.xyzgpu_importons_get.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int64)]
    L.xyzgpu_importons_query.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p]
    L.xyzgpu_render_importon.argtypes = [C.c_void_p, C.POINTER(CameraDesc), C.POINTER(RenderParams), C.c_void_p,
                                         C.c_void_p]
    L.xyzgpu_named_spectrum.argtypes = [C.c_char_p, C.c_void_p]
    L.xyzgpu_spectrum_to_xyz.argtypes = [C.c_void_p, C.c_void_p]
    L.xyzgpu_film_encode_rgbe.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_float, C.c_int, C.c_void_p, C.c_void_p]
    L.xyzgpu_hdr_write.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int]
    L.xyzgpu_tonemap_params_default.argtypes = [C.POINTER(TonemapParams)]
    L.xyzgpu_film_tonemap.argtypes = [C.c_void_p, C.c_int, C.c_int, C.POINTER(TonemapParams), C.c_void_p,
                                      C.c_void_p, C.c_void_p]
    L.xyzgpu_bmp_write.argtypes = [C.c_char_p, C.c_void_p, C.c_int, C.c_int]
    L.xyzgpu_checkpoint_save.argtypes = [C.c_char_p, C.POINTER(RenderParams), C.c_int, C.c_void_p]
    L.xyzgpu_checkpoint_load.argtypes = [C.c_char_p, C.POINTER(RenderParams), C.POINTER(C.c_int), C.c_void_p]
    L.xyzgpu_build_params_default.argtypes = [C.POINTER(BuildParams)]
    L.xyzgpu_render_params_default.argtypes = [C.POINTER(RenderParams)]
    _LIB = L
    return L


def _check(rc: int):
    if rc != 0:
        raise XyzGpuError(rc, _LIB.xyzgpu_last_error().decode(errors="replace"))


def default_build_params(**kw) -> BuildParams:
    bp = BuildParams()
    load_library().xyzgpu_build_params_default(C.byref(bp))
    for k, v in kw.items():
        if k == "builder" and isinstance(v, str):
            v = {"device": XYZGPU_BUILD_DEVICE, "host": XYZGPU_BUILD_HOST}[v]
        setattr(bp, k, v)
    return bp


def camera_desc(camera) -> "CameraDesc":
    cam = CameraDesc()
    for k in range(3):
        cam.eye[k] = float(camera.eye[k])
        cam.at[k] = float(camera.at[k])
    cam.film_size = float(camera.film_size)
    cam.focal_length = float(camera.focal_length)
    cam.f_number = float(camera.f_number)
    cam.pinhole = int(bool(camera.pinhole))
    return cam


def render_params(width: int, height: int, spp: int, *, seed: int = 0, spp_offset: int = 0,
                  max_depth: int = 15, rr_start_depth: int = 1, rr_threshold: float = 0.2,
                  accumulate: bool = False, wave_paths: int = 0, profile: int = 0, spectral="off",
                  hero_wavelengths: int = 4, rows=None) -> "RenderParams":
    rp = RenderParams()
    load_library().xyzgpu_render_params_default(C.byref(rp))
    rp.width, rp.height, rp.spp, rp.spp_offset = width, height, spp, spp_offset
    rp.max_depth, rp.rr_start_depth, rp.rr_threshold = max_depth, rr_start_depth, rr_threshold
    rp.seed = seed
    rp.accumulate = int(bool(accumulate))
    rp.wave_paths = wave_paths
    rp.profile = profile
    rp.spectral = SPECTRAL_MODES[spectral] if isinstance(spectral, str) else int(spectral)
    rp.hero_wavelengths = hero_wavelengths
    if rows is not None:
        # (begin, end) or (begin, end, step): rows begin, begin + step, ... < end
        rp.row_begin, rp.row_end = int(rows[0]), int(rows[1])
        if len(rows) > 2:
            rp.row_step = int(rows[2])
    return rp


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        import torch
        return torch.cuda.current_stream().cuda_stream
    return getattr(stream, "cuda_stream", stream)


class Scene:
    """A scene on the current CUDA device (xyzgpu_scene_create).

    Mirrors the reference's Scene::Load + Scene::Build; trace() is the batch
    Scene::FindIntersection and render() the PathTracer::run loop."""

    def __init__(self, sd, **build_kw):
        L = load_library()
        self._arrays = []

        def keep(a, dt):
            a = np.ascontiguousarray(a, dtype=dt)
            self._arrays.append(a)
            return a.ctypes.data

        d = SceneDesc()
        d.positions = keep(sd.positions, np.float32)
        d.normals = keep(sd.normals, np.float32) if sd.normals is not None else None
        d.n_vertices = int(sd.positions.shape[0])
        d.triangles = keep(sd.tris, np.int32)
        d.tri_material = keep(sd.tri_mat, np.int32)
        d.n_triangles = int(sd.tris.shape[0])
        d.albedo_xyz = keep(sd.albedo_xyz, np.float32)
        d.is_light = keep(sd.is_light, np.int32)
        d.n_materials = int(sd.albedo_xyz.shape[0])
        for k in range(3):
            d.light_power_xyz[k] = float(sd.light_power_xyz[k])
        if getattr(sd, "albedo_spd", None) is not None:
            d.albedo_spd = keep(sd.albedo_spd, np.float32)
            for k in range(31):
                d.light_power_spd[k] = float(sd.light_power_spd[k])
        if getattr(sd, "material_kind", None) is not None:
            d.material_kind = keep(sd.material_kind, np.int32)
            # no exponents: NULL, which the library accepts unless a material is metal
            d.shininess = keep(sd.shininess, np.float32) if sd.shininess is not None else None
        bp = default_build_params(**build_kw)
        h = C.c_void_p()
        _check(L.xyzgpu_scene_create(C.byref(d), C.byref(bp), C.byref(h)))
        self.handle = h
        self._arrays = []
        self.data = sd

    def close(self):
        if getattr(self, "handle", None):
            _LIB.xyzgpu_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def stats(self) -> dict:
        s = SceneStats()
        _check(_LIB.xyzgpu_scene_stats_get(self.handle, C.byref(s)))
        out = {f: getattr(s, f) for f, _ in SceneStats._fields_}
        out["bounds_min"] = list(s.bounds_min)
        out["bounds_max"] = list(s.bounds_max)
        return out

    def tree(self):
        st = self.stats()
        nodes = np.zeros(2 * st["n_nodes"], np.uint32)
        refs = np.zeros(max(1, st["n_leaf_refs"]), np.int32)
        _check(_LIB.xyzgpu_scene_copy_tree(self.handle, nodes.ctypes.data, refs.ctypes.data))
        return nodes.reshape(-1, 2), refs[: st["n_leaf_refs"]]

    # -- closest hit -----------------------------------------------------
    def trace_device(self, rays, hits, stream=None, counted: bool = False):
        """rays: CUDA float32 tensor (n, 8) = o.xyz, tmin, d.xyz, tmax; hits:
        CUDA float32 tensor (n, 4).  Returns TraceCounters if counted."""
        n = int(rays.shape[0])
        sp = _stream_ptr(stream)
        if counted:
            c = TraceCounters()
            _check(_LIB.xyzgpu_trace_closest_counted(self.handle, rays.data_ptr(), n, hits.data_ptr(), sp,
                                                     C.byref(c)))
            return {f: getattr(c, f) for f, _ in TraceCounters._fields_}
        _check(_LIB.xyzgpu_trace_closest(self.handle, rays.data_ptr(), n, hits.data_ptr(), sp))
        return None

    def trace(self, org, dirs, tmin: float = 1e-5, tmax: float = float("inf")):
        """Host convenience: numpy (n,3) origins/directions -> (tri, t, f, g, back)."""
        import torch
        org = np.asarray(org, np.float32)
        dirs = np.asarray(dirs, np.float32)
        n = org.shape[0]
        r = np.empty((n, 8), np.float32)
        r[:, 0:3] = org
        r[:, 3] = tmin
        r[:, 4:7] = dirs
        r[:, 7] = tmax
        rays = torch.from_numpy(r).cuda()
        hits = torch.empty((n, 4), dtype=torch.float32, device="cuda")
        self.trace_device(rays, hits)
        torch.cuda.synchronize()
        h = hits.cpu().numpy()
        code = h[:, 3].view(np.int32)
        tri = np.where(code >= 0, code >> 1, -1).astype(np.int32)
        back = np.where(code >= 0, code & 1, 0).astype(np.int32)
        return tri, h[:, 0].copy(), h[:, 1].copy(), h[:, 2].copy(), back

    # -- rendering --------------------------------------------------------
    def render(self, camera, width: int, height: int, spp: int, *, seed: int = 0,
               spp_offset: int = 0, max_depth: int = 15, rr_start_depth: int = 1,
               rr_threshold: float = 0.2, film=None, accumulate: bool = False,
               wave_paths: int = 0, profile: int = 0, spectral="off", hero_wavelengths: int = 4,
               rows=None, stream=None):
        """Renders into `film`: a CUDA tensor (H, W, 3) (device film) or a numpy
        float32 array (host film).  Allocates a CUDA tensor if film is None.
        rows = (first, end): only that band of image rows.  Returns the film
        (sums over samples, not means)."""
        cam = camera_desc(camera)
        rp = render_params(width, height, spp, seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                           rr_start_depth=rr_start_depth, rr_threshold=rr_threshold,
                           accumulate=accumulate, wave_paths=wave_paths, profile=profile,
                           spectral=spectral, hero_wavelengths=hero_wavelengths, rows=rows)
        if film is None:
            import torch
            film = torch.zeros((height, width, 3), dtype=torch.float32, device="cuda")
        if isinstance(film, np.ndarray):
            assert film.dtype == np.float32 and film.flags["C_CONTIGUOUS"] and film.size == width * height * 3
            rp.film_location = XYZGPU_FILM_HOST
            ptr = film.ctypes.data
        else:
            assert film.is_cuda and film.dtype.__str__() == "torch.float32" and film.is_contiguous()
            rp.film_location = XYZGPU_FILM_DEVICE
            ptr = film.data_ptr()
        _check(_LIB.xyzgpu_render(self.handle, C.byref(cam), C.byref(rp), ptr, _stream_ptr(stream)))
        return film

    def render_noalloc(self, camera, width: int, height: int, spp: int, film, *, seed: int = 0,
                       spp_offset: int = 0, max_depth: int = 15, rr_start_depth: int = 1,
                       rr_threshold: float = 0.2, accumulate: bool = False, wave_paths: int = 0,
                       stream=None):
        """xyzgpu_render_noalloc: same image as render(), for callers that cannot
        allocate device memory while rendering.  `film` must be a CUDA tensor
        (H, W, 3) float32 that the caller owns; nothing is allocated."""
        cam = camera_desc(camera)
        rp = render_params(width, height, spp, seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                           rr_start_depth=rr_start_depth, rr_threshold=rr_threshold,
                           accumulate=accumulate, wave_paths=wave_paths)
        rp.film_location = XYZGPU_FILM_DEVICE
        _check(_LIB.xyzgpu_render_noalloc(self.handle, C.byref(cam), C.byref(rp), film.data_ptr(),
                                          _stream_ptr(stream)))
        return film

    def render_profile(self) -> dict:
        p = RenderProfile()
        _check(_LIB.xyzgpu_render_profile_get(self.handle, C.byref(p)))
        skip = ("launches", "ms", "ext_rays_by_iter", "shadow_rays_by_iter")
        out = {f: getattr(p, f) for f, _ in RenderProfile._fields_ if f not in skip}
        out["ext_rays_by_iter"] = list(p.ext_rays_by_iter)[: p.iterations]
        out["shadow_rays_by_iter"] = list(p.shadow_rays_by_iter)[: p.iterations]
        out["launches"] = dict(zip(KERNEL_CLASSES, list(p.launches)))
        out["ms"] = dict(zip(KERNEL_CLASSES, list(p.ms)))
        return out

    def render_counters(self) -> dict:
        c = RenderCounters()
        _check(_LIB.xyzgpu_render_counters_get(self.handle, C.byref(c)))
        return {f: getattr(c, f) for f, _ in RenderCounters._fields_}

    # -- differentiable rendering ----------------------------------------
    def set_materials(self, albedo_xyz=None, emission=None, stream=None):
        """xyzgpu_scene_set_materials: albedo (n_materials, 3) and / or emission
        scale (n_materials,), as numpy arrays (host) or CUDA float32 tensors
        (device; read on `stream`)."""
        a, e = albedo_xyz, emission
        on_device = any(x is not None and not isinstance(x, np.ndarray) for x in (a, e))
        if on_device:
            for x in (a, e):
                if x is not None:
                    assert x.is_cuda and str(x.dtype) == "torch.float32" and x.is_contiguous()
            _check(_LIB.xyzgpu_scene_set_materials(self.handle, None if a is None else a.data_ptr(),
                                                   None if e is None else e.data_ptr(), XYZGPU_FILM_DEVICE,
                                                   _stream_ptr(stream)))
            return
        keep = []
        ptrs = []
        for x in (a, e):
            if x is None:
                ptrs.append(None)
            else:
                x = np.ascontiguousarray(x, np.float32)
                keep.append(x)
                ptrs.append(x.ctypes.data)
        _check(_LIB.xyzgpu_scene_set_materials(self.handle, ptrs[0], ptrs[1], XYZGPU_FILM_HOST,
                                               _stream_ptr(stream)))

    def get_materials(self):
        """Current (albedo (n_materials, 3), emission scale (n_materials,)) as numpy."""
        nm = int(self.data.albedo_xyz.shape[0])
        a = np.zeros((nm, 3), np.float32)
        e = np.zeros(nm, np.float32)
        _check(_LIB.xyzgpu_scene_get_materials(self.handle, a.ctypes.data, e.ctypes.data))
        return a, e

    def adjoint(self, camera, width: int, height: int, spp: int, d_film, *, seed: int = 0,
                spp_offset: int = 0, max_depth: int = 15, rr_start_depth: int = 1,
                rr_threshold: float = 0.2, wave_paths: int = 0, d_albedo=None, d_emission=None,
                stream=None):
        """xyzgpu_adjoint: gradient of sum(d_film * film) with respect to the
        materials' albedo and emission scale, for the film render() gives with the
        same arguments.  d_film: CUDA float32 tensor (H, W, 3).  Returns
        (d_albedo (n_materials, 3), d_emission (n_materials,)) CUDA tensors
        (accumulated into the given ones)."""
        import torch
        nm = int(self.data.albedo_xyz.shape[0])
        if d_albedo is None:
            d_albedo = torch.zeros((nm, 3), dtype=torch.float32, device=d_film.device)
        if d_emission is None:
            d_emission = torch.zeros(nm, dtype=torch.float32, device=d_film.device)
        assert d_film.is_cuda and d_film.is_contiguous() and tuple(d_film.shape) == (height, width, 3)
        cam = camera_desc(camera)
        rp = render_params(width, height, spp, seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                           rr_start_depth=rr_start_depth, rr_threshold=rr_threshold, wave_paths=wave_paths)
        _check(_LIB.xyzgpu_adjoint(self.handle, C.byref(cam), C.byref(rp), d_film.data_ptr(),
                                   d_albedo.data_ptr(), d_emission.data_ptr(), _stream_ptr(stream)))
        return d_albedo, d_emission


# ------------------------------------------------------------------ importance-driven tracing
class Importons:
    """xyzgpu_importons: the light-importance map of the reference's
    importance-driven path tracer, built by tracing light particles (or from
    given importons, an (n, 6) array of position and incoming direction)."""

    def __init__(self, scene: "Scene", importons=None, stream=None, **config):
        L = load_library()
        cfg = ImportonConfig()
        L.xyzgpu_importon_config_default(C.byref(cfg))
        for k, v in config.items():
            setattr(cfg, k, v)
        h = C.c_void_p()
        ptr, n = None, 0
        if importons is not None:
            arr = np.ascontiguousarray(importons, np.float32).reshape(-1, 6)
            ptr, n = arr.ctypes.data, arr.shape[0]
        _check(L.xyzgpu_importons_create(scene.handle, C.byref(cfg), ptr, n, _stream_ptr(stream), C.byref(h)))
        self.handle = h
        self.scene = scene

    def close(self):
        if getattr(self, "handle", None):
            _LIB.xyzgpu_importons_destroy(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def count(self) -> int:
        n = C.c_int64()
        _check(_LIB.xyzgpu_importons_get(self.handle, None, C.byref(n)))
        return n.value

    def importons(self) -> np.ndarray:
        n = self.count()
        out = np.zeros((max(n, 1), 6), np.float32)
        k = C.c_int64()
        _check(_LIB.xyzgpu_importons_get(self.handle, out.ctypes.data, C.byref(k)))
        return out[:n]

    def query(self, frames, stream=None):
        """frames: CUDA float32 (n, 12) -> cumulative histograms (n, 16)."""
        import torch
        n = int(frames.shape[0])
        out = torch.empty((n, 16), dtype=torch.float32, device=frames.device)
        _check(_LIB.xyzgpu_importons_query(self.handle, frames.contiguous().data_ptr(), n, out.data_ptr(),
                                           _stream_ptr(stream)))
        return out

    def render(self, camera, width: int, height: int, spp: int, *, seed: int = 0, spp_offset: int = 0,
               max_depth: int = 15, rr_start_depth: int = 1, rr_threshold: float = 0.2, film=None,
               accumulate: bool = False, wave_paths: int = 0, rows=None, profile: int = 0, stream=None):
        """xyzgpu_render_importon into a CUDA film (H, W, 3) of sums."""
        import torch
        if film is None:
            film = torch.zeros((height, width, 3), dtype=torch.float32, device="cuda")
        cam = camera_desc(camera)
        rp = render_params(width, height, spp, seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                           rr_start_depth=rr_start_depth, rr_threshold=rr_threshold, accumulate=accumulate,
                           wave_paths=wave_paths, profile=profile, rows=rows)
        rp.film_location = XYZGPU_FILM_DEVICE
        _check(_LIB.xyzgpu_render_importon(self.handle, C.byref(cam), C.byref(rp), film.data_ptr(),
                                           _stream_ptr(stream)))
        return film


# ------------------------------------------------------------------ film output
def encode_rgbe(film, scale: float, xyze: bool = False, stream=None):
    """xyzgpu_film_encode_rgbe: the .hdr pixels of a CUDA film (H, W, 3) of
    sums, as a CUDA uint8 tensor (H, W, 4) in file order."""
    import torch
    H, W = int(film.shape[0]), int(film.shape[1])
    out = torch.empty((H, W, 4), dtype=torch.uint8, device=film.device)
    _check(load_library().xyzgpu_film_encode_rgbe(film.contiguous().data_ptr(), W, H, float(scale), int(xyze),
                                                  out.data_ptr(), _stream_ptr(stream)))
    return out


def write_hdr(path: str, rgbe, xyze: bool = False):
    """xyzgpu_hdr_write from host pixels (H, W, 4) uint8 in file order."""
    a = np.ascontiguousarray(rgbe.cpu().numpy() if hasattr(rgbe, "cpu") else rgbe, np.uint8)
    _check(load_library().xyzgpu_hdr_write(path.encode(), a.ctypes.data, a.shape[1], a.shape[0], int(xyze)))


def save_hdr(path: str, film, spp: float, xyze: bool = False):
    """The reference's ImageFilm::SaveAsHdr for a CUDA film of sums: device
    encode, host file."""
    write_hdr(path, encode_rgbe(film, 1.0 / spp, xyze), xyze)


def tonemap(film, scale: float = 1.0, op="film", exposure: float = 1.0, white: float = 0.0,
            dst_gamma: float = 2.2, src_gamma: float = 1.0, rgb: bool = False, stream=None):
    """xyzgpu_film_tonemap: BMP pixel rows (H, stride) uint8 of a CUDA film."""
    import torch
    L = load_library()
    H, W = int(film.shape[0]), int(film.shape[1])
    tp = TonemapParams()
    L.xyzgpu_tonemap_params_default(C.byref(tp))
    tp.scale, tp.exposure, tp.white = float(scale), float(exposure), float(white)
    tp.op = TONEMAP_OPS[op] if isinstance(op, str) else int(op)
    tp.dst_gamma, tp.src_gamma, tp.rgb = float(dst_gamma), float(src_gamma), int(bool(rgb))
    stride = (3 * W + 3) & ~3
    out = torch.empty((H, stride), dtype=torch.uint8, device=film.device)
    word = torch.zeros(1, dtype=torch.int32, device=film.device)
    _check(L.xyzgpu_film_tonemap(film.contiguous().data_ptr(), W, H, C.byref(tp), out.data_ptr(), word.data_ptr(),
                                 _stream_ptr(stream)))
    return out


def write_bmp(path: str, bgr, width: int, height: int):
    a = np.ascontiguousarray(bgr.cpu().numpy() if hasattr(bgr, "cpu") else bgr, np.uint8)
    _check(load_library().xyzgpu_bmp_write(path.encode(), a.ctypes.data, int(width), int(height)))


def save_checkpoint(path: str, params: "RenderParams", spp_done: int, film):
    """xyzgpu_checkpoint_save from a host film (H, W, 3) float32 of sums."""
    a = np.ascontiguousarray(film.cpu().numpy() if hasattr(film, "cpu") else film, np.float32)
    _check(load_library().xyzgpu_checkpoint_save(path.encode(), C.byref(params), int(spp_done), a.ctypes.data))


def load_checkpoint(path: str):
    """xyzgpu_checkpoint_load -> (RenderParams, spp_done, host film)."""
    L = load_library()
    rp = RenderParams()
    done = C.c_int()
    _check(L.xyzgpu_checkpoint_load(path.encode(), C.byref(rp), C.byref(done), None))
    film = np.zeros((rp.height, rp.width, 3), np.float32)
    _check(L.xyzgpu_checkpoint_load(path.encode(), C.byref(rp), C.byref(done), film.ctypes.data))
    return rp, done.value, film


def philox_u01(seed: int, pixel: int, sample: int, dim: int) -> float:
    return load_library().xyzgpu_philox_u01(seed, pixel, sample, dim)



def batch_config(**kw) -> BatchConfig:
    c = BatchConfig()
    load_library().xyzgpu_batch_config_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, int(v))
    return c


def _config_dict(c: BatchConfig) -> dict:
    return {f: getattr(c, f) for f, _ in BatchConfig._fields_}


class BatchJob:
    """One render of a batch: a scene, camera, image size, samples and a
    device film (allocated if not given)."""

    def __init__(self, scene: Scene, camera, width: int, height: int, spp: int, *, seed: int = 0,
                 spp_offset: int = 0, max_depth: int = 15, rr_start_depth: int = 1,
                 rr_threshold: float = 0.2, accumulate: bool = False, film=None):
        import torch
        self.scene, self.camera = scene, camera
        self.width, self.height, self.spp = width, height, spp
        self.kw = dict(seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                       rr_start_depth=rr_start_depth, rr_threshold=rr_threshold, accumulate=accumulate)
        if film is None:
            film = torch.zeros((height, width, 3), dtype=torch.float32, device="cuda")
        assert film.is_cuda and film.is_contiguous() and tuple(film.shape) == (height, width, 3)
        self.film = film

    def desc(self) -> BatchJobDesc:
        d = BatchJobDesc()
        d.scene = self.scene.handle.value
        d.camera = camera_desc(self.camera)
        d.params = render_params(self.width, self.height, self.spp, **self.kw)
        d.params.film_location = XYZGPU_FILM_DEVICE
        d.film = self.film.data_ptr()
        return d


class Batch:
    """xyzgpu_batch: many renders in every kernel launch, replayed from a CUDA
    graph.  launch() renders every job's samples into its film."""

    def __init__(self, jobs, **config):
        L = load_library()
        self.jobs = list(jobs)
        arr = (BatchJobDesc * len(self.jobs))(*[j.desc() for j in self.jobs])
        cfg = batch_config(**config)
        h = C.c_void_p()
        _check(L.xyzgpu_batch_create(arr, len(self.jobs), C.byref(cfg), C.byref(h)))
        self.handle = h

    def launch(self, stream=None):
        _check(_LIB.xyzgpu_batch_launch(self.handle, _stream_ptr(stream)))

    def set_sample_offsets(self, offsets):
        a = np.ascontiguousarray(offsets, dtype=np.uint32)
        assert a.shape == (len(self.jobs),)
        _check(_LIB.xyzgpu_batch_set_sample_offsets(self.handle, a.ctypes.data))

    def autotune(self, trials: int = 2, probe_spp: int = 4, stream=None) -> dict:
        c = BatchConfig()
        _check(_LIB.xyzgpu_batch_autotune(self.handle, trials, probe_spp, _stream_ptr(stream), C.byref(c)))
        return _config_dict(c)

    def config(self) -> dict:
        c = BatchConfig()
        _check(_LIB.xyzgpu_batch_config_get(self.handle, C.byref(c)))
        return _config_dict(c)

    def stats(self) -> dict:
        st = BatchStats()
        _check(_LIB.xyzgpu_batch_stats_get(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in BatchStats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            _LIB.xyzgpu_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def guide_config(**kw) -> GuideConfig:
    c = GuideConfig()
    load_library().xyzgpu_guide_config_default(C.byref(c))
    for k, v in kw.items():
        setattr(c, k, v)
    return c


class Guide:
    """xyzgpu_guide: the learned path guide of a scene (an MLP on the tensor
    cores from surface point to a von Mises-Fisher mixture)."""

    def __init__(self, scene: Scene, **config):
        L = load_library()
        cfg = guide_config(**config)
        h = C.c_void_p()
        _check(L.xyzgpu_guide_create(scene.handle, C.byref(cfg), C.byref(h)))
        self.handle = h
        self.scene = scene
        st = scene.stats()
        lo = np.array(st["bounds_min"], np.float32)
        hi = np.array(st["bounds_max"], np.float32)
        ext = (hi - lo).astype(np.float32)
        self.lo = lo
        self.inv_ext = np.where(ext > 0, np.float32(1.0) / np.where(ext > 0, ext, 1), 1).astype(np.float32)

    def params(self) -> np.ndarray:
        p = np.zeros(GUIDE_PARAMS, np.float32)
        _check(_LIB.xyzgpu_guide_get_params(self.handle, p.ctypes.data))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        assert p.shape == (GUIDE_PARAMS,)
        _check(_LIB.xyzgpu_guide_set_params(self.handle, p.ctypes.data))

    def forward(self, features, stream=None):
        """features: CUDA float32 (n, 6) -> outputs (n, 64)."""
        import torch
        n = int(features.shape[0])
        out = torch.empty((n, GUIDE_OUTPUTS), dtype=torch.float32, device=features.device)
        _check(_LIB.xyzgpu_guide_forward(self.handle, features.contiguous().data_ptr(), n, out.data_ptr(),
                                         _stream_ptr(stream)))
        return out

    def gradient(self, records, scale: float = 1.0, grad=None, stream=None):
        """records: CUDA float32 (n, 10) -> flat gradient (accumulated into grad)."""
        import torch
        n = int(records.shape[0])
        if grad is None:
            grad = torch.zeros(GUIDE_PARAMS, dtype=torch.float32, device=records.device)
        _check(_LIB.xyzgpu_guide_gradient(self.handle, records.contiguous().data_ptr(), n, float(scale),
                                          grad.data_ptr(), _stream_ptr(stream)))
        return grad

    def reserve(self, wave_paths: int, train: bool = True, stream=None):
        """xyzgpu_guide_reserve: allocate the guided-wave buffers (mixtures and,
        with train, training records) for waves of up to wave_paths paths now,
        so that no later render_guided call allocates."""
        _check(_LIB.xyzgpu_guide_reserve(self.handle, int(wave_paths), int(bool(train)), _stream_ptr(stream)))

    def train_step(self, records, stream=None):
        _check(_LIB.xyzgpu_guide_train_step(self.handle, records.contiguous().data_ptr(), int(records.shape[0]),
                                            _stream_ptr(stream)))

    def render(self, camera, width: int, height: int, spp: int, *, train: bool = False, seed: int = 0,
               spp_offset: int = 0, max_depth: int = 15, rr_start_depth: int = 1, rr_threshold: float = 0.2,
               film=None, accumulate: bool = False, wave_paths: int = 0, rows=None, profile: int = 0,
               stream=None):
        """xyzgpu_render_guided into a CUDA film (H, W, 3) of sums; train: learn
        from this render's paths (Adam steps after each wave); profile=1: per
        kernel class timing (Scene.render_profile, class "guide" = the network)."""
        import torch
        if film is None:
            film = torch.zeros((height, width, 3), dtype=torch.float32, device="cuda")
        cam = camera_desc(camera)
        rp = render_params(width, height, spp, seed=seed, spp_offset=spp_offset, max_depth=max_depth,
                           rr_start_depth=rr_start_depth, rr_threshold=rr_threshold, accumulate=accumulate,
                           wave_paths=wave_paths, rows=rows)
        rp.profile = profile
        rp.film_location = XYZGPU_FILM_DEVICE
        _check(_LIB.xyzgpu_render_guided(self.handle, C.byref(cam), C.byref(rp), int(bool(train)),
                                         film.data_ptr(), _stream_ptr(stream)))
        return film

    def stats(self) -> dict:
        st = GuideStats()
        _check(_LIB.xyzgpu_guide_stats_get(self.handle, C.byref(st)))
        return {f: getattr(st, f) for f, _ in GuideStats._fields_}

    def close(self):
        if getattr(self, "handle", None):
            _LIB.xyzgpu_guide_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
