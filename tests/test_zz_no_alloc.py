"""xyzgpu_render_noalloc: rendering for callers that cannot allocate device
memory while they run (an application that gives all GPU memory to its own
pool at start-up, a real-time loop that may not call the allocator mid-frame).
Its path state lives in a fixed file-scope device array; the image must be the
one xyzgpu_render produces.  This file is collected last on purpose."""

import pytest

pytestmark = pytest.mark.gpu


def _render_pair(s, c):
    import torch
    ref = s.render(c["cam"], c["W"], c["H"], c["spp"], seed=c["seed"], max_depth=c["depth"])
    film = torch.full((c["H"], c["W"], 3), float("nan"), device="cuda")
    s.render_noalloc(c["cam"], c["W"], c["H"], c["spp"], film, seed=c["seed"],
                     max_depth=c["depth"], wave_paths=c.get("wave_paths", 0))
    torch.cuda.synchronize()
    return film, ref


def test_noalloc_render_equals_render_on_two_calls_in_a_row():
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box(pinhole=True)
    thin = scenes.cornell_box(pinhole=False).camera
    # the second call is smaller and shallower, so stale queue lengths or
    # radiance left in the shared array by the first call would show up
    cases = [dict(cam=sd.camera, W=96, H=64, spp=5, seed=3, depth=12),
             dict(cam=thin, W=40, H=30, spp=2, seed=9, depth=6)]
    with api.Scene(sd) as s:
        for c in cases:
            film, ref = _render_pair(s, c)
            # per-path results do not depend on the wave size: identical films
            assert torch.equal(film, ref)


def test_noalloc_render_splits_pixels_and_samples_over_waves():
    """Calls larger than one wave of the fixed array: the image is cut into
    runs of pixels (more pixels than a wave holds), into runs of samples (few
    pixels, many samples), or both (a small explicit wave size); every film
    equals xyzgpu_render's, and a second call in a row still does."""
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box(pinhole=True)
    cases = [dict(cam=sd.camera, W=320, H=240, spp=1, seed=5, depth=8),     # 76,800 pixels: 2 pixel runs
             dict(cam=sd.camera, W=64, H=64, spp=40, seed=6, depth=8),      # 16 + 16 + 8 samples
             dict(cam=sd.camera, W=64, H=48, spp=6, seed=7, depth=8, wave_paths=1000),  # 4 x 6 waves
             dict(cam=sd.camera, W=64, H=48, spp=6, seed=7, depth=8, wave_paths=1000)]
    with api.Scene(sd) as s:
        for c in cases:
            film, ref = _render_pair(s, c)
            assert torch.equal(film, ref), c


def test_noalloc_render_takes_mirror_scenes():
    """Mirror materials (no per-path shadow-record extras) render as
    xyzgpu_render does; metal scenes are refused (test_materials_gpu)."""
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_specular()
    kinds = sd.material_kind.copy()
    kinds[kinds == api.MATERIAL_METAL] = api.MATERIAL_LAMBERT
    sd.material_kind = kinds
    assert (kinds == api.MATERIAL_MIRROR).any()
    with api.Scene(sd) as s:
        for c in (dict(cam=sd.camera, W=64, H=48, spp=4, seed=2, depth=9),
                  dict(cam=sd.camera, W=32, H=24, spp=3, seed=4, depth=5, wave_paths=700)):
            film, ref = _render_pair(s, c)
            assert torch.equal(film, ref), c


def test_noalloc_render_rejects_sizes_beyond_its_limits():
    import numpy as np
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    film = torch.zeros((8, 8, 3), device="cuda")
    with api.Scene(sd) as s:
        with pytest.raises(api.XyzGpuError) as e:
            s.render_noalloc(sd.camera, 8, 8, 1, film, max_depth=65)
        assert e.value.code == -4 and "max_depth" in str(e.value)
        with pytest.raises(api.XyzGpuError) as e:
            s.render_noalloc(sd.camera, 8, 8, 1, film, wave_paths=65537)
        assert e.value.code == -4 and "wave_paths" in str(e.value)
        # a host film would need a device staging buffer
        L = api.load_library()
        cam = api.CameraDesc()
        for k in range(3):
            cam.eye[k], cam.at[k] = sd.camera.eye[k], sd.camera.at[k]
        cam.film_size, cam.focal_length, cam.f_number, cam.pinhole = (
            sd.camera.film_size, sd.camera.focal_length, sd.camera.f_number, 1)
        rp = api.RenderParams()
        L.xyzgpu_render_params_default(api.C.byref(rp))
        rp.width = rp.height = 8
        rp.film_location = api.XYZGPU_FILM_HOST
        host = np.zeros((8, 8, 3), np.float32)
        assert L.xyzgpu_render_noalloc(s.handle, api.C.byref(cam), api.C.byref(rp),
                                       host.ctypes.data, None) == -1
