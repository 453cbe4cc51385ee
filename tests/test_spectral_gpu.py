"""Spectral film modes of the CUDA path tracer against the C restatement of the
reference's spectral estimator on the same random streams."""

import numpy as np
import pytest

from tests.helpers import ensure_port

pytestmark = pytest.mark.gpu


def _close_fraction(a, b, rtol=1e-4, atol=1e-6):
    return (np.abs(a - b) <= atol + rtol * np.abs(b)).all(axis=-1).mean()


@pytest.mark.parametrize("mode,hero", [("binned", 1), ("binned", 4), ("continuous", 4), ("continuous", 1)])
@pytest.mark.parametrize("pinhole", [True, False])
def test_spectral_film_matches_oracle_on_same_streams(mode, hero, pinhole):
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box(pinhole=pinhole)
    W, H, spp, seed, depth = 48, 36, 4, 17, 7
    P = ensure_port()
    P.scene_create(sd)
    P.set_spectra(sd.albedo_spd, sd.light_power_spd)
    P.set_spectral({"binned": 1, "continuous": 2}[mode], hero)
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=depth)
    ref = P.render(spp, seed=seed, nthreads=0)
    P.set_spectral(0, 1)
    with api.Scene(sd) as s:
        film = s.render(sd.camera, W, H, spp, seed=seed, max_depth=depth, spectral=mode,
                        hero_wavelengths=hero).cpu().numpy()
    assert _close_fraction(film, ref) >= 0.98
    assert abs(film.sum() - ref.sum()) / ref.sum() < 1e-2


def test_spectral_needs_spectra_and_valid_hero_count():
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    with api.Scene(sd) as s:
        with pytest.raises(api.XyzGpuError):
            s.render(sd.camera, 8, 8, 1, spectral="binned", hero_wavelengths=5)
    sd.albedo_spd = None
    with api.Scene(sd) as s:
        with pytest.raises(api.XyzGpuError) as e:
            s.render(sd.camera, 8, 8, 1, spectral="binned")
        assert "spectra" in str(e.value)


def test_spectral_wave_size_invariance_and_large_mesh():
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.spheres_scene(level=4, n_spheres=3)
    with api.Scene(sd) as s:
        a = s.render(sd.camera, 64, 48, 4, seed=2, max_depth=10, spectral="continuous")
        b = s.render(sd.camera, 64, 48, 4, seed=2, max_depth=10, spectral="continuous", wave_paths=3000)
        torch.cuda.synchronize()
        assert torch.equal(a, b)
        assert float(a.sum()) > 0
