"""The FP64 CPU reference of the path-guiding benchmark (no GPU): the
oracle's per-pixel double sums equal its film render, and the committed
fixture (tests/golden/guide_reference_fp64.npz) still describes the scene the
generator makes."""

import os

import numpy as np

from tests.helpers import ROOT, ensure_port
from tests.test_guide_reference_gpu import FIXTURE, _digest


def test_pixel_sums_equal_the_film_render():
    from xyz_b200 import scenes
    sd = scenes.cornell_box()
    P = ensure_port()
    P.set_spectral(0, 1)
    P.scene_create(sd)
    P.set_camera(sd.camera, 32, 24)
    P.set_path_params(max_depth=8)
    film = P.render(16, seed=4, nthreads=0).astype(np.float64)
    rng = np.random.default_rng(0)
    px, py = rng.integers(0, 32, 50), rng.integers(0, 24, 50)
    acc = P.render_pixels(px, py, 10, seed=4)
    P.render_pixels(px, py, 6, seed=4, s0=10, acc=acc)
    np.testing.assert_allclose(acc[:, :3], film[py, px], rtol=1e-5, atol=1e-9)
    ys = np.stack([P.render(1, seed=4, s0=k, nthreads=0)[py, px, 1].astype(np.float64) for k in range(16)])
    np.testing.assert_allclose(acc[:, 3], (ys ** 2).sum(axis=0), rtol=1e-6, atol=1e-12)


def test_fixture_matches_the_scene_generator():
    from xyz_b200 import scenes
    fx = np.load(FIXTURE)
    assert os.path.exists(os.path.join(ROOT, "tests", "golden", "make_guide_reference.py"))
    assert _digest(scenes.occluded_room()) == str(fx["scene_sha256"])
    assert fx["acc"].shape == (1024, 4) and int(fx["spp"]) == 65536
    assert set(np.unique(fx["py"])) == set(range(16, 1024, 32))
    assert (fx["acc"][:, 1] > 0).all()
