"""Guided rendering (xyzgpu_render_guided): the estimator stays unbiased with
an untrained and with a trained guide (statistical agreement with the plain
tracer), training runs during the render, the trained guide lowers the error
at equal samples on the indirect-lit room, argument checks; and row bands of
a plain render."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _block_stats(passes, b=8):
    """Per-block mean of Y over passes and its standard error."""
    a = np.stack([p[..., 1] for p in passes]).astype(np.float64)   # (K, H, W)
    k, h, w = a.shape
    blocks = a.reshape(k, h // b, b, w // b, b).mean(axis=(2, 4))
    return blocks.mean(axis=0), blocks.std(axis=0, ddof=1) / np.sqrt(k)


@pytest.mark.parametrize("trained", [False, True])
def test_guided_estimate_agrees_with_plain(trained):
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    W = H = 64
    spp, K = 32, 16
    with api.Scene(sd) as s:
        g = api.Guide(s, seed=3)
        try:
            if trained:
                for p in range(8):
                    g.render(sd.camera, W, H, 8, seed=11, spp_offset=8 * p, max_depth=8, train=True)
                assert g.stats()["adam_steps"] > 0
            else:
                # an arbitrary (untrained, perturbed) network: the estimate must not depend on it
                rng = np.random.default_rng(1)
                g.set_params(g.params() + rng.normal(0, 0.3, 28992).astype(np.float32))
            plain = [s.render(sd.camera, W, H, spp, seed=5, spp_offset=spp * k, max_depth=8).cpu().numpy() / spp
                     for k in range(K)]
            guided = [g.render(sd.camera, W, H, spp, seed=7, spp_offset=spp * k, max_depth=8).cpu().numpy() / spp
                      for k in range(K)]
        finally:
            g.close()
    mp, sp = _block_stats(plain)
    mg, sg = _block_stats(guided)
    z = np.abs(mp - mg) / np.sqrt(sp ** 2 + sg ** 2 + 1e-30)
    assert z.max() < 5.0, z.max()
    assert abs(mg.mean() / mp.mean() - 1.0) < 0.02


def test_training_lowers_error_at_equal_samples_on_the_indirect_room():
    """The room lit only through a 0.1 m gap: after training on the first
    passes, the guided tracer's relative MSE at 256 spp is well below the
    plain tracer's at 256 spp (both against a 4096-spp plain reference)."""
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.occluded_room()
    cam = scenes.Camera.with_fov((0.0, 1.5, 1.2), (0.0, 1.1, -2.0), 60.0, pinhole=True)
    W = H = 128
    with api.Scene(sd) as s:
        ref = torch.zeros((H, W, 3), dtype=torch.float64, device="cuda")
        for k in range(0, 4096, 512):
            ref += s.render(cam, W, H, 512, seed=99, spp_offset=k, max_depth=10).double()
        ref /= 4096
        scale = 1.0 / float(ref[..., 1].mean())
        ry = ref[..., 1] * scale

        def relmse(img):
            return float((((img[..., 1] * scale - ry) ** 2) / (ry ** 2 + 1e-2)).mean())

        plain = relmse(s.render(cam, W, H, 256, seed=1, max_depth=10).double() / 256)
        g = api.Guide(s, train_bounces=3)
        try:
            for p in range(24):
                g.render(cam, W, H, 4, seed=2, spp_offset=4 * p, max_depth=10, train=True)
            st = g.stats()
            guided = relmse(g.render(cam, W, H, 256, seed=3, max_depth=10).double() / 256)
        finally:
            g.close()
    assert st["adam_steps"] == 24 * 16 and st["trained_records"] > 10000
    assert guided * 2.0 < plain, (plain, guided)


def test_guided_render_argument_checks():
    import ctypes as C
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    with api.Scene(sd) as s:
        g = api.Guide(s)
        try:
            film = torch.zeros((8, 8, 3), device="cuda")
            cam = api.camera_desc(sd.camera)
            for field, value in (("spectral", 1), ("profile", 2), ("row_end", 9)):
                rp = api.render_params(8, 8, 1)
                setattr(rp, field, value)
                rc = api.load_library().xyzgpu_render_guided(g.handle, C.byref(cam), C.byref(rp), 0,
                                                             film.data_ptr(), None)
                assert rc == -1, field
        finally:
            g.close()


def test_row_band_renders_the_same_pixels():
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    W, H = 48, 40
    with api.Scene(sd) as s:
        full = s.render(sd.camera, W, H, 3, seed=4, max_depth=8)
        band = s.render(sd.camera, W, H, 3, seed=4, max_depth=8, rows=(13, 29))
    assert torch.equal(band[13:29].view(torch.int32), full[13:29].view(torch.int32))
    assert float(band[:13].abs().sum()) == 0.0 and float(band[29:].abs().sum()) == 0.0


def test_plain_tracer_matches_the_oracle_on_the_occluded_room():
    """The guided benchmark's reference image is the plain GPU tracer at high
    spp; on the same scene, camera and estimator settings its image agrees
    with the CPU oracle (the reference's path tracer restated in C, equal to
    the reference build bit for bit) over independent passes."""
    from tests.helpers import ensure_port
    from xyz_b200 import scenes
    sd = scenes.occluded_room()
    cam = scenes.Camera.with_fov((0.0, 1.5, 1.2), (0.0, 1.1, -2.0), 60.0, pinhole=True)
    W = H = 128
    y0, y1 = 56, 72
    spp, K = 32, 16
    P = ensure_port()
    P.scene_create(sd)
    P.set_camera(cam, W, H)
    P.set_path_params(max_depth=10)
    cpu = [P.render(spp, seed=77, s0=spp * k, y0=y0, y1=y1, nthreads=0)[y0:y1] / spp for k in range(K)]
    from xyz_b200 import api
    with api.Scene(sd) as s:
        gpu = [s.render(cam, W, H, spp, seed=5, spp_offset=spp * k, max_depth=10, rows=(y0, y1))
               .cpu().numpy()[y0:y1] / spp for k in range(K)]
    mc, sc = _block_stats(cpu)
    mg, sg = _block_stats(gpu)
    z = np.abs(mc - mg) / np.sqrt(sc ** 2 + sg ** 2 + 1e-30)
    assert z.max() < 5.0, z.max()
    assert abs(mg.mean() / mc.mean() - 1.0) < 0.03
