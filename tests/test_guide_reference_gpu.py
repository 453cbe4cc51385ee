"""The path-guiding benchmark's reference image against the FP64 CPU oracle:
tests/golden/guide_reference_fp64.npz holds 65,536-sample per-pixel sums (in
double) of the CPU restatement of the reference's estimator on a 32 x 32 pixel
grid of the occluded room (made by tests/golden/make_guide_reference.py).  The
GPU tracer, on independent random streams, must agree with it per pixel within
3 sigma of the two estimates' combined noise."""

import hashlib
import os

import numpy as np
import pytest

from tests.helpers import ROOT

pytestmark = pytest.mark.gpu

FIXTURE = os.path.join(ROOT, "tests", "golden", "guide_reference_fp64.npz")


def _digest(sd):
    h = hashlib.sha256()
    for a in (sd.positions, sd.tris, sd.tri_mat, sd.albedo_xyz, sd.is_light, sd.light_power_xyz):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def test_gpu_render_agrees_with_the_fp64_cpu_oracle_per_pixel():
    import torch
    from xyz_b200 import api, scenes
    fx = np.load(FIXTURE)
    sd = scenes.occluded_room()
    assert _digest(sd) == str(fx["scene_sha256"]), "the occluded-room generator changed"
    W, H, depth, n_cpu = int(fx["width"]), int(fx["height"]), int(fx["max_depth"]), int(fx["spp"])
    c = fx["camera"]
    cam = scenes.Camera.with_fov(tuple(c[:3]), tuple(c[3:6]), float(c[6]), pinhole=True)
    px, py = fx["px"], fx["py"]
    rows = (16, H, 32)                                   # the fixture's pixel rows
    row_of = {y: i for i, y in enumerate(range(*rows))}
    spp, chunk = 16384, 4096
    acc = torch.zeros((len(row_of), W, 3), dtype=torch.float64, device="cuda")
    with api.Scene(sd) as s:
        for k in range(0, spp, chunk):
            f = s.render(cam, W, H, chunk, seed=31, spp_offset=k, max_depth=depth, rows=rows)
            acc += f[list(row_of)].double()
    g = acc.cpu().numpy()[[row_of[int(y)] for y in py], px] / spp
    cpu = fx["acc"]
    mean_c = cpu[:, 1] / n_cpu
    var_sample = np.maximum(cpu[:, 3] / n_cpu - mean_c ** 2, 0.0)
    z = (g[:, 1] - mean_c) / np.sqrt(var_sample * (1.0 / spp + 1.0 / n_cpu) + 1e-30)
    assert (np.abs(z) > 3).mean() < 0.02, np.sort(np.abs(z))[-10:]
    assert abs(g[:, 1].mean() / mean_c.mean() - 1.0) < 0.015
    # X and Z follow Y's light: the channels' ratios agree as well
    assert abs(g[:, 0].sum() / (cpu[:, 0].sum() / n_cpu) - 1.0) < 0.015
    assert abs(g[:, 2].sum() / (cpu[:, 2].sum() / n_cpu) - 1.0) < 0.015


def _passes_vs_oracle(render_pass, K, spp):
    """Per-pixel z of the mean of K independent passes (spp samples each, on
    the fixture's rows) against the FP64 CPU oracle, with each estimate's
    variance of the mean: the passes' sample variance / K, the oracle's
    per-sample variance / its sample count."""
    import torch
    fx = np.load(FIXTURE)
    px, py = fx["px"], fx["py"]
    ri = (py - 16) // 32
    n_cpu = int(fx["spp"])
    ys = []
    for k in range(K):
        f = render_pass(k)
        ys.append(f[16::32][ri, px, 1].double().cpu().numpy() / spp)
        torch.cuda.synchronize()
    ys = np.stack(ys)
    mg, vg = ys.mean(axis=0), ys.var(axis=0, ddof=1) / K
    mc = fx["acc"][:, 1] / n_cpu
    vc = np.maximum(fx["acc"][:, 3] / n_cpu - mc ** 2, 0.0) / n_cpu
    z = (mg - mc) / np.sqrt(vg + vc + 1e-30)
    return z, mg, mc


def _guide_scene():
    from xyz_b200 import scenes
    fx = np.load(FIXTURE)
    c = fx["camera"]
    cam = scenes.Camera.with_fov(tuple(c[:3]), tuple(c[3:6]), float(c[6]), pinhole=True)
    return scenes.occluded_room(), cam, int(fx["width"]), int(fx["height"]), int(fx["max_depth"])


def test_trained_guide_agrees_with_the_fp64_cpu_oracle_per_pixel():
    """The learned guide (trained online on these rows, as in the benchmark)
    leaves the estimate unbiased: per pixel within 3 sigma of the oracle."""
    from xyz_b200 import api
    sd, cam, W, H, depth = _guide_scene()
    rows = (16, H, 32)
    K, spp = 32, 128
    with api.Scene(sd) as s, api.Guide(s, train_bounces=5, guide_bounces=9, alpha=0.5, steps_per_pass=512,
                                       batch_size=16384) as g:
        for p in range(8):
            g.render(cam, W, H, 64, seed=41, spp_offset=64 * p, max_depth=depth, rows=rows, train=True)
        assert g.stats()["adam_steps"] > 0
        z, mg, mc = _passes_vs_oracle(
            lambda k: g.render(cam, W, H, spp, seed=43, spp_offset=spp * k, max_depth=depth, rows=rows), K, spp)
    assert (np.abs(z) > 3).mean() < 0.025, np.sort(np.abs(z))[-8:]
    assert abs(mg.mean() / mc.mean() - 1.0) < 0.02


def test_importance_driven_tracer_agrees_with_the_fp64_cpu_oracle_per_pixel():
    from xyz_b200 import api
    sd, cam, W, H, depth = _guide_scene()
    rows = (16, H, 32)
    K, spp = 32, 128
    with api.Scene(sd) as s, api.Importons(s, particles=100000, seed=5) as m:
        z, mg, mc = _passes_vs_oracle(
            lambda k: m.render(cam, W, H, spp, seed=47, spp_offset=spp * k, max_depth=depth, rows=rows), K, spp)
    assert (np.abs(z) > 3).mean() < 0.025, np.sort(np.abs(z))[-8:]
    assert abs(mg.mean() / mc.mean() - 1.0) < 0.02
