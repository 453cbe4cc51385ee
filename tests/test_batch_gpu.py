"""Batched rendering (xyzgpu_batch_*): every job's film equals a single-scene
xyzgpu_render of the same scene and parameters, bit for bit, whatever the
wave size, pixel tile, trace grid or graph replay; progressive sample offsets;
the autotuner; argument checks."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _workload(n=6):
    from xyz_b200 import scenes
    entries = []
    sizes = [(64, 48, 3), (128, 128, 2), (32, 32, 5), (96, 64, 1), (128, 96, 4), (16, 16, 7)]
    for k in range(n):
        sd = scenes.batch_scene(k, target_tris=[1500, 4000, 12000, 2500, 30000, 1000][k % 6])
        w, h, spp = sizes[k % len(sizes)]
        entries.append((sd, w, h, spp))
    return entries


def _singles(scenes_, entries, seeds, depth=8):
    out = []
    for s, (sd, w, h, spp), seed in zip(scenes_, entries, seeds):
        f = s.render(sd.camera, w, h, spp, seed=seed, max_depth=depth)
        out.append(f.clone())
    return out


@pytest.mark.parametrize("cfg", [dict(), dict(tile=8), dict(wave_paths=40000),
                                  dict(wave_paths=20000, tile=4, trace_ctas_per_sm=3),
                                  dict(use_graph=0, tile=16)])
def test_batch_films_equal_single_renders(cfg):
    import torch
    from xyz_b200 import api
    entries = _workload()
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    seeds = [11 * k + 1 for k in range(len(entries))]
    try:
        ref = _singles(scenes_, entries, seeds)
        jobs = [api.BatchJob(s, sd.camera, w, h, spp, seed=seed, max_depth=8)
                for s, (sd, w, h, spp), seed in zip(scenes_, entries, seeds)]
        with api.Batch(jobs, **cfg) as b:
            b.launch()
            torch.cuda.synchronize()
            st = b.stats()
            assert st["paths"] == sum(w * h * spp for _, w, h, spp in entries)
            if cfg.get("wave_paths") == 20000:
                assert st["waves"] > 3
            if cfg.get("use_graph", 1):
                # one start kernel and the wave loop at the top; the loops'
                # bodies hold the same dozen nodes however many waves there are
                assert st["graph_top_nodes"] == 2
                assert st["graph_nodes"] == 12
            for j, r in zip(jobs, ref):
                assert torch.equal(j.film.view(torch.int32), r.view(torch.int32))
            # a second replay gives the same films
            b.launch()
            torch.cuda.synchronize()
            for j, r in zip(jobs, ref):
                assert torch.equal(j.film.view(torch.int32), r.view(torch.int32))
    finally:
        for s in scenes_:
            s.close()


def test_batch_progressive_offsets_accumulate():
    import torch
    from xyz_b200 import api
    entries = _workload(3)
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    try:
        ref = []
        for s, (sd, w, h, spp) in zip(scenes_, entries):
            ref.append(s.render(sd.camera, w, h, 2 * spp, seed=5, max_depth=8).clone())
        jobs = [api.BatchJob(s, sd.camera, w, h, spp, seed=5, max_depth=8, accumulate=True)
                for s, (sd, w, h, spp) in zip(scenes_, entries)]
        with api.Batch(jobs) as b:
            b.launch()
            b.set_sample_offsets([spp for _, _, _, spp in entries])
            b.launch()
            torch.cuda.synchronize()
            for j, r in zip(jobs, ref):
                assert torch.equal(j.film.view(torch.int32), r.view(torch.int32))
    finally:
        for s in scenes_:
            s.close()


def test_autotune_picks_a_configuration_and_keeps_films_exact():
    import torch
    from xyz_b200 import api
    entries = _workload()
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    try:
        ref = _singles(scenes_, entries, [3] * len(entries))
        jobs = [api.BatchJob(s, sd.camera, w, h, spp, seed=3, max_depth=8)
                for s, (sd, w, h, spp) in zip(scenes_, entries)]
        marker = [j.film.fill_(7.0) for j in jobs]
        with api.Batch(jobs) as b:
            chosen = b.autotune(trials=1, probe_spp=2)
            torch.cuda.synchronize()
            # the search renders into scratch films
            assert all(bool((m == 7.0).all()) for m in marker)
            assert chosen == b.config()
            assert chosen["tile"] in (1, 4, 8, 16) and chosen["wave_paths"] > 0
            b.launch()
            torch.cuda.synchronize()
            for j, r in zip(jobs, ref):
                assert torch.equal(j.film.view(torch.int32), r.view(torch.int32))
    finally:
        for s in scenes_:
            s.close()


def test_batch_argument_checks():
    import torch
    from xyz_b200 import api
    entries = _workload(2)
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    try:
        jobs = [api.BatchJob(s, sd.camera, w, h, spp) for s, (sd, w, h, spp) in zip(scenes_, entries)]
        with pytest.raises(api.XyzGpuError) as e:
            api.Batch(jobs, wave_paths=1000)  # smaller than the largest image
        assert e.value.code == -4
        d = jobs[0].desc()
        d.params.spectral = 1
        arr = (api.BatchJobDesc * 1)(d)
        h = api.C.c_void_p()
        assert api.load_library().xyzgpu_batch_create(arr, 1, None, api.C.byref(h)) == -1
        assert api.load_library().xyzgpu_batch_create(arr, 0, None, api.C.byref(h)) == -1
    finally:
        for s in scenes_:
            s.close()


def test_batch_films_match_the_oracle_on_the_same_streams():
    """Each job of a batch against the CPU oracle (the restatement pinned to
    the reference's renderer) directly, not only through single renders."""
    import torch
    from tests.helpers import ensure_port
    from xyz_b200 import api, scenes
    entries = [(scenes.cornell_box(pinhole=True), 48, 36, 4, 3), (scenes.batch_scene(1, target_tris=4000), 40, 32, 3, 8),
               (scenes.spheres_scene(level=2, n_spheres=2, seed=4), 32, 24, 5, 21)]
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    try:
        jobs = [api.BatchJob(s, sd.camera, w, h, spp, seed=seed, max_depth=8)
                for s, (sd, w, h, spp, seed) in zip(scenes_, entries)]
        with api.Batch(jobs) as b:
            b.launch()
            torch.cuda.synchronize()
            films = [j.film.cpu().numpy() for j in jobs]
    finally:
        for s in scenes_:
            s.close()
    P = ensure_port()
    P.set_spectral(0, 1)
    for (sd, w, h, spp, seed), film in zip(entries, films):
        P.scene_create(sd)
        P.set_camera(sd.camera, w, h)
        P.set_path_params(max_depth=8)
        ref = P.render(spp, seed=seed, nthreads=0)
        close = (np.abs(film - ref) <= 1e-6 + 1e-4 * np.abs(ref)).all(axis=-1).mean()
        assert close >= 0.98, close
        assert abs(film.sum() - ref.sum()) / ref.sum() < 1e-2


@pytest.mark.parametrize("use_graph", [1, 0])
def test_batch_mixed_depths_and_early_ending_waves(use_graph):
    """Jobs of different max_depth share waves (a wave runs the bounces of its
    deepest job), and a job whose camera looks away from its scene ends after
    its first bounce: the device's bounce loop stops there in a graph launch,
    while the host-issued launch runs every bounce; films equal single renders."""
    import dataclasses
    import torch
    from xyz_b200 import api
    entries = _workload()
    depths = [1, 3, 8, 2, 5, 8]
    sd0, w0, h0, spp0 = entries[0]
    cam = sd0.camera
    # up and away from the floor (y = 0, |x|, |z| <= 10), the objects and the
    # light near the origin: every camera ray escapes
    away = dataclasses.replace(cam, at=(cam.eye[0], cam.eye[1] + 1.0, cam.eye[2] + 1.0))
    scenes_ = [api.Scene(sd) for sd, *_ in entries]
    try:
        ref = []
        for s, (sd, w, h, spp), d in zip(scenes_, entries, depths):
            ref.append(s.render(sd.camera, w, h, spp, seed=9, max_depth=d).clone())
        ref_away = scenes_[0].render(away, w0, h0, spp0, seed=9, max_depth=8).clone()
        jobs = [api.BatchJob(s, sd.camera, w, h, spp, seed=9, max_depth=d)
                for s, (sd, w, h, spp), d in zip(scenes_, entries, depths)]
        with api.Batch(jobs, wave_paths=30000, use_graph=use_graph) as b:
            b.launch()
            torch.cuda.synchronize()
            st = b.stats()
            assert st["waves"] > 2
            for j, r in zip(jobs, ref):
                assert torch.equal(j.film.view(torch.int32), r.view(torch.int32))
        lone = api.BatchJob(scenes_[0], away, w0, h0, spp0, seed=9, max_depth=8)
        with api.Batch([lone], use_graph=use_graph) as b:
            b.launch()
            torch.cuda.synchronize()
            st = b.stats()
            assert torch.equal(lone.film.view(torch.int32), ref_away.view(torch.int32))
            assert st["extension_rays"] == w0 * h0 * spp0
            # start kernel + 5 per wave + 4 per bounce run
            assert st["kernel_launches_per_launch"] == (1 + 5 + 4 if use_graph else 1 + 5 + 4 * 8)
    finally:
        for s in scenes_:
            s.close()
