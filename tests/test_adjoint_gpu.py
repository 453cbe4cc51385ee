"""Path-replay adjoint (xyzgpu_adjoint) on the GPU: against the oracle's
per-contribution gradient on the same sample paths (replaying recorded
intersections and re-tracing), against central finite
differences (h = 1e-3) of the GPU's own renders on 256 random parameters of the
differentiable room scene, through the torch.autograd.Function harness, and its
argument checks."""

import numpy as np
import pytest

from tests.helpers import ensure_port

pytestmark = pytest.mark.gpu


# the replay over intersections recorded by the primal pass (the default) and
# the replay that traces its paths again (XYZGPU_ADJOINT_TRACE_REPLAY)
REPLAYS = ["recorded", "traced"]


def _replay_mode(monkeypatch, replay):
    if replay == "traced":
        monkeypatch.setenv("XYZGPU_ADJOINT_TRACE_REPLAY", "1")
    else:
        monkeypatch.delenv("XYZGPU_ADJOINT_TRACE_REPLAY", raising=False)


@pytest.mark.parametrize("replay", REPLAYS)
def test_adjoint_matches_oracle_gradient_on_same_paths(monkeypatch, replay):
    _replay_mode(monkeypatch, replay)
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box(pinhole=True)
    W, H, spp, seed, depth = 48, 40, 4, 7, 6
    nm = len(sd.is_light)
    rng = np.random.default_rng(2)
    dfilm = rng.standard_normal((H, W, 3)).astype(np.float32)
    em = np.full(nm, 1.25, np.float32)
    P = ensure_port()
    P.scene_create(sd)
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=depth, rr_threshold=0.0)
    P.set_materials(None, em)
    ga_ref, ge_ref = P.adjoint(dfilm, spp, seed, nm)
    P.set_materials(None, np.ones(nm, np.float32))
    with api.Scene(sd) as s:
        s.set_materials(None, em)
        ga, ge = s.adjoint(sd.camera, W, H, spp, torch.from_numpy(dfilm).cuda(), seed=seed,
                           max_depth=depth, rr_threshold=0.0)
        ga, ge = ga.cpu().numpy().astype(np.float64), ge.cpu().numpy().astype(np.float64)
    scale = np.abs(ga_ref).max()
    assert np.abs(ga - ga_ref).max() <= 2e-3 * scale, (ga, ga_ref)
    np.testing.assert_allclose(ge, ge_ref, rtol=2e-3, atol=2e-3 * np.abs(ge_ref).max())


@pytest.mark.parametrize("replay", REPLAYS)
def test_adjoint_matches_oracle_with_russian_roulette_held(monkeypatch, replay):
    """With Russian roulette on, both hold the roulette's survival scale
    constant: the same gradient on the same paths."""
    _replay_mode(monkeypatch, replay)
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box(pinhole=True)
    W, H, spp, seed, depth = 40, 32, 4, 11, 8
    nm = len(sd.is_light)
    dfilm = np.ones((H, W, 3), np.float32)
    P = ensure_port()
    P.scene_create(sd)
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=depth, rr_threshold=0.2, rr_start=3)
    ga_ref, ge_ref = P.adjoint(dfilm, spp, seed, nm)
    with api.Scene(sd) as s:
        ga, ge = s.adjoint(sd.camera, W, H, spp, torch.from_numpy(dfilm).cuda(), seed=seed,
                           max_depth=depth, rr_threshold=0.2, rr_start_depth=3)
        ga, ge = ga.cpu().numpy().astype(np.float64), ge.cpu().numpy().astype(np.float64)
    assert np.abs(ga - ga_ref).max() <= 2e-3 * np.abs(ga_ref).max()
    np.testing.assert_allclose(ge, ge_ref, rtol=2e-3)


def _diff_setup():
    from xyz_b200 import api, scenes
    ds = scenes.diff_scene()
    s = api.Scene(ds.scene)
    s.set_materials(ds.albedo, ds.emission)
    return ds, s


def test_adjoint_matches_central_differences_on_256_parameters():
    """Differentiable room (19,392 triangles, one material each): L2 loss to a
    target rendered from perturbed parameters; adjoint gradient on the primal's
    own samples vs central differences h = 1e-3 of the same renders, on 256
    random parameters (albedo channels and light emissions)."""
    W, H, spp, depth = 96, 96, 4, 6
    ds, s = _diff_setup()
    cam = ds.scene.camera
    kw = dict(seed=0, max_depth=depth, rr_threshold=0.0)
    try:
        s.set_materials(ds.target_albedo, ds.target_emission)
        target = (s.render(cam, W, H, spp, **kw) / spp).double()
        alb, em = ds.albedo.copy(), ds.emission.copy()

        def loss(a, e):
            s.set_materials(a, e)
            img = (s.render(cam, W, H, spp, **kw) / spp).double()
            return float(((img - target) ** 2).sum()), img

        l0, img0 = loss(alb, em)
        d_film = (2.0 * (img0 - target) / spp).float().contiguous()
        s.set_materials(alb, em)
        ga, ge = s.adjoint(cam, W, H, spp, d_film, **kw)
        ga, ge = ga.cpu().numpy().astype(np.float64), ge.cpu().numpy().astype(np.float64)

        # 256 parameters: all 32 light emissions and 224 albedo channels of
        # triangles that the camera sees (nonzero gradient), seeded choice
        rng = np.random.default_rng(1)
        seen = np.flatnonzero(np.abs(ga).sum(axis=1) > 0)
        mats = rng.choice(seen, size=224 // 3 + 1, replace=False)
        params = [("e", int(m), 0) for m in ds.light_materials]
        params += [("a", int(m), c) for m in mats for c in range(3)][: 256 - len(params)]
        assert len(params) == 256
        h = 1e-3
        fds, ads = [], []
        for kind, m, c in params:
            if kind == "a":
                a1, a2 = alb.copy(), alb.copy()
                a1[m, c] += h
                a2[m, c] -= h
                lp, _ = loss(a1, em)
                lm, _ = loss(a2, em)
                adj = ga[m, c]
            else:
                e1, e2 = em.copy(), em.copy()
                e1[m] += h
                e2[m] -= h
                lp, _ = loss(alb, e1)
                lm, _ = loss(alb, e2)
                adj = ge[m]
            fd = (lp - lm) / (2 * h)
            fds.append(fd)
            ads.append(adj)
        fds, ads = np.array(fds), np.array(ads)
        rel = np.abs(ads - fds) / np.maximum(np.abs(fds), 1e-12)
        big = np.abs(fds) >= 1e-3 * np.abs(fds).max()
        # the aggregate over the 256 parameters, and each non-negligible one
        assert np.linalg.norm(ads - fds) <= 1e-2 * np.linalg.norm(fds)
        assert (rel[big] <= 1e-2).mean() >= 0.95, np.sort(rel[big])[-10:]
    finally:
        s.close()


def test_autograd_function_gives_adjoint_gradient_and_descends():
    import torch
    from xyz_b200 import diff
    W, H, spp = 64, 64, 4
    ds, s = _diff_setup()
    try:
        R = diff.Renderer(s, ds.scene.camera, W, H, spp, adjoint_offset=0)
        s.set_materials(ds.target_albedo, ds.target_emission)
        target = R.render()
        alb = torch.tensor(ds.albedo, device="cuda", requires_grad=True)
        em = torch.tensor(ds.emission, device="cuda", requires_grad=True)
        img = R(alb, em)
        loss = ((img - target) ** 2).sum()
        loss.backward()
        # the harness's gradient is the library adjoint with d_film = dL/dimage / spp
        d_film = (2.0 * (img.detach() - target) / spp).contiguous()
        s.set_materials(alb.detach(), em.detach())
        ga, ge = s.adjoint(ds.scene.camera, W, H, spp, d_film, max_depth=6, rr_threshold=0.0)
        torch.testing.assert_close(alb.grad, ga, rtol=1e-4, atol=1e-6 * float(ga.abs().max()))
        torch.testing.assert_close(em.grad, ge, rtol=1e-4, atol=1e-6 * float(ge.abs().max()))
        # a few plain gradient steps lower the loss (same samples: deterministic)
        opt = torch.optim.Adam([alb, em], lr=1e-2)
        first = float(loss.detach())
        for _ in range(5):
            opt.zero_grad()
            l = ((R(alb, em) - target) ** 2).sum()
            l.backward()
            opt.step()
            with torch.no_grad():
                alb.clamp_(0.0, 1.0)
        final = float(((R(alb, em) - target) ** 2).sum())
        assert final < first
    finally:
        s.close()


def test_adjoint_rejects_spectral_and_profile_modes():
    import torch
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    with api.Scene(sd) as s:
        d = torch.zeros((8, 8, 3), device="cuda")
        cam = api.camera_desc(sd.camera)
        nm = len(sd.is_light)
        ga = torch.zeros((nm, 3), device="cuda")
        ge = torch.zeros(nm, device="cuda")
        import ctypes as C
        for mode in ("spectral", "profile"):
            rp = api.render_params(8, 8, 1)
            if mode == "spectral":
                rp.spectral = 1
            else:
                rp.profile = 1
            rc = api.load_library().xyzgpu_adjoint(s.handle, C.byref(cam), C.byref(rp), d.data_ptr(),
                                                   ga.data_ptr(), ge.data_ptr(), None)
            assert rc == -1
