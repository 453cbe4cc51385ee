"""The oracle's reference gradient (xyzo_adjoint: per-contribution derivatives of
the XYZ estimator) against central finite differences of the oracle's own
renders on the same random streams, and the emission extension's neutral
default (scale 1 = the reference's film)."""

import numpy as np

from tests.helpers import ensure_port


def _loss(P, spp, dfilm, seed=3):
    f = P.render(spp, seed=seed, nthreads=0).astype(np.float64)
    return float((f * dfilm).sum())


def test_oracle_gradient_matches_central_differences():
    from xyz_b200 import scenes
    sd = scenes.cornell_box(pinhole=True)
    P = ensure_port()
    P.scene_create(sd)
    W, H, spp = 20, 16, 6
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=6, rr_threshold=0.0)
    nm = len(sd.is_light)
    rng = np.random.default_rng(5)
    dfilm = rng.standard_normal((H, W, 3)).astype(np.float32)
    alb = np.asarray(sd.albedo_xyz, np.float32).copy()
    em = np.full(nm, 1.5, np.float32)
    P.set_materials(alb, em)
    ga, ge = P.adjoint(dfilm, spp, 3, nm)
    h = 1e-3
    for m in range(nm):
        if sd.is_light[m]:
            e1, e2 = em.copy(), em.copy()
            e1[m] += h
            e2[m] -= h
            P.set_materials(alb, e1)
            lp = _loss(P, spp, dfilm)
            P.set_materials(alb, e2)
            lm = _loss(P, spp, dfilm)
            fd = (lp - lm) / (2 * h)
            assert abs(ge[m] - fd) <= 1e-3 * abs(fd) + 1e-6, (m, ge[m], fd)
            continue
        assert ge[m] == 0.0
        for c in range(3):
            a1, a2 = alb.copy(), alb.copy()
            a1[m, c] += h
            a2[m, c] -= h
            P.set_materials(a1, em)
            lp = _loss(P, spp, dfilm)
            P.set_materials(a2, em)
            lm = _loss(P, spp, dfilm)
            fd = (lp - lm) / (2 * h)
            assert abs(ga[m, c] - fd) <= 2e-3 * abs(fd) + 1e-3, (m, c, ga[m, c], fd)
    P.set_materials(alb, np.ones(nm, np.float32))


def test_emission_scale_one_is_the_reference_film():
    from xyz_b200 import scenes
    sd = scenes.cornell_box(pinhole=True)
    P = ensure_port()
    P.scene_create(sd)
    P.set_camera(sd.camera, 24, 24)
    P.set_path_params(max_depth=8)
    base = P.render(2, seed=1, nthreads=0)
    nm = len(sd.is_light)
    P.set_materials(None, np.ones(nm, np.float32))
    assert np.array_equal(P.render(2, seed=1, nthreads=0), base)
    P.set_materials(None, np.full(nm, 2.0, np.float32))
    doubled = P.render(2, seed=1, nthreads=0)
    # the film is linear in the (single) light's emission
    np.testing.assert_allclose(doubled, 2.0 * base, rtol=1e-5, atol=1e-6)


def test_albedo_scaling_matches_directional_derivative():
    """Scaling every albedo by s scales a contribution that carries k albedo
    factors by s^k, so d film / d s at s = 1 = sum_k k C_k, which must equal the
    directional derivative sum_m albedo_m . d film / d albedo_m of the
    per-material gradient."""
    from xyz_b200 import scenes
    sd = scenes.cornell_box(pinhole=True)
    P = ensure_port()
    P.scene_create(sd)
    W, H, spp = 16, 16, 4
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=5, rr_threshold=0.0)
    nm = len(sd.is_light)
    alb = np.asarray(sd.albedo_xyz, np.float32).copy()
    dfilm = np.ones((H, W, 3), np.float32)
    P.set_materials(alb, np.ones(nm, np.float32))
    ga, _ = P.adjoint(dfilm, spp, 0, nm)
    directional = float((ga * alb.astype(np.float64)).sum())
    h = 1e-3
    P.set_materials(alb * np.float32(1 + h), None)
    lp = _loss(P, spp, dfilm, seed=0)
    P.set_materials(alb * np.float32(1 - h), None)
    lm = _loss(P, spp, dfilm, seed=0)
    P.set_materials(alb, None)
    fd = (lp - lm) / (2 * h)
    assert abs(directional - fd) <= 1e-3 * abs(fd)
