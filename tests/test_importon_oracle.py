"""The oracle's importance-driven path tracer (the reference's
Scene::EvaluteImportanceDrivenPathTracing with its light-importance map and
ImportanceQuery histograms, restated in oracle/xyz_oracle.c), on the CPU:
the histogram against a direct numpy statement of ImportanceQuery
(xyz/core/photonmap.cpp:321-401), and the estimator against the plain one."""

import numpy as np

from tests.helpers import ensure_port


def _frames(n, rng, lo, hi):
    pos = rng.uniform(lo, hi, (n, 3))
    nrm = rng.normal(size=(n, 3))
    nrm /= np.linalg.norm(nrm, axis=1, keepdims=True)
    t = np.stack([-nrm[:, 2], np.zeros(n), nrm[:, 0]], axis=1)
    t /= np.linalg.norm(t, axis=1, keepdims=True)
    b = np.cross(t, nrm)
    return np.concatenate([pos, t, b, nrm], axis=1).astype(np.float32)


def _numpy_hist(imp, fr, r=0.1):
    """ImportanceQuery over all importons (no spatial structure), float32."""
    f32 = np.float32
    r2 = f32(r) * f32(r)
    out = np.zeros((fr.shape[0], 16), np.float32)
    P, D = imp[:, :3].astype(f32), imp[:, 3:].astype(f32)
    for i, q in enumerate(fr):
        pos, tan, bin_, sn = q[0:3], q[3:6], q[6:9], q[9:12]
        c = np.full(16, f32(16), f32)
        d = P - pos
        near = (d * d).sum(axis=1, dtype=f32) < r2
        for dd, dv in zip(d[near], D[near]):
            cs = -f32(np.dot(dv, sn))
            if cs <= 0:
                continue
            vp = dd + dv * f32(np.dot(dd, sn))
            if f32(np.dot(vp, vp)) >= r2:
                continue
            u = min(int(f32(cs * cs) * f32(2)), 1)
            phi = f32(0.5) * np.arctan2(-f32(np.dot(dv, bin_)), -f32(np.dot(dv, tan)))
            if phi < 0:
                phi = f32(np.float64(phi) + np.pi)
            v = min(int(np.float64(phi) * (8 / np.pi)), 7)
            c[u * 8 + v] += 1
        out[i] = np.cumsum(c, dtype=f32)
    return out


def test_histogram_query_equals_a_direct_statement():
    from xyz_b200 import scenes
    sd = scenes.cornell_box()
    P = ensure_port()
    P.scene_create(sd)
    imp = P.importons_emit(20000, 16, 1, seed=5)
    assert imp.shape[0] > 5000
    P.importons_set(imp, 0.1, enable=False)
    rng = np.random.default_rng(0)
    fr = _frames(300, rng, [-1, 0, -1], [1, 2, 1])
    # put half of the query points on importons, where the histograms fill up
    fr[:150, :3] = imp[rng.integers(0, imp.shape[0], 150), :3]
    got = P.importons_query(fr)
    want = _numpy_hist(imp, fr)
    # atan2f of the C library and numpy's arctan may differ in the last bit
    # on a bin edge: nearly every histogram is identical
    same = (got == want).all(axis=1)
    assert same.mean() >= 0.99
    assert (got[:, -1] == want[:, -1]).all()          # totals always agree
    assert (got[:, -1] >= 256).all() and (got[150:, -1] > 256).mean() < (got[:150, -1] > 256).mean()


def test_importons_are_on_lambert_surfaces_and_unit_directions():
    from xyz_b200 import scenes
    sd = scenes.cornell_box()
    P = ensure_port()
    P.scene_create(sd)
    a = P.importons_emit(3000, 16, 1, seed=2)
    b = P.importons_emit(3000, 16, 1, seed=2)
    assert np.array_equal(a, b)
    assert np.allclose(np.linalg.norm(a[:, 3:], axis=1), 1.0, atol=1e-5)
    assert (a[:, 1] >= -1e-4).all() and (a[:, 1] <= 2.0 + 1e-4).all()
    c = P.importons_emit(3000, 16, 0, seed=2)      # with the light's direct hits
    assert c.shape[0] > a.shape[0]


def test_importance_driven_estimator_agrees_with_the_plain_one():
    """Unbiased: the histogram's every bin has a positive density (16 prior
    counts), so the image has the plain estimator's mean."""
    from xyz_b200 import scenes
    sd = scenes.cornell_box()
    P = ensure_port()
    P.scene_create(sd)
    imp = P.importons_emit(50000, 16, 1, seed=1)
    W, H, spp = 24, 18, 192
    P.set_camera(sd.camera, W, H)
    P.set_path_params(max_depth=8)
    try:
        P.importons_set(imp, 0.1, enable=False)
        a = P.render(spp, seed=10, nthreads=0).astype(np.float64) / spp
        P.importons_set(imp, 0.1, enable=True)
        b = P.render(spp, seed=11, nthreads=0).astype(np.float64) / spp
    finally:
        P.importons_set(imp, 0.1, enable=False)
    assert abs(b.mean() / a.mean() - 1.0) < 0.02
    # 6 x 6 blocks agree loosely (independent streams)
    ba = a.reshape(3, 6, 4, 6, 3).mean(axis=(1, 3))
    bb = b.reshape(3, 6, 4, 6, 3).mean(axis=(1, 3))
    assert np.abs(bb / ba - 1.0).max() < 0.1
