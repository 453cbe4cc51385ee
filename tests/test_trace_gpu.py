"""Closest-hit parity of the CUDA traversal (xyzgpu_trace_closest) with the
reference's Scene::FindIntersection (golden fixtures) and with the oracle."""

import numpy as np
import pytest

from tests.helpers import ensure_port, grazing_mask, load_fixture

pytestmark = pytest.mark.gpu

BUILDERS = ["host", "device"]


def _scene(sd, builder, **kw):
    from xyz_b200 import api
    try:
        return api.Scene(sd, builder=builder, **kw)
    except api.XyzGpuError as e:
        if builder == "device" and "not available" in str(e):
            pytest.skip("device builder not in this build")
        raise


@pytest.mark.parametrize("builder", BUILDERS)
@pytest.mark.parametrize("name", ["cornell_trace.npz", "spheres_l3_trace.npz"])
def test_trace_matches_reference_golden(name, builder):
    sd, z = load_fixture(name)
    sd.light_power_xyz = np.ones(3, np.float32)
    with _scene(sd, builder) as s:
        tri, t, f, g, back = s.trace(z["org"], z["dir"])
    ok = ~grazing_mask(sd, z["org"], z["dir"], z["tri"], z["f"], z["g"])
    assert ok.mean() > 0.95
    assert np.array_equal(tri[ok], z["tri"][ok])
    hit = ok & (z["tri"] >= 0)
    rel = np.abs(t[hit] - z["t"][hit]) / np.abs(z["t"][hit])
    assert rel.max() <= 1e-5
    assert np.array_equal(back[hit], z["back"][hit])


@pytest.mark.parametrize("builder", BUILDERS)
def test_trace_large_mesh_matches_oracle(builder):
    from xyz_b200 import scenes
    sd = scenes.spheres_scene(level=5, n_spheres=3, seed=3)
    P = ensure_port()
    P.scene_create(sd)
    org, d = scenes.random_rays(sd, 100_000, seed=5)
    # also rays from the camera towards random points inside random triangles
    c = np.asarray(sd.camera.eye, np.float32)
    rng = np.random.default_rng(1)
    ti = rng.integers(0, sd.n_tris, 50_000)
    bc = rng.dirichlet([1.0, 1.0, 1.0], 50_000)
    tgt = (bc[:, :, None] * sd.positions[sd.tris[ti]]).sum(axis=1)
    d2 = tgt - c
    d2 /= np.linalg.norm(d2, axis=1, keepdims=True)
    org = np.concatenate([org, np.tile(c, (50_000, 1))]).astype(np.float32)
    d = np.concatenate([d, d2]).astype(np.float32)
    rt, rtt, rf, rg, rb = P.trace(org, d, nthreads=0)
    with _scene(sd, builder) as s:
        tri, t, f, g, back = s.trace(org, d)
        st = s.stats()
    assert st["n_nodes"] > 1000 and st["max_depth"] <= 60
    ok = ~grazing_mask(sd, org, d, rt, rf, rg)
    assert ok.mean() > 0.97
    same = tri[ok] == rt[ok]
    assert same.all(), f"{(~same).sum()} of {ok.sum()} non-grazing rays differ"
    hit = ok & (rt >= 0)
    assert (np.abs(t[hit] - rtt[hit]) <= 1e-5 * np.abs(rtt[hit])).all()


@pytest.mark.parametrize("builder", BUILDERS)
def test_tree_structure_invariants(builder):
    from xyz_b200 import scenes
    sd = scenes.spheres_scene(level=4, n_spheres=2, seed=1)
    with _scene(sd, builder) as s:
        nodes, refs = s.tree()
        st = s.stats()
    n = nodes.shape[0]
    assert n == st["n_nodes"]
    tag = nodes[:, 1] & 3
    interior = tag != 3
    child = nodes[interior, 1] >> 2
    assert (child + 1 < n).all() and (child > np.nonzero(interior)[0]).all()
    leaf = ~interior
    cnt = nodes[leaf, 1] >> 2
    beg = nodes[leaf, 0]
    assert (beg.astype(np.int64) + cnt <= refs.shape[0]).all()
    assert int(cnt.sum()) == refs.shape[0] == st["n_leaf_refs"]
    assert (refs >= 0).all() and (refs < sd.n_tris).all()
    assert np.unique(refs).shape[0] == sd.n_tris   # every triangle reachable
    # each node is the child of exactly one interior node (except the root)
    parents = np.zeros(n, np.int64)
    np.add.at(parents, child, 1)
    np.add.at(parents, child + 1, 1)
    assert parents[0] == 0 and (parents[1:] == 1).all()


def _triangle_soup(n, seed):
    """n random small triangles in a unit box: one flat root node of n
    references (n = 2,050 is just above a multiple of the builder's 128 slices,
    so a big node's last slices hold one reference or none)."""
    from xyz_b200 import scenes
    rng = np.random.default_rng(seed)
    c = rng.uniform(-1.0, 1.0, (n, 1, 3))
    pos = (c + rng.normal(scale=0.05, size=(n, 3, 3))).reshape(-1, 3).astype(np.float32)
    tris = np.arange(3 * n, dtype=np.int32).reshape(n, 3)
    mat = np.zeros(n, np.int32)
    mat[:2] = 1
    sd = scenes.SceneData(pos, tris, mat, np.array([[0.5] * 3, [0.0] * 3], np.float32),
                          np.array([0, 1], np.int32), np.ones(3, np.float32))
    return sd


@pytest.mark.parametrize("case", ["spheres-l4x3", "spheres-l6x4", "soup-2050", "soup-4099",
                                  "spheres-1M"])
def test_device_tree_equals_host_tree(case):
    """The device builder (sliced histograms and counts for big nodes) builds
    the host builder's tree exactly: on a 15k-triangle mesh; on 328k
    triangles, whose upper levels hold many big nodes sharing the slices; on
    flat soups whose root has 2,050 / 4,099 references (empty and one-element
    trailing slices); and on the 984,322-triangle benchmark scene."""
    from xyz_b200 import scenes
    if case == "spheres-l4x3":
        sd = scenes.spheres_scene(level=4, n_spheres=3, seed=2)
    elif case == "spheres-l6x4":
        sd = scenes.spheres_scene(level=6, n_spheres=4, seed=5)
    elif case.startswith("soup"):
        sd = _triangle_soup(int(case.split("-")[1]), seed=3)
    else:
        sd = scenes.spheres_scene(level=7, n_spheres=3, seed=0)
    with _scene(sd, "host") as a, _scene(sd, "device") as b:
        na, ra = a.tree()
        nb, rb = b.tree()
    assert np.array_equal(na, nb)
    assert np.array_equal(ra, rb)


def test_ray_starting_on_a_split_plane():
    """A symmetric scene gets a split plane at x = 0; rays from a camera at
    x = 0 start on it and must still find the closest hit on either side."""
    from xyz_b200 import scenes
    sd = scenes.spheres_scene(level=2, n_spheres=2, seed=0)
    P = ensure_port()
    P.scene_create(sd)
    rng = np.random.default_rng(4)
    d = rng.normal(size=(20000, 3)).astype(np.float32)
    d[:, 1] = -np.abs(d[:, 1])
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    org = np.tile(np.array([0.0, 1.6, 4.8], np.float32), (20000, 1))
    rt, rtt, rf, rg, _ = P.trace(org, d)
    with _scene(sd, "host") as s:
        tri, t, *_ = s.trace(org, d)
    ok = ~grazing_mask(sd, org, d, rt, rf, rg)
    assert (tri[ok] == rt[ok]).all()


def test_ray_interval_is_honoured():
    from xyz_b200 import scenes
    sd = scenes.cornell_box()
    org = np.array([[0.0, 1.0, 0.0]] * 3, np.float32)
    d = np.array([[0.0, -1.0, 0.0]] * 3, np.float32)   # floor at distance 1
    with _scene(sd, "host") as s:
        tri, t, *_ = s.trace(org, d)
        assert (tri >= 0).all() and np.allclose(t, 1.0)
        tri2, *_ = s.trace(org, d, tmax=0.5)
        assert (tri2 == -1).all()
        tri3, t3, *_ = s.trace(org, d, tmin=1.5)
        assert (tri3 == -1).all()


def test_trace_counters_and_empty_batch():
    import torch
    from xyz_b200 import scenes
    sd = scenes.spheres_scene(level=3, n_spheres=1)
    org, d = scenes.random_rays(sd, 4096, seed=9)
    r = np.zeros((4096, 8), np.float32)
    r[:, 0:3], r[:, 3], r[:, 4:7], r[:, 7] = org, 1e-5, d, np.inf
    with _scene(sd, "host") as s:
        rays = torch.from_numpy(r).cuda()
        hits = torch.empty((4096, 4), device="cuda")
        c = s.trace_device(rays, hits, counted=True)
        hits2 = torch.empty((4096, 4), device="cuda")
        s.trace_device(rays, hits2)
        torch.cuda.synchronize()
        assert torch.equal(hits.view(torch.int32), hits2.view(torch.int32))
        assert c["rays"] == 4096 and c["nodes_visited"] >= 4096
        assert c["hits"] == int((hits[:, 3].contiguous().view(torch.int32) >= 0).sum())
        s.trace_device(rays[:0], hits[:0])   # n = 0 is a no-op
