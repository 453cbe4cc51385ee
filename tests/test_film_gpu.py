"""Film output on the GPU: the Radiance pixels of ImageFilm::SaveAsHdr
(xyz/core/imagefilm_hdr.cpp) and the float2bmp tone operators
(float2bmp/main.cpp:69-118) computed by kernels, against the C oracle (whose
Radiance pixels tests/test_film_io.py pins to the reference's own writer) and
the reference's writer itself; and resuming a render from a checkpoint."""

import numpy as np
import pytest

from tests.helpers import ensure_port, read_hdr, sample_films

pytestmark = pytest.mark.gpu


def _films():
    import torch
    from xyz_b200 import api, scenes
    out = [sample_films(s) for s in range(3)]
    sd = scenes.cornell_box()
    with api.Scene(sd) as s:
        out.append(s.render(sd.camera, 64, 48, 4, seed=1, max_depth=8).cpu().numpy())
        out.append(s.render(sd.camera, 64, 48, 4, seed=1, max_depth=8, spectral="continuous").cpu().numpy())
    torch.cuda.synchronize()
    return out


@pytest.mark.parametrize("xyze", [False, True])
def test_rgbe_kernel_equals_the_oracle(xyze):
    import torch
    from xyz_b200 import api
    P = ensure_port()
    for film in _films():
        for spp in (1.0, 4.0, 7.0):
            scale = np.float32(1.0) / np.float32(spp)
            g = api.encode_rgbe(torch.from_numpy(film).cuda(), float(scale), xyze=xyze).cpu().numpy()
            assert np.array_equal(g, P.encode_rgbe(film, scale, xyze))


def test_hdr_file_equals_the_reference_writer(tmp_path):
    import torch
    from oracle import refbind
    from xyz_b200 import api
    if not refbind.ref_film_available():
        pytest.skip("reference film writer not built")
    R = refbind.RefFilmLib()
    for k, film in enumerate(_films()):
        mine, ref = str(tmp_path / f"m{k}.hdr"), str(tmp_path / f"r{k}.hdr")
        api.save_hdr(mine, torch.from_numpy(film).cuda(), 4.0)
        R.save_hdr(ref, film, 4.0)
        hm, pm = read_hdr(mine)
        hr, pr = read_hdr(ref)
        assert hm[-1] == hr[-1] and np.array_equal(pm, pr)


@pytest.mark.parametrize("op,white", [("film", 0.0), ("linear", 0.0), ("reinhard", 0.0),
                                      ("reinhard_white", 0.0), ("reinhard_white", 2.5)])
@pytest.mark.parametrize("rgb", [False, True])
def test_tonemap_kernel_matches_the_oracle(op, white, rgb):
    """Same arithmetic as the tool; expf / powf of the device and of the host
    C library may differ in the last bit, which moves a byte by one where
    256 v lies on an integer: at most 1 apart, nearly all equal."""
    import torch
    from xyz_b200 import api
    P = ensure_port()
    for film in _films():
        for scale, exposure in ((0.25, 1.0), (1.0, 3.0)):
            g = api.tonemap(torch.from_numpy(np.nan_to_num(film)).cuda(), scale=scale, op=op, exposure=exposure,
                            white=white, rgb=rgb).cpu().numpy().astype(np.int32)
            c = P.tonemap(np.nan_to_num(film), scale=scale, op=api.TONEMAP_OPS[op], exposure=exposure,
                          white=white, rgb=rgb).astype(np.int32)
            assert g.shape == c.shape
            assert np.abs(g - c).max() <= 1
            assert (g == c).mean() >= 0.999


@pytest.mark.parametrize("spectral", ["off", "continuous"])
def test_render_resumed_from_a_checkpoint_equals_an_uninterrupted_render(tmp_path, spectral):
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    W, H, total, first = 48, 36, 9, 4
    kw = dict(seed=5, max_depth=8, spectral=spectral)
    path = str(tmp_path / "r.ckpt")
    with api.Scene(sd) as s:
        whole = np.zeros((H, W, 3), np.float32)
        s.render(sd.camera, W, H, total, film=whole, **kw)
        part = np.zeros((H, W, 3), np.float32)
        s.render(sd.camera, W, H, first, film=part, **kw)
        rp = api.render_params(W, H, first, seed=5, max_depth=8, spectral=spectral)
        api.save_checkpoint(path, rp, first, part)
        rp2, done, film = api.load_checkpoint(path)
        assert done == first and rp2.seed == 5 and rp2.spectral == rp.spectral
        s.render(sd.camera, W, H, total - done, spp_offset=done, film=film, accumulate=True, **kw)
    assert np.array_equal(film, whole)
