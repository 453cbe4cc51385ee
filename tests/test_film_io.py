"""Film output formats (no GPU): the C oracle's Radiance pixels against the
reference's own ImageFilm::SaveAsHdr (xyz/core/imagefilm_hdr.cpp, built from
its sources into oracle/_ref), the library's host-side .hdr / .bmp writers
and the render checkpoint file."""

import os

import numpy as np
import pytest

from tests.helpers import ensure_port, read_hdr, sample_films


def test_oracle_rgbe_pixels_equal_the_reference_hdr_file(tmp_path):
    from oracle import refbind
    if not refbind.ref_film_available():
        pytest.skip("reference film writer not built (make -C oracle ref)")
    R, P = refbind.RefFilmLib(), ensure_port()
    for seed, spp in ((0, 1.0), (1, 3.0), (2, 64.0)):
        film = sample_films(seed)
        path = str(tmp_path / f"ref{seed}.hdr")
        R.save_hdr(path, film, spp)
        head, px = read_hdr(path)
        assert "FORMAT=32-bit_rle_rgbe" in head and head[-1] == f"-Y {film.shape[0]} +X {film.shape[1]}"
        mine = P.encode_rgbe(film, np.float32(1.0) / np.float32(spp))
        assert np.array_equal(mine, px)


def test_hdr_writer_round_trips_and_matches_the_reference_file_layout(tmp_path):
    """xyzgpu_hdr_write (host): header, run-length scanlines that decode to the
    given pixels; narrow images (< 8 pixels) are written flat."""
    from xyz_b200 import api
    rng = np.random.default_rng(3)
    for H, W in ((5, 40), (3, 7), (2, 300)):
        px = rng.integers(0, 256, (H, W, 4), dtype=np.uint8)
        px[:, 3:20] = px[:, 3:4]          # runs longer than 4
        px[0, : W // 2, 1] = 9
        path = str(tmp_path / f"a{W}.hdr")
        api.write_hdr(path, px)
        head, back = read_hdr(path)
        assert head[0] == "#?RADIANCE" and head[-1] == f"-Y {H} +X {W}"
        assert np.array_equal(back, px)
    api.write_hdr(str(tmp_path / "x.hdr"), px, xyze=True)
    head, back = read_hdr(str(tmp_path / "x.hdr"))
    assert "FORMAT=32-bit_rle_xyze" in head and head[-1].startswith("+Y")


def test_bmp_writer_header_and_rows(tmp_path):
    from xyz_b200 import api
    H, W = 3, 5
    stride = (3 * W + 3) & ~3
    rows = np.arange(H * stride, dtype=np.uint32).astype(np.uint8).reshape(H, stride)
    path = str(tmp_path / "a.bmp")
    api.write_bmp(path, rows, W, H)
    b = open(path, "rb").read()
    assert b[:2] == b"BM" and int.from_bytes(b[2:6], "little") == len(b) == 54 + H * stride
    assert int.from_bytes(b[10:14], "little") == 54 and int.from_bytes(b[18:22], "little") == W
    assert int.from_bytes(b[22:26], "little") == H and b[28] == 24
    assert b[54:] == rows.tobytes()


def test_checkpoint_round_trip_and_damage_is_detected(tmp_path):
    from xyz_b200 import api
    rp = api.render_params(37, 19, 6, seed=11, spp_offset=2, max_depth=9, rr_start_depth=3, spectral="continuous",
                           hero_wavelengths=4)
    film = sample_films(4)
    path = str(tmp_path / "c.ckpt")
    api.save_checkpoint(path, rp, 8, film)
    rp2, done, film2 = api.load_checkpoint(path)
    assert done == 8 and np.array_equal(film2, film, equal_nan=True)
    for f, _ in api.RenderParams._fields_:
        assert getattr(rp2, f) == getattr(rp, f), f
    raw = bytearray(open(path, "rb").read())
    raw[-5] ^= 0x10
    open(path, "wb").write(bytes(raw))
    with pytest.raises(api.XyzGpuError) as e:
        api.load_checkpoint(path)
    assert "damaged" in str(e.value)
    open(path, "wb").write(bytes(raw[:100]))
    with pytest.raises(api.XyzGpuError):
        api.load_checkpoint(path)
    assert not os.path.exists(path + ".part")
