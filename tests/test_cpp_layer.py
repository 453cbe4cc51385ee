"""The C++ host layer (include/xyzgpu_scene.hpp) used from a C++ program."""

import os
import subprocess

import numpy as np
import pytest

from tests.helpers import ROOT

SRC = os.path.join(ROOT, "tests", "cpp", "xyz_render.cpp")


def _compile(tmp_path):
    exe = str(tmp_path / "xyz_render")
    libdir = os.path.join(ROOT, "xyz_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC,
                    "-o", exe, "-L", libdir, "-lxyzgpu", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline() == b"PF\n"
        w, h = (int(v) for v in f.readline().split())
        assert float(f.readline()) == -1.0
        data = np.frombuffer(f.read(), dtype="<f4")
    assert data.size == w * h * 3
    return data.reshape(h, w, 3)


def test_film_writers_match_the_reference_formats(tmp_path):
    exe = _compile(tmp_path)
    pfm, flt = str(tmp_path / "a.pfm"), str(tmp_path / "a.float")
    subprocess.run([exe, "--film-selftest", pfm, flt], check=True)
    film = (0.5 * np.arange(18, dtype=np.float32) - 2.0).reshape(2, 3, 3)
    s = np.float32(1.0) / np.float32(2.0)
    want = (film * s).astype(np.float32)
    want[1, 2, :] = 0.0                      # a non-finite pixel is written as 0
    assert np.array_equal(read_pfm(pfm), want)
    rgb = np.fromfile(flt, dtype="<f4").reshape(2, 3, 3)
    x, y, z = (film * s)[..., 0], (film * s)[..., 1], (film * s)[..., 2]
    r = np.float32(1.9104) * x - np.float32(0.5338) * y - np.float32(0.2891) * z
    assert np.allclose(rgb[..., 0][:1], np.maximum(r, 0)[:1], atol=1e-6)
    fin = np.isfinite(rgb)
    assert (rgb[fin] >= 0).all()
    # like the reference's SaveAsFloat, a non-finite pixel passes through
    assert not fin[1, 2].all()


@pytest.mark.gpu
def test_cpp_path_tracer_equals_the_c_abi_render(tmp_path):
    import torch
    from xyz_b200 import api, scenes
    exe = _compile(tmp_path)
    sd = scenes.cornell_box(pinhole=True)
    d = tmp_path / "scene"
    d.mkdir()
    sd.positions.astype("<f4").tofile(d / "positions.f32")
    sd.tris.astype("<i4").tofile(d / "triangles.i32")
    sd.tri_mat.astype("<i4").tofile(d / "material.i32")
    sd.albedo_xyz.astype("<f4").tofile(d / "albedo.f32")
    sd.is_light.astype("<i4").tofile(d / "is_light.i32")
    sd.light_power_xyz.astype("<f4").tofile(d / "power.f32")
    c = sd.camera
    np.array(list(c.eye) + list(c.at) + [c.film_size, c.focal_length, c.f_number, float(c.pinhole)],
             "<f4").tofile(d / "camera.f32")
    np.array([64, 48], "<i4").tofile(d / "dims.i32")
    out = str(tmp_path / "film.pfm")
    r = subprocess.run([exe, str(d), out, "12", "5", "21", "8"], check=True, capture_output=True, text=True)
    assert "passes 3 spp 12" in r.stdout
    with api.Scene(sd) as s:
        film = s.render(sd.camera, 64, 48, 12, seed=21, max_depth=8)
        torch.cuda.synchronize()
        ref = film.cpu().numpy()
    inv = np.float32(1.0) / np.float32(12.0)
    # progressive passes add the same samples in the same order: identical film
    assert np.array_equal(read_pfm(out), (ref * inv).astype(np.float32))


@pytest.mark.gpu
def test_cpp_guided_path_tracer(tmp_path):
    """GuidedPathTracer: the first quarter of the samples train the guide and
    stay out of the film; the film holds the rest, rendered with the guide,
    and its image agrees with the plain tracer's."""
    import torch
    from xyz_b200 import api, scenes
    exe = _compile(tmp_path)
    sd = scenes.cornell_box(pinhole=True)
    d = tmp_path / "scene"
    d.mkdir()
    sd.positions.astype("<f4").tofile(d / "positions.f32")
    sd.tris.astype("<i4").tofile(d / "triangles.i32")
    sd.tri_mat.astype("<i4").tofile(d / "material.i32")
    sd.albedo_xyz.astype("<f4").tofile(d / "albedo.f32")
    sd.is_light.astype("<i4").tofile(d / "is_light.i32")
    sd.light_power_xyz.astype("<f4").tofile(d / "power.f32")
    c = sd.camera
    np.array(list(c.eye) + list(c.at) + [c.film_size, c.focal_length, c.f_number, float(c.pinhole)],
             "<f4").tofile(d / "camera.f32")
    np.array([64, 48], "<i4").tofile(d / "dims.i32")
    out = str(tmp_path / "guided.pfm")
    r = subprocess.run([exe, str(d), out, "64", "16", "3", "8", "--guided"], check=True, capture_output=True,
                       text=True)
    assert "passes 3 spp 48" in r.stdout, r.stdout
    img = read_pfm(out)
    with api.Scene(sd) as s:
        plain = s.render(sd.camera, 64, 48, 64, seed=9, max_depth=8)
        torch.cuda.synchronize()
        plain = plain.cpu().numpy() / 64
    assert np.isfinite(img).all() and (img >= 0).all()
    assert abs(img.mean() / plain.mean() - 1.0) < 0.05


def _write_scene(sd, d, W=64, H=48):
    d.mkdir()
    sd.positions.astype("<f4").tofile(d / "positions.f32")
    sd.tris.astype("<i4").tofile(d / "triangles.i32")
    sd.tri_mat.astype("<i4").tofile(d / "material.i32")
    sd.albedo_xyz.astype("<f4").tofile(d / "albedo.f32")
    sd.is_light.astype("<i4").tofile(d / "is_light.i32")
    sd.light_power_xyz.astype("<f4").tofile(d / "power.f32")
    c = sd.camera
    np.array(list(c.eye) + list(c.at) + [c.film_size, c.focal_length, c.f_number, float(c.pinhole)],
             "<f4").tofile(d / "camera.f32")
    np.array([W, H], "<i4").tofile(d / "dims.i32")


@pytest.mark.gpu
def test_cpp_path_tracer_resumes_from_its_checkpoint(tmp_path):
    """PathTracer with a checkpoint: a render stopped after 6 of 12 samples and
    run again continues from the file, and its film is the uninterrupted
    render's film bit for bit; the .hdr and .bmp outputs come from the GPU."""
    from tests.helpers import read_hdr
    from xyz_b200 import scenes
    exe = _compile(tmp_path)
    sd = scenes.cornell_box(pinhole=True)
    d = tmp_path / "scene"
    _write_scene(sd, d)
    ck = str(tmp_path / "r.ckpt")
    a, b = str(tmp_path / "a.pfm"), str(tmp_path / "b.pfm")
    r = subprocess.run([exe, str(d), b, "6", "3", "21", "8", "--checkpoint", ck], check=True,
                       capture_output=True, text=True)
    assert "passes 2 spp 6" in r.stdout
    r = subprocess.run([exe, str(d), b, "12", "3", "21", "8", "--checkpoint", ck], check=True,
                       capture_output=True, text=True)
    assert "passes 2 spp 12" in r.stdout, r.stdout     # resumed at 6: two more passes
    subprocess.run([exe, str(d), a, "12", "3", "21", "8"], check=True, capture_output=True)
    assert np.array_equal(read_pfm(a), read_pfm(b))
    h = str(tmp_path / "c.hdr")
    subprocess.run([exe, str(d), h, "4", "4", "21", "8"], check=True, capture_output=True)
    head, px = read_hdr(h)
    assert head[-1] == "-Y 48 +X 64" and px[..., 3].max() > 0
    bm = str(tmp_path / "c.bmp")
    subprocess.run([exe, str(d), bm, "4", "4", "21", "8"], check=True, capture_output=True)
    raw = open(bm, "rb").read()
    assert raw[:2] == b"BM" and len(raw) == 54 + 64 * 3 * 48
