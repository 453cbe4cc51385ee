"""The .ren shell (include/xyzgpu_shell.hpp, program xyz_b200/xyzgpu_shell)
against the reference's shell semantics (xyz/core/shell.cpp:204-497): the
script grammar, the saved .ren document, the output folder and image names;
on the GPU, the images it writes against renders of the same scene through
the library."""

import glob
import os
import re
import subprocess

import numpy as np
import pytest

from tests.helpers import ROOT
from tests.test_mqo import _box_obj, _icosphere_obj, dump_exe  # noqa: F401 (fixture)

SHELL = os.path.join(ROOT, "xyz_b200", "xyzgpu_shell")


@pytest.fixture(scope="module")
def shell_exe():
    if not os.path.exists(SHELL):
        subprocess.run(["make", "-C", os.path.join(ROOT, "xyz_b200", "csrc"), "-j8"], check=True)
    return SHELL


def _run(exe, cwd, script, name="job", timeout=600):
    with open(os.path.join(cwd, name + ".ren"), "w") as f:
        f.write(script)
    return subprocess.run([exe, name], cwd=cwd, capture_output=True, text=True, timeout=timeout, check=True)


def test_saved_script_has_the_reference_layout(shell_exe, tmp_path):
    script = "\n".join([
        "rem settings of a test", "=begin", "set dim 1 1", "load nothing", "=end",
        "  set dim 64 0  ",                     # trimmed; a size below 1 becomes 1
        "set eye 1.5 2.25 -3.125", "set at 0 1 0.1",
        "set it 1 min 30 s",
        "set rt 2 hours 5 sec",
        "set rep 1",
        "load missing_scene",                   # the name is kept though the file is absent
        "save demo",
        "frobnicate",
        "quit",                                 # no effect in a script
        "set it 1 d 2 hr 3 m 4 s 9 fortnights",
        "save demo2",
        "ren",                                  # nothing is loaded: an error, then the script goes on
        "set rt 0 s", "set it 0 s",
        "save demo3",
    ]) + "\n"
    out = _run(shell_exe, str(tmp_path), script)
    assert "undefined" in out.stderr
    assert open(tmp_path / "demo.ren").read() == (
        "load missing_scene\n\nset eye 1.5 2.25 -3.125\nset at  0 1 0.1\n\nset dim 64 1\n"
        "set it  1 minute 30 seconds\nset rt  2 hours 5 seconds\n\nset rep 1\nren\n")
    # `it` longer than `rt` raises `rt` (shell.cpp:240-246)
    assert open(tmp_path / "demo2.ren").read().splitlines()[6:8] == [
        "set it  1 day 2 hours 3 minutes 4 seconds", "set rt  1 day 2 hours 3 minutes 4 seconds"]
    assert open(tmp_path / "demo3.ren").read().splitlines()[6:8] == ["set it   0 s", "set rt   0 s"]
    assert "no scene is loaded" in out.stderr


def test_saved_script_reads_back_to_the_same_state(shell_exe, tmp_path):
    _run(shell_exe, str(tmp_path), "set eye 0.1 0.2 0.3\nset at 4 5 6\nset dim 320 200\nset rt 3 m\n"
                                   "set it 45 s\nset rep 0\nsave a\n")
    text = open(tmp_path / "a.ren").read()
    # the saved script, without its last line (ren), run again and saved again
    _run(shell_exe, str(tmp_path), text.replace("ren\n", "") + "save b\n", name="again")
    assert open(tmp_path / "b.ren").read() == text


def test_algorithms_the_tracer_lacks_are_refused(shell_exe, tmp_path):
    out = _run(shell_exe, str(tmp_path), "set rt 1 s\nset rep 8\nren\nset rep 15\nren\n")
    assert "rep 8 (BPT/) is not available" in out.stderr
    assert not os.path.exists(tmp_path / "xyzgpu_shell")


def _lambert_document(path):
    mats = ['\t"white" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) emi(0.000) spc(0.700) power(5.00)',
            '\t"lamp" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) emi(1.000) spc(0.000) power(5.00)',
            '\t"cloth mcc-red" shader(3) col(0.2 0.3 0.4 1.000) dif(0.800) amb(0.600) emi(0.000) spc(0.500) power(5.00)']
    # the camera inside the room (its boxes' faces point inwards), the lamp a
    # ceiling quad facing down
    lines = ["Metasequoia Document", "Format Text Ver 1.0", "",
             "Scene {", "\tpos 0.0000 0.0000 95.0000", "\tlookat 0.0000 100.0000 0.0000", "\thead 0.0000",
             "\tpich 0.0000", "}", f"Material {len(mats)} {{"] + mats + ["}"]
    lines += _box_obj("room", (-100, 0, -100), (100, 200, 100), 0)
    lines += ['Object "lamp" {', "\tvisible 15", "\tshading 0", "\tvertex 4 {",
              "\t\t-25.0000 199.0000 -25.0000", "\t\t25.0000 199.0000 -25.0000", "\t\t25.0000 199.0000 25.0000",
              "\t\t-25.0000 199.0000 25.0000", "\t}", "\tface 2 {", "\t\t3 V(0 2 1) M(1)", "\t\t3 V(0 3 2) M(1)",
              "\t}", "}"]
    lines += _icosphere_obj("ball", (-30, 40, 0), 35, 1, 2)
    lines += ["Eof"]
    open(path, "w").write("\n".join(lines) + "\n")


def _scene_from_dump(dump, path, pre):
    from xyz_b200 import scenes
    subprocess.run([dump, "--desc", path, pre], check=True)
    subprocess.run([dump, path, pre], check=True)
    f32 = lambda e: np.fromfile(pre + e, np.float32)   # noqa: E731
    i32 = lambda e: np.fromfile(pre + e, np.int32)     # noqa: E731
    nrm = f32(".nrm")
    cam = f32(".cam")
    return scenes.SceneData(
        positions=f32(".pos").reshape(-1, 3), tris=i32(".tri").reshape(-1, 3), tri_mat=i32(".mat"),
        albedo_xyz=f32(".alb").reshape(-1, 3), is_light=i32(".light"), light_power_xyz=f32(".power"),
        normals=nrm.reshape(-1, 3) if nrm.size else None,
        camera=scenes.Camera(eye=tuple(cam[:3]), at=tuple(cam[3:])),
        material_kind=i32(".kind"), shininess=f32(".shin"))


def _read_pfm(path):
    with open(path, "rb") as f:
        assert f.readline() == b"PF\n"
        w, h = map(int, f.readline().split())
        assert float(f.readline()) < 0
        return np.frombuffer(f.read(), "<f4").reshape(h, w, 3)


def _mean_image(film, spp):
    img = (np.asarray(film, np.float32) * np.float32(1.0 / spp)).astype(np.float32)
    img[~np.isfinite(img).all(axis=-1)] = 0.0
    return img


@pytest.mark.gpu
@pytest.mark.parametrize("rep", [0, 1])
def test_shell_images_are_the_librarys_render(shell_exe, dump_exe, tmp_path, rep):  # noqa: F811
    from xyz_b200 import api
    W, H, spp, seed = 48, 36, 24, 5
    doc = str(tmp_path / "room.mqo")
    _lambert_document(doc)
    _run(shell_exe, str(tmp_path), f"load room\nset dim {W} {H}\nset spp {spp}\nset seed {seed}\n"
                                   f"set rt 1 hour\nset it 1 hour\nset rep {rep}\nren\nexit\n")
    folder = "IDPT" if rep else "PT"
    pfms = glob.glob(str(tmp_path / "xyzgpu_shell" / f"room 0048x0036 *T*.*.* {folder}" / "*.pfm"))
    assert len(pfms) == 1, pfms
    m = re.fullmatch(r"\d\dh\d\dm\d\ds 0000(\d\d)spp (\d{12})\.pfm", os.path.basename(pfms[0]))
    assert m and int(m.group(1)) == spp
    img = _read_pfm(pfms[0])
    sd = _scene_from_dump(dump_exe, doc, str(tmp_path / "desc"))
    with api.Scene(sd) as s:
        if rep == 0:
            film = s.render(sd.camera, W, H, spp, seed=seed).cpu().numpy()
            c = s.render_counters()
            assert int(m.group(2)) == c["extension_rays"] + c["shadow_rays"]
        else:
            with api.Importons(s, seed=seed) as imp:
                film = imp.render(sd.camera, W, H, spp, seed=seed).cpu().numpy()
    # the shell renders in passes of growing size into one host film; the sums
    # do not depend on the passes
    assert np.array_equal(img, _mean_image(film, spp))
    assert img.mean() > 0
