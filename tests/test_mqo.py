"""Scene files (include/xyzgpu_mqo.hpp) against the reference's own code,
built from its sources (no GPU): Metasequoia documents against Scene::Load
(xyz/core/scene_mqo.cpp:547-696) and PLY meshes against its ply2mqo tool
(ply2mqo/main.cpp with librply)."""

import os
import struct
import subprocess

import numpy as np
import pytest

from tests.helpers import ROOT, ref_lib

SRC = os.path.join(ROOT, "tests", "cpp", "mqo_dump.cpp")


@pytest.fixture(scope="module")
def dump_exe(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("bin") / "mqo_dump")
    libdir = os.path.join(ROOT, "xyz_b200")
    subprocess.run(["g++", "-std=c++17", "-O2", "-Wall", "-I", os.path.join(ROOT, "include"), SRC, "-o", exe,
                    "-L", libdir, "-lxyzgpu", f"-Wl,-rpath,{libdir}"], check=True)
    return exe


def _icosphere_obj(name, centre, radius, shading, mat):
    from xyz_b200 import scenes
    v, f = scenes.icosphere(1)
    v = v * radius + np.asarray(centre)
    lines = [f'Object "{name}" {{', "\tdepth 0", "\tfolding 0", "\tscale 1.000000 1.000000 1.000000",
             "\tvisible 15", "\tlocking 0", f"\tshading {shading}", "\tfacet 59.5", "\tcolor 0.898 0.498 0.698",
             "\tcolor_type 0", f"\tvertex {len(v)} {{"]
    lines += [f"\t\t{x:.4f} {y:.4f} {z:.4f}" for x, y, z in v]
    lines += ["\t}", f"\tface {len(f)} {{"]
    lines += [f"\t\t3 V({a} {b} {c}) M({mat}) UV(0 0 1 0 0 1)" for a, b, c in f]
    lines += ["\t}", "}"]
    return lines


def _box_obj(name, lo, hi, mat, visible=15, quad=False):
    x0, y0, z0 = lo
    x1, y1, z1 = hi
    v = [(x0, y0, z0), (x1, y0, z0), (x1, y1, z0), (x0, y1, z0), (x0, y0, z1), (x1, y0, z1), (x1, y1, z1),
         (x0, y1, z1)]
    f = [(0, 2, 1), (0, 3, 2), (4, 5, 6), (4, 6, 7), (0, 1, 5), (0, 5, 4), (3, 7, 6), (3, 6, 2), (0, 4, 7),
         (0, 7, 3), (1, 2, 6), (1, 6, 5)]
    lines = [f'Object "{name}" {{', f"\tvisible {visible}", "\tshading 0", f"\tvertex {len(v)} {{"]
    lines += [f"\t\t{x:.4f} {y:.4f} {z:.4f}" for x, y, z in v]
    n = len(f) + (1 if quad else 0)
    lines += ["\t}", f"\tface {n} {{"]
    lines += [f"\t\t3 V({a} {b} {c}) M({mat})" for a, b, c in f]
    if quad:
        lines.append(f"\t\t4 V(0 1 2 3) M({mat})")     # the reference leaves a default triangle
    lines += ["\t}", "}"]
    return lines


def _document(path, scene=True):
    mats = ['\t"white" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) emi(0.000) spc(0.900) power(5.00)',
            '\t"lamp" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) emi(1.000) spc(0.000) power(5.00)',
            '\t"mirror" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) emi(0.000) spc(1.000) power(100.00)',
            '\t"gold" shader(3) col(1.000 0.780 0.340 1.000) dif(0.800) amb(0.600) emi(0.000) spc(1.000) power(40.00)',
            '\t"cloth mcc-orange-yellow" shader(3) col(0.2 0.3 0.4 1.000) dif(0.800) amb(0.600) emi(0.000) spc(0.500) power(5.00)',
            '\t"copper mcc-red" shader(3) col(0.2 0.3 0.4 1.000) dif(0.800) amb(0.600) emi(0.000) spc(1.000) power(20.00)']
    lines = ["Metasequoia Document", "Format Text Ver 1.0", ""]
    if scene:
        lines += ["Scene {", "\tpos 12.0000 -30.0000 1500.0000", "\tlookat 0.0000 100.0000 0.0000",
                  "\thead -0.5236", "\tpich 0.3000", "\tortho 0", "\tzoom2 5.0000", "\tamb 0.250 0.250 0.250",
                  "\tdirlights 1 {", "\t\tlight {", "\t\t\tdir 0.408 0.408 0.816", "\t\t}", "\t}", "}"]
    lines += [f"Material {len(mats)} {{"] + mats + ["}"]
    lines += _box_obj("room", (-100, 0, -100), (100, 200, 100), 0, quad=True)
    lines += _box_obj("hidden", (-10, 0, -10), (10, 20, 10), 0, visible=0)
    lines += _box_obj("lamp", (-20, 199, -20), (20, 199.9, 20), 1)
    lines += _icosphere_obj("ball", (-40, 40, 0), 35, 1, 3)
    lines += _icosphere_obj("orb", (40, 40, 10), 30, 1, 2)
    lines += _icosphere_obj("cloth", (0, 120, -40), 20, 1, 4)
    lines += _box_obj("block", (10, 0, 30), (50, 30, 60), 5)
    lines += ["Eof"]
    open(path, "w").write("\n".join(lines) + "\n")


def _mine(exe, path, pre):
    subprocess.run([exe, path, pre], check=True)
    geo = np.fromfile(pre + ".geo", np.float32).reshape(-1, 21)
    mat = np.fromfile(pre + ".mat", np.int32)
    key = np.fromfile(pre + ".key", np.int32)
    mats = np.fromfile(pre + ".mats", np.float32).reshape(-1, 5)
    cam = np.fromfile(pre + ".cam", np.float32)
    return geo, mat, key, mats, cam


def _rows(geo, mat):
    """Triangles as comparable rows.  A degenerate triangle (zero area: its
    normal is 0 / 0) keeps only its vertices and material: its normals are NaN
    in either form and no ray can hit it."""
    g = geo.copy()
    g[np.isnan(g[:, 9]), 9:] = 0.0
    return {tuple(r.tobytes() for r in (a, np.int32(m).reshape(1))) for a, m in zip(g, mat)}


@pytest.mark.parametrize("scene", [True, False])
def test_mqo_loader_builds_the_reference_scene(dump_exe, tmp_path, scene):
    R = ref_lib(True)
    if R is None:
        pytest.skip("reference oracle not built (make -C oracle)")
    path = str(tmp_path / "room.mqo")
    _document(path, scene)
    geo, mat, key, mats, cam = _mine(dump_exe, path, str(tmp_path / "mine"))
    ref = R.load_mqo(path)
    # the same triangles (the stored geometry bit for bit) and materials
    assert geo.shape == ref["geo"].shape
    assert _rows(geo, mat) == _rows(ref["geo"], ref["mat"])
    # the reference's order is Morton order too: its triangles carry
    # non-decreasing keys under this loader's key of the same triangle
    def tag(g, m):
        return g[:9].tobytes() + struct.pack("i", int(m))

    k_of = {tag(g, m): int(k) for g, m, k in zip(geo, mat, key)}
    ref_keys = np.array([k_of[tag(g, m)] for g, m in zip(ref["geo"], ref["mat"])])
    assert (np.diff(key) >= 0).all() and (np.diff(ref_keys) >= 0).all()
    assert np.array_equal(mats[:, 0].astype(np.int32), ref["kind"])
    assert np.array_equal(mats[:, 1:4], ref["albedo"])
    assert np.array_equal(mats[:, 4], ref["shininess"])
    if scene:
        assert np.array_equal(cam[:3], ref["eye"]) and np.array_equal(cam[3:], ref["at"])
    # a quad face leaves the reference's default triangle (0, 0, 0, material 0)
    assert (np.abs(geo[:, 3:9]).sum(axis=1) == 0).sum() == 1


def _ply(path, fmt):
    rng = np.random.default_rng(1)
    v = rng.uniform(-100, 100, (40, 3)).astype(np.float32)
    faces = [tuple(rng.choice(40, 3, replace=False)) for _ in range(30)] + [(1, 2, 3, 4)]
    strip = [0, 1, 2, 3, 4, -1, 5, 6, 7, 8]
    head = ["ply", f"format {fmt} 1.0", "comment made by a test", "element vertex 40", "property float x",
            "property float y", "property float z", "property uchar red", f"element face {len(faces)}",
            "property list uchar int vertex_indices", "element tristrips 1",
            "property list int int vertex_indices", "end_header"]
    with open(path, "wb") as f:
        f.write(("\n".join(head) + "\n").encode())
        if fmt == "ascii":
            for p in v:
                f.write(f"{float(p[0])!r} {float(p[1])!r} {float(p[2])!r} 7\n".encode())
            for fc in faces:
                f.write((f"{len(fc)} " + " ".join(str(i) for i in fc) + "\n").encode())
            f.write((f"{len(strip)} " + " ".join(str(i) for i in strip) + "\n").encode())
        else:
            e = "<" if fmt == "binary_little_endian" else ">"
            for p in v:
                f.write(struct.pack(e + "fffB", *p, 7))
            for fc in faces:
                f.write(struct.pack(e + "B" + "i" * len(fc), len(fc), *fc))
            f.write(struct.pack(e + "i" + "i" * len(strip), len(strip), *strip))


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_ply_conversion_writes_the_reference_tools_document(dump_exe, tmp_path, fmt):
    tool = os.path.join(ROOT, "oracle", "_ref", "xyzref_ply2mqo")
    if not os.path.exists(tool):
        pytest.skip("reference ply2mqo not built (make -C oracle)")
    ply = str(tmp_path / "mesh.ply")
    _ply(ply, fmt)
    subprocess.run([tool, ply], check=True, capture_output=True)
    mine = str(tmp_path / "mine.mqo")
    subprocess.run([dump_exe, "--ply2mqo", ply, mine], check=True)
    assert open(mine, "rb").read() == open(ply + ".mqo", "rb").read()
    # and as a scene, against the reference's Scene::Load of its tool's
    # document given the one material LoadPly adds.  The tool writes the faces
    # and the strips as two face chunks of one object, and Scene::Load resizes
    # its face array for each chunk (scene_mqo.cpp:384), so the strips'
    # 5 triangles overwrite the first faces and are all that is left.
    geo, mat, key, mats, cam = _mine(dump_exe, ply, str(tmp_path / "ply"))
    assert geo.shape[0] == 5 and mats.shape[0] == 1
    R = ref_lib(True)
    if R is None:
        pytest.skip("reference oracle not built (make -C oracle)")
    text = open(ply + ".mqo").read()
    at = text.index('Object "obj1"')
    text = (text[:at] + 'Material 1 {\n\t"mcc-white" shader(3) col(1.000 1.000 1.000 1.000) dif(0.800) amb(0.600) '
            'emi(0.000) spc(0.000) power(5.00)\n}\n' + text[at:])
    doc = str(tmp_path / "ref.mqo")
    open(doc, "w").write(text)
    ref = R.load_mqo(doc)
    assert _rows(geo, mat) == _rows(ref["geo"], ref["mat"])
    assert np.array_equal(mats[:, 1:4], ref["albedo"])
