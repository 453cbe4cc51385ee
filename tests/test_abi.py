"""The C ABI library without a GPU: it loads, exports every function the
public header declares, and its host-side pieces behave."""

import ctypes as C
import os
import re

import numpy as np
import pytest

from tests.helpers import ROOT, ensure_port


def header_functions():
    src = open(os.path.join(ROOT, "include", "xyzgpu.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(xyzgpu_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_function():
    from xyz_b200 import api
    L = api.load_library()
    declared = header_functions()
    assert len(declared) >= 13
    for name in declared:
        assert hasattr(L, name), name
    assert sorted(api.EXPORTED) == sorted(declared)
    assert L.xyzgpu_abi_version() == 1


def test_philox_stream_matches_oracle():
    from xyz_b200 import api
    P = ensure_port()
    rng = np.random.default_rng(3)
    for _ in range(500):
        seed = int(rng.integers(0, 2**63))
        px, s, d = (int(v) for v in rng.integers(0, 2**31, size=3))
        d %= 64
        assert api.philox_u01(seed, px, s, d) == P.philox_u01(seed, px, s, d)


def test_philox_known_answer():
    """Philox4x32-10 known-answer vector from the Random123 distribution
    (counter = key = 0)."""
    from xyz_b200 import api
    # words of Philox4x32-10(ctr=0, key=0): 0x6627e8d5 0xe169c58d 0xbc57ac4c 0x9b00dbd8
    expect = [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    for k in range(4):
        assert api.philox_u01(0, 0, 0, k) == np.float32((expect[k] >> 8) * 2.0**-24)


def test_defaults():
    from xyz_b200 import api
    bp = api.default_build_params()
    assert (bp.leaf_max_tris, bp.bins, bp.empty_bonus) == (8, 64, 0.0)
    assert abs(bp.cost_traversal - 1.0) < 1e-7 and abs(bp.cost_intersect - 1.5) < 1e-7
    rp = api.RenderParams()
    api.load_library().xyzgpu_render_params_default(C.byref(rp))
    assert (rp.max_depth, rp.rr_start_depth) == (15, 1)
    assert abs(rp.rr_threshold - 0.2) < 1e-7


def test_null_arguments_are_errors_without_touching_a_device():
    from xyz_b200 import api
    L = api.load_library()
    assert L.xyzgpu_scene_create(None, None, None) == -1
    assert b"null" in L.xyzgpu_last_error()
    assert L.xyzgpu_trace_closest(None, None, 0, None, None) == -1
    assert L.xyzgpu_render(None, None, None, None, None) == -1
    L.xyzgpu_scene_destroy(None)


def test_scene_create_reports_missing_device_or_succeeds():
    torch = pytest.importorskip("torch")
    from xyz_b200 import api, scenes
    if torch.cuda.is_available():
        pytest.skip("device present; covered by GPU tests")
    with pytest.raises(api.XyzGpuError) as e:
        api.Scene(scenes.cornell_box())
    assert e.value.code in (-5, -2)
