"""The spectral estimator restated in C (oracle/xyz_oracle.c, one wavelength
bin per path) against the reference's own spectral renderer built from its
sources (renderer/, oracle/_ref/libxyztwin_thinlens.so).  The reference draws
from std::mt19937_64, so the comparison is statistical: per-pixel means within
3 sigma and the image mean within 5 sigma."""

import numpy as np
import pytest

from tests.helpers import ensure_port


def _stats(render, spp):
    s1 = s2 = 0.0
    for s in range(spp):
        f = render(s).astype(np.float64)
        s1 = s1 + f
        s2 = s2 + f * f
    m = s1 / spp
    return m, np.sqrt(np.maximum(s2 / spp - m * m, 0.0) / spp)


def test_spectral_port_matches_the_reference_spectral_renderer():
    from oracle import refbind
    from xyz_b200 import scenes
    if not refbind.twin_available():
        pytest.skip("spectral reference oracle not built (make -C oracle)")
    sd = scenes.cornell_box(pinhole=False)
    T = refbind.TwinLib()
    sd.light_power_spd = T.light_spd()       # the reference lights with its Mercury arc
    T.scene_create(sd)
    P = ensure_port()
    P.scene_create(sd)
    P.set_spectra(sd.albedo_spd, sd.light_power_spd)
    P.set_spectral(1, 1)
    W, H, spp = 20, 14, 160
    for L in (T, P):
        L.set_camera(sd.camera, W, H)
        L.set_path_params(max_depth=7)
    mt, st = _stats(lambda s: T.render(1, seed=3, s0=s, nthreads=4), spp)
    mp, sp = _stats(lambda s: P.render(1, seed=4, s0=s, nthreads=4), spp)
    P.set_spectral(0, 1)
    se = np.sqrt(st ** 2 + sp ** 2)
    lum = (slice(None), slice(None), 1)
    valid = se[lum] > 0
    z = np.abs(mt[lum] - mp[lum])[valid] / se[lum][valid]
    assert (z > 3).mean() < 0.03, (z > 3).mean()
    gse = np.sqrt((se[lum] ** 2).sum()) / se[lum].size
    assert abs(mt[lum].mean() - mp[lum].mean()) < 5 * gse


def test_spectral_port_binned_one_hero_is_unbiased_against_xyz_for_grey_scenes():
    """With grey (flat) albedos and a flat emitter, spectral and XYZ estimators
    share their expectation up to the CMF normalisation."""
    from xyz_b200 import scenes, spectrum
    sd = scenes.spheres_scene(level=1, n_spheres=2)
    P = ensure_port()
    P.scene_create(sd)
    P.set_spectra(sd.albedo_spd, sd.light_power_spd)
    P.set_camera(sd.camera, 16, 12)
    P.set_path_params(max_depth=6)
    P.set_spectral(0, 1)
    xyz = P.render(96, seed=1, nthreads=4).sum(axis=(0, 1))
    P.set_spectral(1, 4)
    spec = P.render(96, seed=2, nthreads=4).sum(axis=(0, 1))
    P.set_spectral(0, 1)
    # XYZ mode uses albedo = grey * XYZ(white) and Phi_xyz = pi A L * XYZ(flat);
    # spectral mode integrates grey * L * CMF: the same image up to XYZ(white)
    # versus the flat-spectrum XYZ per channel
    white = spectrum.ccir601_rgb_to_xyz((1, 1, 1)).astype(np.float64)
    ratio = spec / xyz
    assert np.all(np.abs(ratio - 1.0) < 0.25), ratio


def test_named_spectra_are_the_reference_tables():
    """xyz_b200.spectrum.NAMED_SPECTRA (illuminants and the Macbeth
    ColorChecker) against the reference's own tables, read from its build."""
    import re
    from tests.helpers import ref_lib
    from xyz_b200 import spectrum
    R = ref_lib(True)
    if R is None:
        pytest.skip("reference oracle not built (make -C oracle)")
    ref = R.named_spectra()
    assert len(ref) == len(spectrum.NAMED_SPECTRA) == 37
    for name, v in ref.items():
        mine = spectrum.named_spectrum(re.sub(r"(?<!^)(?=[A-Z])", "_", name).lower())
        assert np.array_equal(mine, v), name


def test_library_spectra_tables_equal_the_package_tables():
    """xyzgpu_named_spectrum / xyzgpu_spectrum_to_xyz (the C ABI for scene
    loaders) hold the same tables as xyz_b200.spectrum, pinned above."""
    import ctypes as C
    from xyz_b200 import api, spectrum
    L = api.load_library()
    out = np.zeros(31, np.float32)
    xyz = np.zeros(3, np.float32)
    for name, v in spectrum.NAMED_SPECTRA.items():
        assert L.xyzgpu_named_spectrum(name.encode(), out.ctypes.data) == 0, name
        assert np.array_equal(out, np.asarray(v, np.float32)), name
        L.xyzgpu_spectrum_to_xyz(out.ctypes.data, xyz.ctypes.data)
        assert np.array_equal(xyz, spectrum.spd_to_xyz(v)), name
    assert L.xyzgpu_named_spectrum(b"mcc_nothing", out.ctypes.data) == -1
