"""Measurement logic of bench.py that runs without a GPU: the noise-corrected
relative MSE used for the guided tracer's time-to-relMSE figure."""

import numpy as np


def test_relmse_removes_the_reference_noise():
    import bench
    rng = np.random.default_rng(0)
    n = 400_000
    truth = rng.uniform(0.5, 2.0, n)
    sig_ref, sig_img = 0.05, 0.08   # relative noise of the reference halves / of the image
    a = truth * (1 + sig_ref * rng.standard_normal(n))
    b = truth * (1 + sig_ref * rng.standard_normal(n))
    img = truth * (1 + sig_img * rng.standard_normal(n))
    relmse, ref_noise, scale = bench.relmse_estimator(a, b)
    est = relmse(img)
    ry = (a + b) / 2 * scale
    den = ry ** 2 + 1e-2
    want = float(((sig_img * truth * scale) ** 2 / den).mean())   # the image's own error
    assert abs(est - want) < 0.03 * want, (est, want)
    # the subtracted term is the reference's variance, (sig_ref^2 / 2) relative
    ref_want = float(((sig_ref * truth * scale) ** 2 / 2 / den).mean())
    assert abs(ref_noise - ref_want) < 0.03 * ref_want, (ref_noise, ref_want)
    # exposure: the reference's mean maps to 1
    assert abs(float(((a + b) / 2).mean()) * scale - 1.0) < 1e-12


def test_relmse_of_the_reference_itself_is_zero_on_average():
    import bench
    rng = np.random.default_rng(1)
    n = 200_000
    truth = rng.uniform(0.5, 2.0, n)
    # small relative noise, as in the benchmark (the reference's own relMSE is
    # ~0.002): the reference's noise in the denominator then does not matter
    a = truth * (1 + 0.05 * rng.standard_normal(n))
    b = truth * (1 + 0.05 * rng.standard_normal(n))
    c = truth * (1 + 0.05 * rng.standard_normal(n))   # independent, as noisy as one half
    relmse, ref_noise, _ = bench.relmse_estimator(a, b)
    # an image as noisy as one half has twice the reference's own noise
    assert abs(relmse(c) - 2 * ref_noise) < 0.05 * ref_noise
