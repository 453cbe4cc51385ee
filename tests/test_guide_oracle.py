"""The guide's CPU specification (oracle/guide_ref.py) checked on its own:
the mixture is a normalised density, the closed-form output gradient is the
derivative of -log p, and backpropagation through the network (without bf16
rounding) matches central differences of the loss."""

import math

import numpy as np

from oracle import guide_ref as G


def _params(seed=0, scale=0.5):
    rng = np.random.default_rng(seed)
    p = np.zeros(G.N_PARAMS, np.float32)
    for l in range(G.LAYERS):
        k = G.layer_in(l)
        p[G.param_w(l): G.param_w(l) + k * G.WIDTH] = rng.uniform(-1, 1, k * G.WIDTH) * scale * math.sqrt(6 / k)
        p[G.param_w(l) + k * G.WIDTH: G.param_w(l) + k * G.WIDTH + G.WIDTH] = rng.uniform(-0.1, 0.1, G.WIDTH)
    return p


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def test_mixture_integrates_to_one():
    rng = np.random.default_rng(1)
    o = rng.normal(size=(3, 64))
    o[:, 8:16] = rng.uniform(-3, 4, size=(3, 8))
    # Fibonacci sphere quadrature
    n = 200000
    i = np.arange(n) + 0.5
    z = 1 - 2 * i / n
    phi = math.pi * (1 + 5 ** 0.5) * i
    r = np.sqrt(1 - z * z)
    d = np.stack([r * np.cos(phi), r * np.sin(phi), z], 1)
    for row in o:
        lp = G.log_pdf(np.repeat(row[None], n, 0), d)
        assert abs(np.exp(lp).mean() * 4 * math.pi - 1.0) < 2e-3


def test_output_gradient_is_derivative_of_log_pdf():
    rng = np.random.default_rng(2)
    o = rng.normal(size=(5, 64))
    o[:, 8:16] = rng.uniform(-2, 3, size=(5, 8))
    d = _unit(rng.normal(size=(5, 3)))
    g = G.loss_grad(o, d, np.ones(5))
    h = 1e-6
    for j in list(range(40)):
        e = np.zeros(64)
        e[j] = h
        fd = -(G.log_pdf(o + e, d) - G.log_pdf(o - e, d)) / (2 * h)
        np.testing.assert_allclose(g[:, j], fd, rtol=1e-5, atol=1e-7)


def test_backprop_matches_central_differences():
    rng = np.random.default_rng(3)
    p = _params(3)
    n = 16
    rec = np.zeros((n, 10), np.float32)
    rec[:, :3] = rng.uniform(0, 1, (n, 3))
    rec[:, 3:6] = _unit(rng.normal(size=(n, 3)))
    rec[:, 6:9] = _unit(rng.normal(size=(n, 3)))
    rec[:, 9] = rng.uniform(0.5, 2.0, n)
    lo, inv = np.zeros(3, np.float32), np.ones(3, np.float32)
    g = G.gradient(p, rec, lo, inv, 0.1, rounding=False)
    h = 1e-3
    idx = rng.choice(G.N_PARAMS, size=60, replace=False)
    for i in idx:
        pp, pm = p.astype(np.float64).copy(), p.astype(np.float64).copy()
        pp[i] += h
        pm[i] -= h
        fd = (G.loss(pp, rec, lo, inv, 0.1, rounding=False) - G.loss(pm, rec, lo, inv, 0.1, rounding=False)) / (2 * h)
        assert abs(g[i] - fd) <= 1e-4 * max(1.0, abs(fd)), (i, g[i], fd)
