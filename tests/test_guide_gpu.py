"""Learned path guide kernels (tcgen05 BF16 MLP) against the CPU
specification oracle/guide_ref.py: forward outputs, the loss gradient of a
training batch (all layers, weights and biases), the Adam step, and training
that lowers the loss on a position-dependent target distribution."""

import math

import numpy as np
import pytest

from oracle import guide_ref as G

pytestmark = pytest.mark.gpu


def _guide(seed=0, **cfg):
    from xyz_b200 import api, scenes
    sd = scenes.cornell_box()
    s = api.Scene(sd)
    g = api.Guide(s, seed=seed, **cfg)
    return s, g


def _unit(v):
    return v / np.linalg.norm(v, axis=-1, keepdims=True)


def _records(n, seed, lo, hi):
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 10), np.float32)
    rec[:, :3] = rng.uniform(lo, hi, (n, 3))
    rec[:, 3:6] = _unit(rng.normal(size=(n, 3)))
    rec[:, 6:9] = _unit(rng.normal(size=(n, 3)))
    rec[:, 9] = rng.exponential(1.0, n)
    rec[rng.uniform(size=n) < 0.1, 9] = 0.0   # some records carry no weight
    return rec


def _trained_like_params(g, seed):
    """Random parameters with non-trivial outputs (the initial output layer is small)."""
    rng = np.random.default_rng(seed)
    p = g.params()
    p += rng.normal(0, 0.05, p.shape).astype(np.float32)
    return p


def test_forward_matches_oracle():
    import torch
    s, g = _guide(1)
    try:
        p = _trained_like_params(g, 1)
        g.set_params(p)
        st = s.stats()
        n = 1000   # 8 tiles, the last one partial
        rec = _records(n, 2, np.array(st["bounds_min"]), np.array(st["bounds_max"]))
        out = g.forward(torch.from_numpy(rec[:, :6].copy()).cuda()).cpu().numpy()
        ref, _ = G.forward(p, G.encode(rec[:, :6], g.lo, g.inv_ext))
        scale = np.abs(ref).max()
        assert np.abs(out - ref).max() <= 1e-2 * scale, np.abs(out - ref).max() / scale
        assert np.sqrt(((out - ref) ** 2).mean()) <= 2e-3 * scale
    finally:
        g.close()
        s.close()


def test_gradient_matches_oracle():
    import torch
    s, g = _guide(2)
    try:
        p = _trained_like_params(g, 2)
        g.set_params(p)
        st = s.stats()
        n = 700
        rec = _records(n, 3, np.array(st["bounds_min"]), np.array(st["bounds_max"]))
        gpu = g.gradient(torch.from_numpy(rec).cuda(), scale=1.0 / n).cpu().numpy().astype(np.float64)
        ref = G.gradient(p, rec, g.lo, g.inv_ext, 1.0 / n)
        for l in range(G.LAYERS):
            k = G.layer_in(l)
            sl = slice(G.param_w(l), G.param_w(l) + k * G.WIDTH + G.WIDTH)
            a, b = gpu[sl], ref[sl]
            err = np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)
            assert err <= 2e-2, (l, err)
        assert np.linalg.norm(gpu - ref) <= 1e-2 * np.linalg.norm(ref)
        # gradients accumulate: a second call adds the same amount
        acc = torch.from_numpy(gpu.astype(np.float32)).cuda()
        g.gradient(torch.from_numpy(rec).cuda(), scale=1.0 / n, grad=acc)
        np.testing.assert_allclose(acc.cpu().numpy(), 2 * gpu, rtol=1e-3, atol=1e-6 * np.abs(gpu).max())
    finally:
        g.close()
        s.close()


def test_train_step_is_gradient_plus_adam():
    import torch
    s, g = _guide(3, learning_rate=1e-3)
    try:
        p = _trained_like_params(g, 3)
        g.set_params(p)
        st = s.stats()
        n = 512
        rec = torch.from_numpy(_records(n, 4, np.array(st["bounds_min"]), np.array(st["bounds_max"]))).cuda()
        grad = g.gradient(rec, scale=1.0 / n).cpu().numpy()
        g.train_step(rec)
        after = g.params()
        z = np.zeros_like(p)
        expect, _, _ = G.adam(p, grad, z, z, 1, lr=1e-3)
        # the first Adam step is about lr * sign(gradient); summation order
        # differs between the two gradient evaluations, so compare where the
        # gradient is clearly non-zero, and bound the step elsewhere
        big = np.abs(grad) > 1e-4 * np.abs(grad).max()
        np.testing.assert_allclose(after[big], expect[big], rtol=0, atol=2e-6)
        assert np.abs(after - p).max() <= 1.01e-3
        assert np.abs(after - p).max() > 5e-4
    finally:
        g.close()
        s.close()


def test_training_lowers_the_loss_on_a_target_distribution():
    """Directions drawn from a position-dependent vMF lobe (mean pointing from
    the point to a fixed target); the guide learns to put its mass there."""
    import torch
    s, g = _guide(4, learning_rate=3e-3)
    try:
        rng = np.random.default_rng(5)
        st = s.stats()
        lo, hi = np.array(st["bounds_min"]), np.array(st["bounds_max"])
        target = np.array([0.0, 1.9, 0.0])

        def batch(n):
            rec = np.zeros((n, 10), np.float32)
            pos = rng.uniform(lo, hi, (n, 3))
            rec[:, :3] = pos
            rec[:, 3:6] = np.array([0, 1, 0])
            mean = _unit(target - pos)
            # vMF(kappa = 20) around mean (Wood's method via rejection-free w)
            kappa = 20.0
            u = rng.uniform(size=n)
            w = 1 + np.log(u + (1 - u) * math.exp(-2 * kappa)) / kappa
            phi = rng.uniform(0, 2 * math.pi, n)
            t = _unit(np.cross(mean, np.where(np.abs(mean[:, :1]) < 0.9, [[1, 0, 0]], [[0, 1, 0]])))
            b = np.cross(mean, t)
            sw = np.sqrt(np.maximum(0, 1 - w * w))[:, None]
            d = t * (sw * np.cos(phi)[:, None]) + b * (sw * np.sin(phi)[:, None]) + mean * w[:, None]
            rec[:, 6:9] = _unit(d)
            rec[:, 9] = 1.0
            return rec

        test = batch(4096)
        lt = torch.from_numpy(test).cuda()

        def mean_nll():
            out = g.forward(lt[:, :6]).cpu().numpy()
            return float(-G.log_pdf(out, test[:, 6:9]).mean())

        before = mean_nll()
        for _ in range(300):
            g.train_step(torch.from_numpy(batch(8192)).cuda())
        after = mean_nll()
        # uniform on the sphere: log(4 pi) = 2.53; the target lobe: about -1.6
        assert before > 2.0
        assert after < 0.5, (before, after)
    finally:
        g.close()
        s.close()
