"""CPU restatement of the learned path guide's network, for tests only.

TEST INFRASTRUCTURE: the guide has no counterpart in the reference renderer
(its non-learned analogue is the importon histogram of
xyz/core/photonmap.cpp:365-494), so this is the specification the CUDA
kernels (xyz_b200/csrc/guide.cu) are checked against: the one-blob encoding,
the MLP with the same bf16 rounding points (weights, inputs, hidden
activations, output deltas; float64 accumulation here instead of the tensor
cores' fp32), the von Mises-Fisher mixture and the gradient of the loss
-w * log p(direction).  Parameters use the C ABI's flat layout: for each layer
W_l as [in][64] row-major, then b_l[64].
"""

from __future__ import annotations

import math

import numpy as np

BINS = 32
N_IN = 6 * BINS
WIDTH = 64
LAYERS = 5
LOBES = 8
N_PARAMS = N_IN * WIDTH + WIDTH + 4 * (WIDTH * WIDTH + WIDTH)


def layer_in(l: int) -> int:
    return N_IN if l == 0 else WIDTH


def param_w(l: int) -> int:
    return 0 if l == 0 else (N_IN * WIDTH + WIDTH) + (l - 1) * (WIDTH * WIDTH + WIDTH)


def unpack(params):
    """Flat parameters -> [(W_l (in, 64), b_l (64,))]."""
    p = np.asarray(params, np.float32)
    out = []
    for l in range(LAYERS):
        k = layer_in(l)
        w = p[param_w(l): param_w(l) + k * WIDTH].reshape(k, WIDTH)
        b = p[param_w(l) + k * WIDTH: param_w(l) + k * WIDTH + WIDTH]
        out.append((w, b))
    return out


def bf16(x) -> np.ndarray:
    """Round float32 values to bfloat16 (nearest even), returned as float32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out)


def encode(features, lo, inv_ext) -> np.ndarray:
    """One-blob encoding of (position, normal) rows: 32 Gaussian bins
    (sigma 1/32) per input, bins beyond 4.5 sigma set to 0; positions
    normalised by the scene bounds."""
    f = np.asarray(features, np.float32)
    s = np.empty((f.shape[0], 6), np.float32)
    s[:, :3] = (f[:, :3] - np.asarray(lo, np.float32)) * np.asarray(inv_ext, np.float32)
    s[:, 3:] = (f[:, 3:] + np.float32(1.0)) * np.float32(0.5)
    s = np.clip(s, 0.0, 1.0).astype(np.float32)
    centres = ((np.arange(BINS, dtype=np.float32) + np.float32(0.5)) * np.float32(1.0 / BINS)).astype(np.float32)
    d = (s[:, :, None] - centres[None, None, :]).astype(np.float32)
    v = np.exp(-d * d * np.float32(0.5 * BINS * BINS)).astype(np.float32)
    # bins more than 4.5 sigma away are exactly 0
    u = (s * np.float32(BINS)).astype(np.float32)
    far = np.abs(u[:, :, None] - (np.arange(BINS, dtype=np.float32) + np.float32(0.5))[None, None, :]) > 4.5
    v[far] = 0.0
    return bf16(v.reshape(f.shape[0], N_IN))


def _round(x, rounding):
    return bf16(np.asarray(x, np.float32)).astype(np.float64) if rounding else np.asarray(x, np.float64)


def forward(params, x, rounding=True):
    """x: encoded (n, 192).  Returns (outputs (n, 64) float64, activations
    [x, h1..h4]); rounding: bf16 weights and activations as on the GPU (else
    plain float64, for checking the derivatives)."""
    acts = [np.asarray(x, np.float64)]
    a = acts[0]
    layers = unpack(params)
    for l, (w, b) in enumerate(layers):
        z = a @ _round(w, rounding) + b.astype(np.float64)
        if l == LAYERS - 1:
            return z, acts
        a = _round(np.maximum(z, 0.0), rounding)
        acts.append(a)
    raise AssertionError


def mixture(o):
    """Outputs -> (weights (n,8), kappa (n,8), means (n,8,3), kappa clamped mask)."""
    o = np.asarray(o, np.float64)
    logits = o[:, :LOBES]
    w = np.exp(logits - logits.max(axis=1, keepdims=True))
    w /= w.sum(axis=1, keepdims=True)
    lk = o[:, LOBES:2 * LOBES]
    clamped = (lk < -5.0) | (lk > 8.0)
    kappa = np.exp(np.clip(lk, -5.0, 8.0))
    mu = o[:, 16:40].reshape(-1, LOBES, 3)
    ln = np.sqrt((mu * mu).sum(axis=2, keepdims=True) + 1e-12)
    return w, kappa, mu / ln, clamped, ln[..., 0]


def log_pdf(o, d):
    """log p(d) of the mixture of outputs o at unit directions d."""
    w, k, mu, _, _ = mixture(o)
    dot = (mu * np.asarray(d, np.float64)[:, None, :]).sum(axis=2)
    logv = np.log(k) - math.log(2 * math.pi) - np.log(-np.expm1(-2 * k)) + k * (dot - 1)
    s = np.log(w) + logv
    m = s.max(axis=1, keepdims=True)
    return (m + np.log(np.exp(s - m).sum(axis=1, keepdims=True)))[:, 0]


def loss_grad(o, d, scale):
    """d(-scale * log p(d)) / d outputs, (n, 64); scale per row."""
    o = np.asarray(o, np.float64)
    d = np.asarray(d, np.float64)
    w, k, mu, clamped, ln = mixture(o)
    dot = (mu * d[:, None, :]).sum(axis=2)
    logv = np.log(k) - math.log(2 * math.pi) - np.log(-np.expm1(-2 * k)) + k * (dot - 1)
    s = np.log(w) + logv
    m = s.max(axis=1, keepdims=True)
    logp = m + np.log(np.exp(s - m).sum(axis=1, keepdims=True))
    r = np.exp(s - logp)
    g = np.zeros_like(o)
    sc = np.asarray(scale, np.float64).reshape(-1, 1)
    g[:, :LOBES] = -sc * (r - w)
    with np.errstate(over="ignore"):
        dlk = r * (1 - 2 * k / np.expm1(2 * k) + k * (dot - 1))
    g[:, LOBES:2 * LOBES] = -sc * np.where(clamped, 0.0, dlk)
    c = (r * k / ln)[..., None]
    g[:, 16:40] = (-sc[..., None] * c * (d[:, None, :] - dot[..., None] * mu)).reshape(-1, 24)
    return g


def loss(params, records, lo, inv_ext, scale, rounding=True):
    """scale * sum_i -w_i log p(d_i | x_i)."""
    rec = np.asarray(records, np.float32)
    o, _ = forward(params, encode(rec[:, :6], lo, inv_ext), rounding)
    return float(-(scale * rec[:, 9].astype(np.float64) * log_pdf(o, rec[:, 6:9])).sum())


def gradient(params, records, lo, inv_ext, scale, rounding=True):
    """Flat gradient of scale * sum_i -w_i log p(d_i | x_i), emulating the
    GPU's bf16 rounding of output and hidden deltas (unless rounding=False)."""
    rec = np.asarray(records, np.float32)
    x = encode(rec[:, :6], lo, inv_ext)
    o, acts = forward(params, x, rounding)
    wgt = rec[:, 9].astype(np.float64)
    g = loss_grad(o, rec[:, 6:9], wgt * scale)
    g[wgt == 0] = 0.0
    delta = _round(g, rounding)
    layers = unpack(params)
    out = np.zeros(N_PARAMS, np.float64)
    for l in range(LAYERS - 1, -1, -1):
        a = acts[l]
        kin = layer_in(l)
        out[param_w(l): param_w(l) + kin * WIDTH] = (a.T @ delta).reshape(-1)
        out[param_w(l) + kin * WIDTH: param_w(l) + kin * WIDTH + WIDTH] = delta.sum(axis=0)
        if l > 0:
            w = _round(layers[l][0], rounding)
            dprev = (delta @ w.T) * (acts[l] > 0)
            delta = _round(dprev, rounding)
    return out


def adam(params, grad, m, v, t, lr=1e-3, b1=0.9, b2=0.99, eps=1e-8):
    """One Adam step (float32, the update rule of the CUDA kernel)."""
    p = np.asarray(params, np.float32).copy()
    g = np.asarray(grad, np.float32)
    m = (np.float32(b1) * m + np.float32(1 - b1) * g).astype(np.float32)
    v = (np.float32(b2) * v + np.float32(1 - b2) * g * g).astype(np.float32)
    c1 = np.float32(1 - b1 ** t)
    c2 = np.float32(1 - b2 ** t)
    p = (p - np.float32(lr) * (m / c1) / (np.sqrt(v / c2) + np.float32(eps))).astype(np.float32)
    return p, m, v
