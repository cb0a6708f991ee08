"""FP64 oracle of the warm-start MLP (test infrastructure, not product code).

The network (8 -> 32 -> 32 -> 1, SiLU) and its loss 1/(2n) sum (y - t)^2 restated in
numpy, forward and backward, in FP64. With ``bf16=True`` the operands are rounded to
bfloat16 at the same points as the tensor-core kernels (inputs, weights, the hidden
activations fed to the next layer, the pre-activation gradients fed to the weight-
gradient and back-propagation products); every sum is then exact-ish FP64, so the
GPU's FP32-accumulated results differ only by accumulation rounding. With
``bf16=False`` it is the plain FP64 model, checked against central finite differences.

Parameter vector layout (1377 floats): W1[8][32], b1[32], W2[32][32], b2[32], W3[32], b3.
"""
from __future__ import annotations

import numpy as np

N_PARAMS = 1377
OFF = {"W1": 0, "b1": 256, "W2": 288, "b2": 1312, "W3": 1344, "b3": 1376}


def bf16(x):
    """Round to the nearest bfloat16 (ties to even), returned as float64."""
    f = np.asarray(x, np.float32)
    b = f.view(np.uint32).astype(np.uint64)
    rounded = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return (rounded.astype(np.uint32) << 16).view(np.float32).astype(np.float64)


def unpack(w):
    w = np.asarray(w, np.float64)
    return (w[0:256].reshape(8, 32), w[256:288], w[288:1312].reshape(32, 32), w[1312:1344], w[1344:1376], w[1376])


def _sig(z):
    return 1.0 / (1.0 + np.exp(-z))


def silu(z):
    return z * _sig(z)


def silu_grad(z):
    s = _sig(z)
    return s * (1.0 + z * (1.0 - s))


def forward(w, x, bf16_points=True):
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(w)
    xb = r(x)
    z1 = xb @ r(W1) + b1
    h1 = r(silu(z1))
    z2 = h1 @ r(W2) + b2
    h2 = r(silu(z2))
    y = h2 @ r(W3) + b3
    return y, (xb, z1, h1, z2, h2)


def loss_and_grad(w, x, t, bf16_points=True):
    r = bf16 if bf16_points else (lambda a: np.asarray(a, np.float64))
    W1, b1, W2, b2, W3, b3 = unpack(w)
    n = x.shape[0]
    y, (xb, z1, h1, z2, h2) = forward(w, x, bf16_points)
    t = np.asarray(t, np.float64)
    loss = 0.5 * np.sum((y - t) ** 2) / n
    dy = (y - t) / n
    g = np.zeros(N_PARAMS)
    g[OFF["W3"]:OFF["W3"] + 32] = h2.T @ dy
    g[OFF["b3"]] = dy.sum()
    dz2 = np.outer(dy, r(W3)) * silu_grad(z2)
    g[OFF["b2"]:OFF["b2"] + 32] = dz2.sum(0)
    dz2b = r(dz2)
    g[OFF["W2"]:OFF["W2"] + 1024] = (h1.T @ dz2b).ravel()
    dh1 = dz2b @ r(W2).T
    dz1 = dh1 * silu_grad(z1)
    g[OFF["b1"]:OFF["b1"] + 32] = dz1.sum(0)
    g[OFF["W1"]:OFF["W1"] + 256] = (xb.T @ r(dz1)).ravel()
    return loss, g


def finite_difference(w, x, t, eps=1e-6, params=None):
    """Central differences of the plain FP64 loss for the given parameter indices."""
    w = np.asarray(w, np.float64)
    idx = range(N_PARAMS) if params is None else params
    out = {}
    for p in idx:
        wp = w.copy()
        wp[p] += eps
        wm = w.copy()
        wm[p] -= eps
        lp, _ = loss_and_grad(wp, x, t, bf16_points=False)
        lm, _ = loss_and_grad(wm, x, t, bf16_points=False)
        out[p] = (lp - lm) / (2 * eps)
    return out


def init(seed=0):
    """Xavier-uniform weights, zero biases, output layer scaled by 0.1 (same scheme as the
    library's lsp_mlp_reset, different generator)."""
    rng = np.random.default_rng(seed)
    w = np.zeros(N_PARAMS)
    for name, fi, fo, sc in (("W1", 8, 32, 1.0), ("W2", 32, 32, 1.0), ("W3", 32, 1, 0.1)):
        a = sc * np.sqrt(6.0 / (fi + fo))
        w[OFF[name]:OFF[name] + fi * fo] = rng.uniform(-a, a, fi * fo)
    return w
