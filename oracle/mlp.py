"""NumPy statement of the cost-model MLP (forward, masked-MSE loss, backward)
in float64: the CPU oracle the CUDA training kernels
(2024pra_conv_b200/csrc/mlp.cu) are checked against.

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).  The reference has no
learned component; this restates the project's own network: F inputs ->
64 ReLU -> 64 ReLU -> O outputs, parameters in one flat array
W1[64][F], b1[64], W2[64][64], b2[64], W3[O][64], b3[O], loss
L = sum m (y - t)^2 / sum m.
"""
from __future__ import annotations

import numpy as np

H = 64


def nparams(F, O):
    return H * F + H + H * H + H + O * H + O


def unpack(p, F, O):
    p = np.asarray(p, np.float64)
    i = 0
    out = []
    for shape in [(H, F), (H,), (H, H), (H,), (O, H), (O,)]:
        n = int(np.prod(shape))
        out.append(p[i:i + n].reshape(shape))
        i += n
    return out


def forward(p, x, F, O):
    W1, b1, W2, b2, W3, b3 = unpack(p, F, O)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    return h2 @ W3.T + b3, (z1, h1, z2, h2)


def loss_and_grad(p, x, t, m, F, O):
    x = np.asarray(x, np.float64)
    y, (z1, h1, z2, h2) = forward(p, x, F, O)
    W1, b1, W2, b2, W3, b3 = unpack(p, F, O)
    cnt = float(np.sum(m))
    d = y - t
    loss = float(np.sum(m * d * d) / cnt)
    dy = 2.0 * m * d / cnt
    gW3 = dy.T @ h2
    gb3 = dy.sum(0)
    dz2 = (dy @ W3) * (z2 > 0)
    gW2 = dz2.T @ h1
    gb2 = dz2.sum(0)
    dz1 = (dz2 @ W2) * (z1 > 0)
    gW1 = dz1.T @ x
    gb1 = dz1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3])
    return loss, g


def init_params(F, O, seed=0):
    """He-style initialisation (the same one the CUDA trainer starts from)."""
    rng = np.random.default_rng(seed)
    parts = [rng.standard_normal((H, F)) * np.sqrt(2.0 / F), np.zeros(H),
             rng.standard_normal((H, H)) * np.sqrt(2.0 / H), np.zeros(H),
             rng.standard_normal((O, H)) * np.sqrt(1.0 / H), np.zeros(O)]
    return np.concatenate([a.ravel() for a in parts]).astype(np.float32)
