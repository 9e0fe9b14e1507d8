"""CPU oracle of the learned rank predictor -- TEST INFRASTRUCTURE ONLY.

The library's rank model (an MLP 8 -> 64 -> 64 -> 1 with ReLU, FP32) is
trained and evaluated by its own CUDA kernels.  This module restates the same
network in numpy (float64) so the tests can check the GPU forward pass, the
mean-squared-error gradient and the Adam update against it.  It has no
counterpart in hmat_lib (the reference has no learned component); it is
pinned by the finite-difference gradient check in tests/test_oracle.py.

Parameter layout (the same vector the library uses): feature mean[8], feature
scale[8], W1[8][64], b1[64], W2[64][64], b2[64], W3[64], b3.
"""
from __future__ import annotations

import numpy as np

IN, H = 8, 64
NORM = 2 * IN
W1 = NORM
B1 = W1 + IN * H
W2 = B1 + H
B2 = W2 + H * H
W3 = B2 + H
B3 = W3 + H
SIZE = B3 + 1


def unpack(p: np.ndarray):
    p = np.asarray(p, dtype=np.float64)
    return dict(mean=p[:IN], scale=p[IN:NORM], W1=p[W1:B1].reshape(IN, H), b1=p[B1:W2],
                W2=p[W2:B2].reshape(H, H), b2=p[B2:W3], W3=p[W3:B3], b3=p[B3])


def forward(p: np.ndarray, x: np.ndarray):
    """Outputs and the intermediate values of every sample (x: n x 8)."""
    q = unpack(p)
    xn = (np.asarray(x, dtype=np.float64) - q["mean"]) / q["scale"]
    a1 = xn @ q["W1"] + q["b1"]
    h1 = np.maximum(a1, 0.0)
    a2 = h1 @ q["W2"] + q["b2"]
    h2 = np.maximum(a2, 0.0)
    y = h2 @ q["W3"] + q["b3"]
    return y, dict(xn=xn, a1=a1, h1=h1, a2=a2, h2=h2)


def loss_and_gradient(p: np.ndarray, x: np.ndarray, t: np.ndarray):
    """Mean squared error and its gradient (normalisation entries zero)."""
    q = unpack(p)
    y, c = forward(p, x)
    n = len(y)
    e = y - np.asarray(t, dtype=np.float64)
    loss = float(np.mean(e * e))
    dy = 2.0 * e / n
    g = np.zeros(SIZE)
    g[B3] = dy.sum()
    g[W3:B3] = c["h2"].T @ dy
    d2 = (dy[:, None] * q["W3"][None, :]) * (c["a2"] > 0)
    g[B2:W3] = d2.sum(axis=0)
    g[W2:B2] = (c["h1"].T @ d2).reshape(-1)
    d1 = (d2 @ q["W2"].T) * (c["a1"] > 0)
    g[B1:W2] = d1.sum(axis=0)
    g[W1:B1] = (c["xn"].T @ d1).reshape(-1)
    return loss, g


def adam_step(p, g, m, v, step, lr, b1=0.9, b2=0.999, eps=1e-8):
    """One Adam update of the trainable entries (index NORM onwards)."""
    p, m, v = p.copy(), m.copy(), v.copy()
    s = slice(NORM, SIZE)
    m[s] = b1 * m[s] + (1 - b1) * g[s]
    v[s] = b2 * v[s] + (1 - b2) * g[s] ** 2
    mh = m[s] / (1 - b1 ** step)
    vh = v[s] / (1 - b2 ** step)
    p[s] = p[s] - lr * mh / (np.sqrt(vh) + eps)
    return p, m, v


def random_params(rng, x=None):
    """He-style random parameters; normalisation from x when given."""
    p = np.zeros(SIZE)
    if x is not None:
        p[:IN] = x.mean(axis=0)
        p[IN:NORM] = np.maximum(x.std(axis=0), 1e-3)
    else:
        p[IN:NORM] = 1.0
    p[W1:B1] = rng.standard_normal(IN * H) * np.sqrt(2.0 / IN)
    p[B1:W2] = rng.standard_normal(H) * 0.1
    p[W2:B2] = rng.standard_normal(H * H) * np.sqrt(2.0 / H)
    p[B2:W3] = rng.standard_normal(H) * 0.1
    p[W3:B3] = rng.standard_normal(H) * np.sqrt(1.0 / H)
    p[B3] = 0.3
    return p
