"""FP64 CPU restatement of the neighbour-radius network of
sapporo2_b200/csrc/sapb_mlp.cu (5 -> 64 -> 64 -> 64 -> 1, ReLU hidden layers,
loss 1/(2n) sum (y - t)^2) and of its gradient.

TEST INFRASTRUCTURE ONLY: the checker of the GPU forward/backward kernels.
Its own gradient is pinned by central finite differences in the tests.
"""
from __future__ import annotations

import numpy as np

IN, H = 5, 64
SHAPES = [("W1", (H, IN)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
          ("b3", (H,)), ("W4", (H,)), ("b4", (1,))]
NP = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    out, k = {}, 0
    for name, shp in SHAPES:
        n = int(np.prod(shp))
        out[name] = p[k:k + n].reshape(shp)
        k += n
    return out


def forward(p, x):
    w = unpack(p)
    x = np.asarray(x, dtype=np.float64)
    z1 = x @ w["W1"].T + w["b1"]
    h1 = np.maximum(z1, 0)
    z2 = h1 @ w["W2"].T + w["b2"]
    h2 = np.maximum(z2, 0)
    z3 = h2 @ w["W3"].T + w["b3"]
    h3 = np.maximum(z3, 0)
    y = h3 @ w["W4"] + w["b4"][0]
    return y, (x, z1, h1, z2, h2, z3, h3)


def loss(p, x, t):
    y, _ = forward(p, x)
    return 0.5 * np.mean((y - np.asarray(t, dtype=np.float64)) ** 2)


def gradient(p, x, t):
    """Gradient of `loss` with respect to the packed parameters."""
    w = unpack(p)
    y, (x, z1, h1, z2, h2, z3, h3) = forward(p, x)
    n = len(y)
    dy = (y - np.asarray(t, dtype=np.float64)) / n
    g = {"W4": h3.T @ dy, "b4": np.array([dy.sum()])}
    d3 = np.outer(dy, w["W4"]) * (z3 > 0)
    g["W3"], g["b3"] = d3.T @ h2, d3.sum(0)
    d2 = (d3 @ w["W3"]) * (z2 > 0)
    g["W2"], g["b2"] = d2.T @ h1, d2.sum(0)
    d1 = (d2 @ w["W2"]) * (z1 > 0)
    g["W1"], g["b1"] = d1.T @ x, d1.sum(0)
    return np.concatenate([g[name].ravel() for name, _ in SHAPES])
