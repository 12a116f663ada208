"""FP64 CPU oracle of the planner's cost MLP (24 -> 64 -> 64 -> 2, ReLU).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA forward/backward/Adam kernels
(mordred_b200/csrc/mlp.cu), never the product. Parameter layout as the library's:
W1[24][64], b1[64], W2[64][64], b2[64], W3[64][2], b3[2] in one flat array. The loss is
1/(2B) * sum over the batch and both outputs of (y - t)^2. The reference has no learned
planner (it plans with src/gpudb/CostModel.cu), so this oracle is pinned by finite
differences of its own loss (tests/test_mlp.py), not by reference vectors.
"""
from __future__ import annotations

import numpy as np

IN, HID, OUT = 24, 64, 2
SHAPES = [("W1", (IN, HID)), ("b1", (HID,)), ("W2", (HID, HID)), ("b2", (HID,)), ("W3", (HID, OUT)), ("b3", (OUT,))]
NPARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def unpack(p: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = np.asarray(p[off: off + n], np.float64).reshape(shape)
        off += n
    return out


def forward(p: np.ndarray, x: np.ndarray):
    w = unpack(p)
    x = np.asarray(x, np.float64)
    a1 = x @ w["W1"] + w["b1"]
    h1 = np.maximum(a1, 0)
    a2 = h1 @ w["W2"] + w["b2"]
    h2 = np.maximum(a2, 0)
    y = h2 @ w["W3"] + w["b3"]
    return y, (x, a1, h1, a2, h2)


def loss(p, x, t) -> float:
    y, _ = forward(p, x)
    return 0.5 * float(((y - np.asarray(t, np.float64)) ** 2).sum()) / len(x)


def grad(p, x, t) -> np.ndarray:
    w = unpack(p)
    y, (x, a1, h1, a2, h2) = forward(p, x)
    dy = (y - np.asarray(t, np.float64)) / len(x)
    gW3 = h2.T @ dy
    gb3 = dy.sum(0)
    d2 = (dy @ w["W3"].T) * (a2 > 0)
    gW2 = h1.T @ d2
    gb2 = d2.sum(0)
    d1 = (d2 @ w["W2"].T) * (a1 > 0)
    gW1 = x.T @ d1
    gb1 = d1.sum(0)
    return np.concatenate([g.reshape(-1) for g in (gW1, gb1, gW2, gb2, gW3, gb3)])


def adam(p, g, m, v, step, lr, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0):
    """One Adam step in float64; returns new (p, m, v)."""
    g = np.asarray(g, np.float64) + weight_decay * np.asarray(p, np.float64)
    m = beta1 * m + (1 - beta1) * g
    v = beta2 * v + (1 - beta2) * g * g
    mh = m / (1 - beta1 ** step)
    vh = v / (1 - beta2 ** step)
    return p - lr * mh / (np.sqrt(vh) + eps), m, v
