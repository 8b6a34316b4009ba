"""CPU oracle of the exchange-energy surrogate network (test infrastructure only).

Mirrors the GPU network of the control variate: y = w3 . gelu(W2 gelu(W1 x + b1) + b2) + b3
with exact-erf GELU, weights rounded to bfloat16 (round to nearest even) in the products,
biases in full precision, loss L = 1/(2B) sum (y - t)^2, Adam(0.9, 0.999, 1e-8).
Everything here is float64, so it checks the GPU's fp32 gradients to ~1e-5."""
from __future__ import annotations

import numpy as np
from scipy.special import erf


def bf16(x: np.ndarray) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even) -> float64."""
    a = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    lsb = (a >> 16) & 1
    r = ((a + 0x7FFF + lsb) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def layout(nin: int, H: int):
    o = {}
    o["W1"] = (0, H * nin)
    o["b1"] = (o["W1"][1], o["W1"][1] + H)
    o["W2"] = (o["b1"][1], o["b1"][1] + H * H)
    o["b2"] = (o["W2"][1], o["W2"][1] + H)
    o["w3"] = (o["b2"][1], o["b2"][1] + H)
    o["b3"] = (o["w3"][1], o["w3"][1] + 1)
    return o


def unpack(p: np.ndarray, nin: int, H: int, round_weights: bool = True):
    o = layout(nin, H)
    g = {k: p[a:b] for k, (a, b) in o.items()}
    q = bf16 if round_weights else (lambda v: np.asarray(v, np.float64))
    return (q(g["W1"]).reshape(H, nin), g["b1"].astype(np.float64),
            q(g["W2"]).reshape(H, H), g["b2"].astype(np.float64), q(g["w3"]),
            float(g["b3"][0]))


def gelu(z):
    return 0.5 * z * (1.0 + erf(z / np.sqrt(2.0)))


def gelu_d(z):
    return 0.5 * (1.0 + erf(z / np.sqrt(2.0))) + z * np.exp(-0.5 * z * z) / np.sqrt(2.0 * np.pi)


def forward(p, x, nin, H, round_weights: bool = True):
    W1, b1, W2, b2, w3, b3 = unpack(p, nin, H, round_weights)
    x = np.asarray(x, np.float64)
    z1 = x @ W1.T + b1
    h1 = gelu(z1)
    z2 = h1 @ W2.T + b2
    h2 = gelu(z2)
    return h2 @ w3 + b3, (x, z1, h1, z2, h2)


def gradient(p, x, t, nin, H, round_weights: bool = True):
    W1, b1, W2, b2, w3, b3 = unpack(p, nin, H, round_weights)
    y, (x, z1, h1, z2, h2) = forward(p, x, nin, H, round_weights)
    B = x.shape[0]
    r = y - np.asarray(t, np.float64)
    loss = 0.5 * np.mean(r * r)
    dy = r / B
    dz2 = dy[:, None] * w3[None, :] * gelu_d(z2)
    dz1 = (dz2 @ W2) * gelu_d(z1)
    g = np.concatenate([(dz1.T @ x).ravel(), dz1.sum(0), (dz2.T @ h1).ravel(), dz2.sum(0),
                        h2.T @ dy, [dy.sum()]])
    return g, loss
