"""CPU oracle for the reluctivity-predictor MLP (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in the reference; this restates the GPU
kernels' mathematics in float64 with BF16 rounding applied at exactly the
points where the kernels round (every tensor-core GEMM input): a 4 -> 64 -> 64
-> 64 -> 1 SiLU MLP, parameters packed as W1[64][4] b1 W2[64][64] b2 W3[64][64]
b3 w4[64] b4, loss L = sum_i s/2 (y_i - t_i)^2.
"""
from __future__ import annotations

import numpy as np

H = 64
NPARAMS = H * 4 + H + H * H + H + H * H + H + H + 1


def bf16(x):
    """Round to bfloat16 (round to nearest even), returned as float64."""
    f = np.asarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    p = np.asarray(p, dtype=np.float64)
    o = 0
    out = {}
    for name, shape in (("W1", (H, 4)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (H, H)),
                        ("b3", (H,)), ("w4", (H,)), ("b4", (1,))):
        n = int(np.prod(shape))
        out[name] = p[o:o + n].reshape(shape)
        o += n
    return out


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward(p, x):
    P = unpack(p)
    xb = bf16(x)
    z1 = xb @ bf16(P["W1"]).T + P["b1"]
    h1b = bf16(silu(z1))
    z2 = h1b @ bf16(P["W2"]).T + P["b2"]
    h2b = bf16(silu(z2))
    z3 = h2b @ bf16(P["W3"]).T + P["b3"]
    y = silu(z3) @ P["w4"] + P["b4"][0]
    return y, (xb, z1, h1b, z2, h2b, z3)


def gradient(p, x, t, loss_scale):
    P = unpack(p)
    y, (xb, z1, h1b, z2, h2b, z3) = forward(p, x)
    dy = (y - t) * loss_scale
    g = {}
    g["w4"] = silu(z3).T @ dy
    g["b4"] = np.array([dy.sum()])
    dz3 = dy[:, None] * P["w4"][None, :] * dsilu(z3)
    g["W3"] = dz3.T @ h2b
    g["b3"] = dz3.sum(0)
    dz2 = (bf16(dz3) @ bf16(P["W3"])) * dsilu(z2)
    g["W2"] = dz2.T @ h1b
    g["b2"] = dz2.sum(0)
    dz1 = (bf16(dz2) @ bf16(P["W2"])) * dsilu(z1)
    g["W1"] = dz1.T @ xb
    g["b1"] = dz1.sum(0)
    flat = np.concatenate([g[k].ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3", "w4", "b4")])
    return y, flat
