"""CPU restatement of the learned-schedule MLP (test infrastructure only).

Forward, loss and gradients of the 48 -> 128 -> 128 -> 2 ReLU network with the GPU kernels'
rounding points: inputs, weights and both hidden activations rounded to BF16 (round to
nearest even); every product and sum here is exact-ish float64, where the GPU accumulates
in FP32.  Biases stay FP32.  Parameter layout (one f32 vector): W1 [128 x 48], b1 [128],
W2 [128 x 128], b2 [128], W3 [2 x 128], b3 [2].

Loss (mean over rows): (z0 - y0)^2 + BCE(sigmoid(z1), y1).
This oracle is itself pinned by central finite differences in the CPU test suite.
"""
from __future__ import annotations

import numpy as np

F, H, O = 48, 128, 2
SHAPES = [("W1", (H, F)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (O, H)), ("b3", (O,))]
N_PARAMS = sum(int(np.prod(s)) for _, s in SHAPES)


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest BF16 (ties to even) -> float32; finite inputs."""
    u = np.asarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32)


def unpack(params: np.ndarray) -> dict:
    p = np.asarray(params)
    p = p if p.dtype == np.float64 else p.astype(np.float32)
    assert p.size == N_PARAMS
    out, off = {}, 0
    for name, shape in SHAPES:
        n = int(np.prod(shape))
        out[name] = p[off:off + n].reshape(shape)
        off += n
    return out


def forward(params, x, rounding=True):
    """Returns z [n x 2] and the cached activations (xr, a1, a2).  rounding=False drops every
    BF16 rounding and keeps float64 (the smooth network the finite-difference check uses)."""
    w = unpack(params)
    if rounding:
        r, dt = bf16_round, np.float32
    else:
        r, dt = (lambda a: np.asarray(a, np.float64)), np.float64
    xr = r(np.asarray(x, np.float32))
    z1 = (np.asarray(xr, np.float64) @ np.asarray(r(w["W1"]), np.float64).T).astype(dt) + w["b1"]
    a1 = r(np.maximum(z1, 0.0).astype(dt))
    z2 = (np.asarray(a1, np.float64) @ np.asarray(r(w["W2"]), np.float64).T).astype(dt) + w["b2"]
    a2 = r(np.maximum(z2, 0.0).astype(dt))
    z = (np.asarray(a2, np.float64) @ np.asarray(r(w["W3"]), np.float64).T).astype(dt) + w["b3"]
    return z, (xr, a1, a2)


def loss_and_grad(params, x, y, rounding=True):
    """Mean loss and its gradient w.r.t. every parameter (straight through the BF16
    rounding of weights and activations, as the GPU backward kernels compute it)."""
    w = unpack(params)
    y = np.asarray(y, np.float64)
    r = bf16_round if rounding else (lambda a: np.asarray(a, np.float64))
    z, (xr, a1, a2) = forward(params, x, rounding)
    z = z.astype(np.float64)
    n = z.shape[0]
    s = 1.0 / (1.0 + np.exp(-z[:, 1]))
    loss = np.mean((z[:, 0] - y[:, 0]) ** 2 + np.maximum(z[:, 1], 0) - z[:, 1] * y[:, 1]
                   + np.log1p(np.exp(-np.abs(z[:, 1]))))
    dz = np.stack([2.0 * (z[:, 0] - y[:, 0]) / n, (s - y[:, 1]) / n], axis=1)
    a1d, a2d, xrd = a1.astype(np.float64), a2.astype(np.float64), xr.astype(np.float64)
    g = {}
    g["W3"] = dz.T @ a2d
    g["b3"] = dz.sum(0)
    dh2 = (dz @ np.asarray(r(w["W3"]), np.float64)) * (a2d > 0)
    g["W2"] = dh2.T @ a1d
    g["b2"] = dh2.sum(0)
    dh1 = (dh2 @ np.asarray(r(w["W2"]), np.float64)) * (a1d > 0)
    g["W1"] = dh1.T @ xrd
    g["b1"] = dh1.sum(0)
    flat = np.concatenate([g[name].reshape(-1) for name, _ in SHAPES])
    return float(loss), flat


def split(flat: np.ndarray) -> dict:
    out, off = {}, 0
    for name, shape in SHAPES:
        k = int(np.prod(shape))
        out[name] = np.asarray(flat[off:off + k])
        off += k
    return out
