"""CPU oracle of the surrogate MLP (test infrastructure only: the tests call it as the
checker of the GPU training kernels; nothing in the product path imports it).

The network has no counterpart in the reference; this is a plain numpy restatement of
the forward pass, the beta-weighted Gaussian negative log-likelihood and its gradient
with respect to every parameter, in the parameter layout of ucb_mlp_get_params (per
layer W[out][in] then b[out]; the last layer has 2 outputs: mean and log-variance).

With bf16=True it rounds to bfloat16 (round to nearest even) at the points where the GPU
kernels hand BF16 operands to the tensor cores: features, weights, hidden activations,
the output gradient and the pre-activation gradients; every product then accumulates in
float64 (the GPU accumulates in FP32 tensor memory). With bf16=False the arithmetic is
float64 throughout: the exact gradient, which finite differences pin.
"""
from __future__ import annotations

import numpy as np


def bf16_round(x) -> np.ndarray:
    """float32 -> nearest bfloat16 (ties to even), returned as float64."""
    f = np.ascontiguousarray(x, dtype=np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def layer_shapes(fourier: int, hidden: int, layers: int):
    shapes = []
    for l in range(layers + 1):
        i = 2 * fourier if l == 0 else hidden
        o = 2 if l == layers else hidden
        shapes.append((o, i))
    return shapes


def unpack(p, fourier, hidden, layers):
    out, off = [], 0
    for o, i in layer_shapes(fourier, hidden, layers):
        W = np.asarray(p[off:off + o * i], dtype=np.float64).reshape(o, i)
        off += o * i
        b = np.asarray(p[off:off + o], dtype=np.float64)
        off += o
        out.append((W, b))
    assert off == len(p)
    return out


C0, C1 = np.sqrt(2.0 / np.pi), 0.044715


def gelu(z):
    """GELU, tanh form (Hendrycks and Gimpel 2016), as the GPU kernels evaluate it."""
    return 0.5 * z * (1.0 + np.tanh(C0 * (z + C1 * z ** 3)))


def gelu_grad(z):
    t = np.tanh(C0 * (z + C1 * z ** 3))
    return 0.5 * (1.0 + t) + 0.5 * z * (1.0 - t * t) * C0 * (1.0 + 3.0 * C1 * z * z)


def features(u, B):
    ph = 2.0 * np.pi * (np.asarray(u, np.float64) @ np.asarray(B, np.float64).T)
    return np.concatenate([np.sin(ph), np.cos(ph)], axis=1)


def forward(p, B, u, hidden, layers, bf16=True):
    """Returns (out[n, 2], cache) for rows u[n, 2]."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    fourier = B.shape[0]
    params = unpack(p, fourier, hidden, layers)
    x = r(features(u, B))
    cache = {"x": [x], "z": []}
    for l in range(layers):
        W, b = params[l]
        z = x @ r(W).T + b
        x = r(gelu(z))
        cache["z"].append(z)
        cache["x"].append(x)
    W, b = params[layers]
    out = x @ r(W).T + b
    cache["params"] = params
    return out, cache


def loss_and_grad(p, B, u, y, hidden, layers, beta=0.5, y_mean=0.0, y_std=1.0, bf16=True):
    """Mean beta-NLL of the standardised targets and its gradient (flat, float64)."""
    r = bf16_round if bf16 else (lambda a: np.asarray(a, np.float64))
    n = len(y)
    out, c = forward(p, B, u, hidden, layers, bf16)
    ys = (np.asarray(y, np.float64) - y_mean) / y_std
    mu, lv_raw = out[:, 0], out[:, 1]
    lv = np.clip(lv_raw, -16.0, 16.0)
    iv = np.exp(-lv)
    d = mu - ys
    w = np.exp(beta * lv) if beta > 0 else np.ones_like(lv)
    loss = float(np.sum(w * 0.5 * (lv + d * d * iv)) / n)
    g0 = w * d * iv / n
    g1 = np.where(lv_raw == lv, w * 0.5 * (1.0 - d * d * iv) / n, 0.0)
    dout = r(np.stack([g0, g1], axis=1))
    params = c["params"]
    grads = [None] * (layers + 1)
    W, _ = params[layers]
    grads[layers] = (dout.T @ c["x"][layers], dout.sum(axis=0))
    dh = dout @ r(W)
    for l in range(layers - 1, -1, -1):
        dz = r(dh * gelu_grad(c["z"][l]))
        W, _ = params[l]
        grads[l] = (dz.T @ c["x"][l], dz.sum(axis=0))
        dh = dz @ r(W)
    flat = np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
    return loss, flat


def predict(p, B, u, hidden, layers, y_mean=0.0, y_std=1.0, bf16=True):
    out, _ = forward(p, B, u, hidden, layers, bf16)
    mean = out[:, 0] * y_std + y_mean
    sd = np.exp(0.5 * np.clip(out[:, 1], -16.0, 16.0)) * y_std
    return mean, sd
