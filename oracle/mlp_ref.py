"""TEST INFRASTRUCTURE — CPU reference of the learned plasticity surrogate.

Only tests/ use this module. It restates the network of
mpm_snow_sim2d_b200/csrc/mpm_mlp.cuh in numpy (FP64 arithmetic):
10 -> 64 -> 64 -> 64 -> 10, GELU (tanh form), mean over samples of the summed
squared error on the normalised outputs, and its exact gradient by backprop.
With ``bf16=True`` values are rounded to bfloat16 (round to nearest even) at
the points where the GPU kernels store bfloat16: network inputs, weights,
hidden activations and the back-propagated pre-activation gradients; the
gradient check then isolates accumulation order and the hardware tanh.
"""
from __future__ import annotations

import math

import numpy as np

from mpm_snow_sim2d_b200.mlp import HID, OFF, features, targets

def bf16(a: np.ndarray) -> np.ndarray:
    """Round float values to bfloat16 (nearest even), returned as float64."""
    f = np.ascontiguousarray(a, np.float32)
    u = f.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


_C = math.sqrt(2.0 / math.pi)
_A = 0.044715


def gelu(x):
    """GELU, tanh form (the kernels' activation)."""
    return 0.5 * x * (1.0 + np.tanh(_C * (x + _A * x ** 3)))


def gelu_grad(x):
    th = np.tanh(_C * (x + _A * x ** 3))
    return 0.5 * (1.0 + th) + 0.5 * x * (1.0 - th * th) * _C * (1.0 + 3.0 * _A * x * x)


def unpack(params: np.ndarray):
    p = np.asarray(params, np.float64)

    def get(name, shape):
        o, n = OFF[name]
        return p[o:o + n].reshape(shape)
    return [(get("W1", (HID, 16)), get("b1", (HID,))), (get("W2", (HID, HID)), get("b2", (HID,))),
            (get("W3", (HID, HID)), get("b3", (HID,))), (get("W4", (16, HID)), get("b4", (16,)))]


def loss_and_grad(params, pairs, norm, bf16_emulation=True):
    """Loss (mean over rows of the summed squared error) and its gradient."""
    in_mean, in_std, out_mean, out_std = (np.asarray(a, np.float64) for a in norm)
    r = (lambda a: bf16(a)) if bf16_emulation else (lambda a: np.asarray(a, np.float64))
    n = pairs.shape[0]
    x = np.zeros((n, 16))
    x[:, :10] = (features(pairs.astype(np.float32).astype(np.float64)) - in_mean) / in_std
    t = np.zeros((n, 16))
    t[:, :10] = (targets(pairs.astype(np.float64)) - out_mean) / out_std
    layers = unpack(params)
    Ws = [r(W) for W, _ in layers]
    bs = [b for _, b in layers]
    h = [r(x)]
    ys = []
    for l in range(4):
        y = h[-1] @ Ws[l].T + bs[l]
        ys.append(y)
        if l < 3:
            h.append(r(gelu(y)))
    out = ys[3]
    diff = out - t
    diff[:, 10:] = 0.0
    loss = float((diff ** 2).sum() / n)
    grads = [None] * 4
    dy = 2.0 * diff / n
    dy_fp = dy.copy()
    dy = r(dy)
    for l in range(3, -1, -1):
        dW = dy.T @ h[l]
        db = (dy_fp if l == 3 else dy).sum(0)
        grads[l] = (dW, db)
        if l == 0:
            break
        dh = dy @ Ws[l]
        dy = r(dh * gelu_grad(ys[l - 1]))
    g = np.zeros(OFF["b4"][0] + OFF["b4"][1])
    for l, (name_w, name_b) in enumerate((("W1", "b1"), ("W2", "b2"), ("W3", "b3"), ("W4", "b4"))):
        o, sz = OFF[name_w]
        g[o:o + sz] = grads[l][0].ravel()
        o, sz = OFF[name_b]
        g[o:o + sz] = grads[l][1]
    return loss, g


def forward(params, rows, norm, bf16_emulation=True):
    """Denormalised network outputs (F_E' - F_hat, log J_p' - log J_p) for rows
    whose first 10 values are F_hat[9], J_p: the quantity mpm_mlp_predict and
    mpm_mlp_predict_noalloc return. Returns (outputs, normalised outputs)."""
    in_mean, in_std, out_mean, out_std = (np.asarray(a, np.float64) for a in norm)
    r = (lambda a: bf16(a)) if bf16_emulation else (lambda a: np.asarray(a, np.float64))
    rows = np.asarray(rows, np.float32)
    n = rows.shape[0]
    pairs = np.zeros((n, 20), np.float64)
    pairs[:, :10] = rows[:, :10]
    x = np.zeros((n, 16))
    x[:, :10] = (features(pairs) - in_mean) / in_std
    h = r(x)
    layers = unpack(params)
    for l, (W, b) in enumerate(layers):
        y = h @ r(W).T + b
        h = r(gelu(y)) if l < 3 else y
    out_n = h[:, :10]
    return out_n * out_std + out_mean, out_n
