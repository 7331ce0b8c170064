"""Learned plasticity surrogate: Python handle over the C ABI (mpm_mlp_*).

The network (10 -> 64 -> 64 -> 64 -> 10, GELU, BF16 weights and activations,
FP32 accumulation on the tensor cores) maps a particle's trial elastic gradient
and plastic volume ratio to the return map's correction. Training runs on the
GPU in the library's own kernels (forward, backward, AdamW); this module only
moves arrays and calls them.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib
from ._lib import check, fptr

N_IN = N_OUT = 10
HID = 64
# parameter block offsets (row-major W[out][in], padded to 16 inputs / outputs)
OFF = {}
_o = 0
for _name, _size in (("W1", HID * 16), ("b1", HID), ("W2", HID * HID), ("b2", HID), ("W3", HID * HID), ("b3", HID),
                     ("W4", 16 * HID), ("b4", 16)):
    OFF[_name] = (_o, _size)
    _o += _size
N_PARAMS = _o


def features(pairs: np.ndarray) -> np.ndarray:
    """Raw network inputs (F_hat - I, log J_p) of pair rows (n, 20)."""
    f = np.empty((pairs.shape[0], 10), np.float64)
    f[:, :9] = pairs[:, :9] - np.eye(3).ravel()
    f[:, 9] = np.log(pairs[:, 9])
    return f


def targets(pairs: np.ndarray) -> np.ndarray:
    """Raw network outputs (F_E' - F_hat, log J_p' - log J_p) of pair rows."""
    t = np.empty((pairs.shape[0], 10), np.float64)
    t[:, :9] = pairs[:, 10:19] - pairs[:, :9]
    t[:, 9] = np.log(pairs[:, 19]) - np.log(pairs[:, 9])
    return t


def normalization(pairs: np.ndarray):
    """Per-feature mean and std of inputs and outputs (std floored at 1e-6)."""
    x, y = features(pairs), targets(pairs)
    return (x.mean(0).astype(np.float32), np.maximum(x.std(0), 1e-6).astype(np.float32),
            y.mean(0).astype(np.float32), np.maximum(y.std(0), 1e-6).astype(np.float32))


class Mlp:
    def __init__(self, seed: int = 0):
        self._lib = _lib.load()
        h = C.c_void_p()
        check(self._lib.mpm_mlp_create(int(seed), C.byref(h)))
        self._h = h
        self.norm = None

    def params(self) -> np.ndarray:
        out = np.empty(N_PARAMS, np.float32)
        check(self._lib.mpm_mlp_get_params(self._h, fptr(out), out.size))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        check(self._lib.mpm_mlp_set_params(self._h, fptr(p), p.size))

    def set_normalization(self, in_mean, in_std, out_mean, out_std) -> None:
        arrs = [np.ascontiguousarray(a, np.float32) for a in (in_mean, in_std, out_mean, out_std)]
        check(self._lib.mpm_mlp_set_normalization(self._h, *[fptr(a) for a in arrs]))
        self.norm = tuple(a.copy() for a in arrs)

    def load_pairs(self, pairs: np.ndarray) -> None:
        p = np.ascontiguousarray(pairs, np.float32)
        check(self._lib.mpm_mlp_load_pairs(self._h, fptr(p), p.shape[0]))

    def train(self, steps: int, batch: int = 8192, lr: float = 2e-3, weight_decay: float = 1e-4,
              seed: int = 1) -> np.ndarray:
        loss = np.empty(max(steps, 1), np.float32)
        check(self._lib.mpm_mlp_train(self._h, int(steps), int(batch), float(lr), float(weight_decay), int(seed),
                                      fptr(loss)))
        return loss[:steps] / batch

    def gradient(self, pairs: np.ndarray):
        p = np.ascontiguousarray(pairs, np.float32)
        g = np.empty(N_PARAMS, np.float32)
        l = C.c_float()
        check(self._lib.mpm_mlp_gradient(self._h, fptr(p), p.shape[0], fptr(g), C.byref(l)))
        return g, float(l.value) / p.shape[0]

    def predict(self, rows: np.ndarray) -> np.ndarray:
        r = np.ascontiguousarray(rows, np.float32)
        out = np.empty((r.shape[0], 10), np.float32)
        check(self._lib.mpm_mlp_predict(self._h, fptr(r), r.shape[0], r.shape[1], fptr(out)))
        return out

    def save(self, path) -> None:
        np.savez(path, params=self.params(), in_mean=self.norm[0], in_std=self.norm[1], out_mean=self.norm[2],
                 out_std=self.norm[3])

    @classmethod
    def load(cls, path) -> "Mlp":
        z = np.load(path)
        m = cls()
        m.set_params(z["params"])
        m.set_normalization(z["in_mean"], z["in_std"], z["out_mean"], z["out_std"])
        return m

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mpm_mlp_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# Trained on exact return-map pairs of snowball-on-slab impacts (64^3, speeds
# 1-8 m/s): the weights for impacts.
DEFAULT_WEIGHTS = Path(__file__).resolve().parent / "data" / "mlp_snow_3d.npz"
# Trained on 30M impact pairs plus 20M pairs of two snowballs colliding (256^3,
# radii 0.12-0.16, relative speeds 1-8 m/s, seeds apart from the two-snowball
# workload's): the weights for collisions. On the unseen impact of the tests
# they keep F within 1.9e-3 after 300 steps against 7.4e-4 for DEFAULT_WEIGHTS.
MIXED_WEIGHTS = Path(__file__).resolve().parent / "data" / "mlp_snow_3d_mixed.npz"
