"""Seeded Poisson-disk sampling of snow shapes on the device (mpm_sample_shapes).

The reference fills each snowball with Bridson's sequential sampler seeded
from std::random_device (src/shared/Shapes.h:17-117 disk, 143-234 sphere),
so its particle sets differ run to run. Here the same minimum-distance
property comes from a grid-phase dart thrower on the GPU whose samples depend
on the seed alone; scenes.reference_snowballs rebuilds the reference's
default scene (src/shared/Parameters.h:42-53, particle init
src/gpu/GPUSolver.cpp:99-155) on top of it.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import SHAPE_BALL, SHAPE_BOX, MpmError, MpmShape, check, fptr, load

_ERR_CAPACITY = 11


def ball(center, radius) -> dict:
    return dict(kind=SHAPE_BALL, center=tuple(center), radius=float(radius), half=(0.0, 0.0, 0.0))


def box(center, half) -> dict:
    return dict(kind=SHAPE_BOX, center=tuple(center), radius=0.0, half=tuple(half))


def _pack(shapes):
    arr = (MpmShape * len(shapes))()
    for a, s in zip(arr, shapes):
        a.kind = int(s["kind"])
        c = list(s["center"]) + [0.0] * (3 - len(s["center"]))
        h = list(s.get("half", (0.0,) * 3)) + [0.0] * (3 - len(s.get("half", (0.0,) * 3)))
        for k in range(3):
            a.center[k] = float(c[k])
            a.half[k] = float(h[k])
        a.radius = float(s.get("radius", 0.0))
    return arr


def _capacity_bound(dim, shapes, min_dist):
    """Samples never outnumber the background cells that overlap a shape."""
    cell = min_dist / math.sqrt(dim)
    total = 0
    for s in shapes:
        ext = [2.0 * (s["radius"] if s["kind"] == SHAPE_BALL else s["half"][k]) for k in range(dim)]
        total += math.prod(int(e / cell) + 3 for e in ext)
    return total


def sample_shapes(dim: int, shapes, min_dist: float, seed: int, rounds: int = 30):
    """Samples at least `min_dist` apart filling the union of `shapes`.

    Returns (positions (n, dim) float32, shape index per sample int32), in the
    background grid's cell order. Raises MpmError on invalid input.
    """
    lib = load()
    arr = _pack(shapes)
    cap = _capacity_bound(dim, shapes, float(min_dist))
    for _ in range(2):
        pos = np.empty((cap, dim), np.float32)
        owner = np.empty(cap, np.int32)
        count = C.c_int64(0)
        st = lib.mpm_sample_shapes(dim, arr, len(shapes), float(min_dist), int(seed) & (2 ** 64 - 1), int(rounds),
                                   fptr(pos), owner.ctypes.data_as(C.POINTER(C.c_int32)), cap, C.byref(count))
        if st == _ERR_CAPACITY and count.value > cap:
            cap = count.value
            continue
        check(st)
        n = count.value
        return pos[:n].copy(), owner[:n].copy()
    raise MpmError(_ERR_CAPACITY, "sample count changed between calls")


__all__ = ["ball", "box", "sample_shapes", "SHAPE_BALL", "SHAPE_BOX"]
