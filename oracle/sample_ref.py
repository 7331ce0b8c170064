"""TEST INFRASTRUCTURE — CPU restatement of the device Poisson-disk sampler.

Only tests/ use this module. It restates mpm_sample_shapes
(mpm_snow_sim2d_b200/csrc/mpm_sample.cu) step for step in numpy float32 with
the same counter-based hash, so its samples equal the device's bit for bit:
background cells of side min_dist / sqrt(dim), phases of cells equal modulo 3,
one candidate per empty live cell per round, acceptance when inside a shape
and no sample of the 5^dim neighbouring cells is closer than min_dist.
"""
from __future__ import annotations

import numpy as np

F = np.float32
U = np.uint64
BALL, BOX = 0, 1


def _mix64(z):
    with np.errstate(over="ignore"):
        z = z + U(0x9E3779B97F4A7C15)
        z = (z ^ (z >> U(30))) * U(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> U(27))) * U(0x94D049BB133111EB)
        return z ^ (z >> U(31))


def _uniform(seed, cell, rnd, axis):
    with np.errstate(over="ignore"):
        inner = cell.astype(U) * U(4) + U(axis) + (U(rnd) << U(40))
        h = _mix64(U(seed) ^ _mix64(inner))
    return (h >> U(40)).astype(F) * F(1.0 / 16777216.0)


def sample_shapes(dim, shapes, min_dist, seed, rounds=30):
    """shapes: list of dicts (kind, center[3], radius, half[3]); returns
    (positions (n, dim) float32 in cell order, shape index per sample)."""
    md = F(min_dist)
    cell = F(md / np.sqrt(F(dim)))
    lo = [None] * 3
    hi = [None] * 3
    for s in shapes:
        for k in range(dim):
            e = F(s["radius"]) if s["kind"] == BALL else F(s["half"][k])
            a, b = F(F(s["center"][k]) - e), F(F(s["center"][k]) + e)
            lo[k] = a if lo[k] is None else min(lo[k], a)
            hi[k] = b if hi[k] is None else max(hi[k], b)
    nc = [max(1, int(np.ceil(F(F(hi[k] - lo[k]) / cell))) + 1) if k < dim else 1 for k in range(3)]
    origin = [lo[k] if k < dim else F(0) for k in range(3)]
    ncells = nc[0] * nc[1] * nc[2]
    ids = np.arange(ncells, dtype=np.int64)
    ic = [ids % nc[0], (ids // nc[0]) % nc[1], ids // (nc[0] * nc[1])]
    # live cells: overlap a shape's bounding box
    live = np.zeros(ncells, bool)
    for s in shapes:
        ok = np.ones(ncells, bool)
        for k in range(dim):
            clo = F(origin[k]) + ic[k].astype(F) * cell
            chi = clo + cell
            e = F(s["radius"]) if s["kind"] == BALL else F(s["half"][k])
            ok &= (chi >= F(F(s["center"][k]) - e)) & (clo <= F(F(s["center"][k]) + e))
        live |= ok
    pts = np.zeros((ncells, 3), F)
    has = np.zeros(ncells, bool)
    r2 = F(md * md)
    for rnd in range(rounds):
        for pz in range(3 if dim == 3 else 1):
            for py in range(3):
                for px in range(3):
                    sel = (ic[0] % 3 == px) & (ic[1] % 3 == py) & ((ic[2] % 3 == pz) if dim == 3 else True)
                    cand = ids[sel & live & ~has]
                    if cand.size == 0:
                        continue
                    p = np.zeros((cand.size, 3), F)
                    for k in range(dim):
                        u = _uniform(seed, cand, rnd, k)
                        p[:, k] = F(origin[k]) + (ic[k][cand].astype(F) + u) * cell
                    inside = np.zeros(cand.size, bool)
                    for s in shapes:
                        if s["kind"] == BALL:
                            d2 = np.zeros(cand.size, F)
                            for k in range(dim):
                                d = p[:, k] - F(s["center"][k])
                                d2 = d2 + d * d
                            inside |= d2 <= F(F(s["radius"]) * F(s["radius"]))
                        else:
                            ok = np.ones(cand.size, bool)
                            for k in range(dim):
                                ok &= np.abs(p[:, k] - F(s["center"][k])) <= F(s["half"][k])
                            inside |= ok
                    keep = inside.copy()
                    cx, cy, cz = ic[0][cand], ic[1][cand], ic[2][cand]
                    zr = 2 if dim == 3 else 0
                    for dz in range(-zr, zr + 1):
                        for dy in range(-2, 3):
                            for dx in range(-2, 3):
                                jx, jy, jz = cx + dx, cy + dy, cz + dz
                                ok = (jx >= 0) & (jy >= 0) & (jz >= 0) & (jx < nc[0]) & (jy < nc[1]) & (jz < nc[2])
                                j = np.where(ok, (jz * nc[1] + jy) * nc[0] + jx, 0)
                                nb = ok & has[j]
                                q = pts[j]
                                ddx, ddy, ddz = q[:, 0] - p[:, 0], q[:, 1] - p[:, 1], q[:, 2] - p[:, 2]
                                close = ((ddx * ddx + ddy * ddy) + ddz * ddz) < r2
                                keep &= ~(nb & close)
                    acc = cand[keep]
                    pts[acc] = p[keep]
                    has[acc] = True
    out = pts[has][:, :dim]
    owner = np.full(out.shape[0], -1, np.int32)
    for i_s in range(len(shapes) - 1, -1, -1):  # the first containing shape wins
        s = shapes[i_s]
        if s["kind"] == BALL:
            d2 = np.zeros(out.shape[0], F)
            for k in range(dim):
                d = out[:, k] - F(s["center"][k])
                d2 = d2 + d * d
            owner[d2 <= F(F(s["radius"]) * F(s["radius"]))] = i_s
        else:
            ok = np.ones(out.shape[0], bool)
            for k in range(dim):
                ok &= np.abs(out[:, k] - F(s["center"][k])) <= F(s["half"][k])
            owner[ok] = i_s
    return out, owner
