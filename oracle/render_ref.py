"""TEST INFRASTRUCTURE — CPU restatement of the headless frame renderer.

Only tests/ use this module. It restates mpm_snow_sim2d_b200/csrc/mpm_render.cuh
and mpm_render (mpm_capi.cu) in numpy, in float32 like the kernels: the
reference's Visualize (src/main.cpp:82-160) — white smoothed points of
PARTICLE_SIZE pixels, the BORDER_MARGIN rectangle / wireframe box as 2-pixel
gray lines — with glOrtho(0, WIDTH, 0, HEIGHT) in 2D and SetupCamera
(main.cpp:56-80: 45 degree perspective, near 1, far 1000, lookAt the grid
centre) in 3D; nearest fragment wins, ties to the brighter; rows top first.
"""
from __future__ import annotations

import math

import numpy as np

F = np.float32


def view(dim, width, height, depth, img_w, img_h, angle=0.0, elevation=30.0, distance=300.0, fov=45.0):
    if dim == 2:
        return dict(dim=2, w=img_w, h=img_h, sx=F(img_w / width), sy=F(img_h / height))
    center = np.array([0.5 * width, 0.5 * height, 0.5 * depth])
    rad, elev = math.radians(angle), math.radians(elevation)
    eye = center + distance * np.array([math.cos(elev) * math.sin(rad), math.sin(elev), math.cos(elev) * math.cos(rad)])
    f = center - eye
    f /= np.linalg.norm(f)
    s = np.cross(f, [0.0, 1.0, 0.0])
    s /= np.linalg.norm(s)
    u = np.cross(s, f)
    t = math.tan(math.radians(fov) / 2)
    return dict(dim=3, w=img_w, h=img_h, eye=eye.astype(F), f=f.astype(F), s=s.astype(F), u=u.astype(F),
                pxs=F(1.0 / (img_w / img_h * t)), pys=F(1.0 / t))


def project(V, p):
    """p: (n, 3) float32 -> px, py, depth (float32), visible mask."""
    p = p.astype(F)
    if V["dim"] == 2:
        return p[:, 0] * V["sx"], F(V["h"]) - p[:, 1] * V["sy"], np.zeros(len(p), F), np.ones(len(p), bool)
    d = p - V["eye"]
    xv = d @ V["s"]
    yv = d @ V["u"]
    w = d @ V["f"]
    ok = (w >= 1) & (w <= 1000)
    with np.errstate(divide="ignore", invalid="ignore"):
        px = (V["pxs"] * xv / w + F(1)) * F(0.5) * F(V["w"])
        py = F(V["h"]) - (V["pys"] * yv / w + F(1)) * F(0.5) * F(V["h"])
    return px.astype(F), py.astype(F), w.astype(F), ok


def splat(V, fb, px, py, depth, radius, intensity, smooth):
    r = F(radius)
    reach = int(math.ceil(radius + 1.0)) + 1
    dbits = np.maximum(depth, F(0)).astype(F).view(np.uint32).astype(np.uint64) << np.uint64(32)
    cx, cy = np.floor(px).astype(np.int64), np.floor(py).astype(np.int64)
    for oy in range(-reach, reach + 1):
        for ox in range(-reach, reach + 1):
            x, y = cx + ox, cy + oy
            x0 = np.floor(px - r - F(0.5)).astype(np.int64)
            x1 = np.floor(px + r + F(0.5)).astype(np.int64)
            y0 = np.floor(py - r - F(0.5)).astype(np.int64)
            y1 = np.floor(py + r + F(0.5)).astype(np.int64)
            ok = (x >= np.maximum(x0, 0)) & (x <= np.minimum(x1, V["w"] - 1)) & \
                 (y >= np.maximum(y0, 0)) & (y <= np.minimum(y1, V["h"] - 1))
            dx = x.astype(F) + F(0.5) - px
            dy = y.astype(F) + F(0.5) - py
            if smooth:
                cover = np.clip(r + F(0.5) - np.sqrt(dx * dx + dy * dy), 0, 1)
            else:
                cover = (dx * dx + dy * dy <= r * r).astype(F)
            level = np.rint(cover * F(intensity)).astype(np.int64)
            ok &= level > 0
            if not ok.any():
                continue
            key = dbits[ok] | (255 - level[ok]).astype(np.uint64)
            np.minimum.at(fb, y[ok] * V["w"] + x[ok], key)


def render(positions, dim, width, height, depth, margin, img_w=1200, img_h=600, point_size=1.0, **camera):
    V = view(dim, width, height, depth, img_w, img_h, **camera)
    fb = np.full(img_w * img_h, np.iinfo(np.uint64).max, np.uint64)
    m, W, H, Dp = float(margin), float(width), float(height), float(depth)
    if dim == 2:
        c = [(m, m, 0), (W - m, m, 0), (W - m, H - m, 0), (m, H - m, 0)]
        edges = [(c[k], c[(k + 1) % 4]) for k in range(4)]
    else:
        x0, y0, z0, x1, y1, z1 = m, m, m, W - m, H - m, Dp - m
        e = [(x0, y0, z0, x1, y0, z0), (x1, y0, z0, x1, y0, z1), (x1, y0, z1, x0, y0, z1), (x0, y0, z1, x0, y0, z0),
             (x0, y1, z0, x1, y1, z0), (x1, y1, z0, x1, y1, z1), (x1, y1, z1, x0, y1, z1), (x0, y1, z1, x0, y1, z0),
             (x0, y0, z0, x0, y1, z0), (x1, y0, z0, x1, y1, z0), (x1, y0, z1, x1, y1, z1), (x0, y0, z1, x0, y1, z1)]
        edges = [(a[:3], a[3:]) for a in e]
    for a, b in edges:
        a, b = np.array(a, F), np.array(b, F)
        pa = project(V, a[None])
        pb = project(V, b[None])
        if pa[3][0] and pb[3][0]:
            ln = math.hypot(float(pb[0][0] - pa[0][0]), float(pb[1][0] - pa[1][0]))
            m_s = int(min(65536.0, math.ceil(2.0 * ln) + 1.0))
        else:
            m_s = 4096
        t = (np.arange(m_s + 1, dtype=F) / F(m_s)) if m_s > 0 else np.zeros(1, F)
        pts = a[None] + t[:, None] * (b - a)[None]
        px, py, dpt, ok = project(V, pts)
        splat(V, fb, px[ok], py[ok], dpt[ok], 1.0, 128, False)
    p = np.zeros((len(positions), 3), F)
    p[:, :dim] = positions
    px, py, dpt, ok = project(V, p)
    ok &= np.isfinite(px) & np.isfinite(py)
    splat(V, fb, px[ok], py[ok], dpt[ok], 0.5 * point_size, 255, True)
    lvl = np.where(fb == np.iinfo(np.uint64).max, 0, 255 - (fb & np.uint64(0xFF)).astype(np.int64)).astype(np.uint8)
    return np.repeat(lvl.reshape(img_h, img_w, 1), 3, axis=2)
