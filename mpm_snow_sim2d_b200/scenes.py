"""Seeded snow scenes in the reference's grid units.

The workloads are stated on the unit square / cube with cell size dx = 1/W.
The reference integrates in grid units (node i at x = i, src/cpu/Grid.cpp:
10-14; p2g.glsl:73), so a physical scene maps as
    x~ = x / dx,  v~ = v / dx,  GRAVITY = g / dx,
    volume~ = 1 / ppc (cell fractions),  RHO~ = rho * dx^2 * 100,
which makes mass~ = volume~ * RHO~ / 100 = rho dx^2 / ppc. With these the
reference's grid-unit force term  V~ sigma (x_p - x_i) 3 dt  and momentum
m~ v~ keep the physical ratio 1 / (rho dx^2) in 2D and 3D alike, so the
scaled step is the physical step divided by dx. E, nu, theta_c, theta_s, xi
and dt are unchanged.

The reference samples with std::random_device (src/shared/Shapes.h:23,150),
which is not reproducible; here every scene draws from numpy's PCG64 with a
fixed seed, and the CUDA solver and the oracles consume the same arrays.
"""
from __future__ import annotations

from dataclasses import dataclass, field, replace

import numpy as np

from ._lib import BOUNDARY_FRICTION, FORMULATION_MLS


@dataclass
class Scene:
    name: str
    dim: int
    width: int
    height: int
    depth: int
    border_margin: int
    delta_time: float
    gravity: float
    friction: float
    theta_c: float
    theta_s: float
    xi: float
    nu: float
    youngs: float
    rho: float
    steps: int
    position: np.ndarray          # (n, dim) float32, grid units
    velocity: np.ndarray          # (n, dim) float32, grid units / s
    volume: np.ndarray            # (n,) float32
    mass: np.ndarray              # (n,) float32
    formulation: int = FORMULATION_MLS
    boundary: int = BOUNDARY_FRICTION
    info: dict = field(default_factory=dict)

    @property
    def count(self) -> int:
        return int(self.position.shape[0])

    @property
    def nodes(self) -> int:
        n = (self.width + 1) * (self.height + 1)
        return n * (self.depth + 1) if self.dim == 3 else n

    def with_(self, **kw) -> "Scene":
        return replace(self, **kw)


# Snow material of the workloads (E, nu, rho, xi, theta_c, theta_s).
MATERIAL = dict(youngs=1.4e5, nu=0.2, rho_phys=400.0, xi=10.0, theta_c=2.5e-2, theta_s=7.5e-3)
FRICTION = 0.3  # Parameters.h:60
MARGIN = 3


def _scene(name, dim, W, dt, steps, pos_phys, vel_phys, ppc, rng_info, *, depth=None, g=-9.8,
           youngs=MATERIAL["youngs"], nu=MATERIAL["nu"]) -> Scene:
    dx = 1.0 / W
    n = pos_phys.shape[0]
    vol = np.full(n, 1.0 / ppc, dtype=np.float32)
    rho_ref = MATERIAL["rho_phys"] * dx * dx * 100.0
    mass = (vol * np.float32(rho_ref)) / np.float32(100.0)  # Particle ctor: vol * RHO / 100
    return Scene(
        name=name, dim=dim, width=W, height=W, depth=(depth or W) if dim == 3 else 0,
        border_margin=MARGIN, delta_time=dt, gravity=g / dx, friction=FRICTION,
        theta_c=MATERIAL["theta_c"], theta_s=MATERIAL["theta_s"], xi=MATERIAL["xi"],
        nu=nu, youngs=youngs, rho=rho_ref, steps=steps,
        position=np.ascontiguousarray((pos_phys / dx).astype(np.float32)),
        velocity=np.ascontiguousarray((vel_phys / dx).astype(np.float32)),
        volume=vol, mass=mass.astype(np.float32), info=dict(rng_info, dx=dx, ppc=ppc),
    )


def _box(rng, lo, hi, ppc, dx):
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    count = int(round(np.prod(hi - lo) / dx ** len(lo) * ppc))
    return lo + rng.random((count, len(lo))) * (hi - lo)


def _ball(rng, center, radius, ppc, dx):
    center = np.asarray(center, np.float64)
    d = len(center)
    vol = (np.pi * radius ** 2) if d == 2 else (4.0 / 3.0 * np.pi * radius ** 3)
    count = int(round(vol / dx ** d * ppc))
    out = np.empty((0, d))
    while out.shape[0] < count:
        cand = rng.random((2 * count, d)) * 2.0 - 1.0
        cand = cand[(cand ** 2).sum(1) <= 1.0]
        out = np.concatenate([out, center + radius * cand])
    return out[:count]


def snow_blocks_2d(ppc: int = 4, seed: int = 1001, steps: int = 1000) -> Scene:
    """Three axis-aligned snow blocks of side 0.15 on a 128^2 grid, dt 1e-4."""
    W, dx = 128, 1.0 / 128
    rng = np.random.Generator(np.random.PCG64(seed))
    pts = [_box(rng, np.array(c) - 0.075, np.array(c) + 0.075, ppc, dx) for c in ((0.3, 0.6), (0.5, 0.8), (0.7, 0.6))]
    pos = np.concatenate(pts)
    vel = np.array([0.0, -1.0]) + rng.uniform(-0.1, 0.1, pos.shape)
    return _scene(f"blocks2d_128_ppc{ppc}", 2, W, 1e-4, steps, pos, vel, ppc, dict(seed=seed))


def impact_2d(W: int = 128, ppc: int = 2, seed: int = 1011, steps: int = 400, dt: float = 1e-4) -> Scene:
    """One block (side 0.2) thrown at the floor with v = (0.5, -4): wall
    separation, Coulomb friction and plastic flow within a few hundred steps."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    pos = _box(rng, (0.4, 0.06), (0.6, 0.26), ppc, dx)
    vel = np.array([0.5, -4.0]) + rng.uniform(-0.05, 0.05, pos.shape)
    return _scene(f"impact2d_{W}_ppc{ppc}", 2, W, dt, steps, pos, vel, ppc, dict(seed=seed))


def impact_3d(W: int = 32, ppc: int = 2, seed: int = 1013, steps: int = 300, dt: float = 1e-4) -> Scene:
    """A snowball dropped onto a slab at 4 m/s on a small grid (contact within ~50 steps)."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    ball = _ball(rng, (0.5, 0.45, 0.5), 0.15, ppc, dx)
    m = MARGIN * dx
    slab = _box(rng, (m, m, m), (1.0 - m, m + 0.2, 1.0 - m), ppc, dx)
    pos = np.concatenate([ball, slab])
    vel = np.zeros_like(pos)
    vel[: ball.shape[0], 1] = -4.0
    vel[: ball.shape[0], 0] = 0.5
    return _scene(f"impact3d_{W}_ppc{ppc}", 3, W, dt, steps, pos, vel, ppc, dict(seed=seed))


def random_blocks_2d(W: int = 512, nblocks: int = 8, ppc: int = 8, seed: int = 1002, steps: int = 2000,
                     dt: float = 2.5e-5, side=(0.05, 0.2)) -> Scene:
    """Non-overlapping square blocks of random side placed by rejection."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    lo_wall, hi_wall = (MARGIN + 2) * dx, 1.0 - (MARGIN + 2) * dx
    boxes = []
    tries = 0
    while len(boxes) < nblocks:
        tries += 1
        if tries > 100000:
            raise RuntimeError("could not place the blocks without overlap")
        s = rng.uniform(*side)
        c = rng.uniform(lo_wall + s / 2, hi_wall - s / 2, 2)
        lo, hi = c - s / 2, c + s / 2
        if all(np.any(hi <= b_lo) or np.any(lo >= b_hi) for b_lo, b_hi in boxes):
            boxes.append((lo, hi))
    pos = np.concatenate([_box(rng, lo, hi, ppc, dx) for lo, hi in boxes])
    vel = np.array([0.0, -1.0]) + rng.uniform(-0.1, 0.1, pos.shape)
    return _scene(f"randblocks2d_{W}_ppc{ppc}", 2, W, dt, steps, pos, vel, ppc,
                  dict(seed=seed, blocks=[(lo.tolist(), hi.tolist()) for lo, hi in boxes]))


def snowball_on_slab_3d(W: int = 128, ppc: int = 8, seed: int = 1003, steps: int = 1000, dt: float = 5e-5,
                        radius: float = 0.12, slab: float = 0.1) -> Scene:
    """A snowball (r 0.12, centre (0.5, 0.7, 0.5), v (0, -3, 0)) above a 0.1-thick slab on the floor."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    ball = _ball(rng, (0.5, 0.7, 0.5), radius, ppc, dx)
    m = MARGIN * dx
    slab_pts = _box(rng, (m, m, m), (1.0 - m, m + slab, 1.0 - m), ppc, dx)
    pos = np.concatenate([ball, slab_pts])
    vel = np.zeros_like(pos)
    vel[: ball.shape[0], 1] = -3.0
    return _scene(f"snowball_slab3d_{W}_ppc{ppc}", 3, W, dt, steps, pos, vel, ppc,
                  dict(seed=seed, ball_particles=int(ball.shape[0])))


def two_snowballs_3d(W: int = 256, ppc: int = 8, seed: int = 1005, steps: int = 1000, dt: float = 5e-5,
                     radius: float = 0.15, speed: float = 6.0) -> Scene:
    """Two snowballs (r 0.15) colliding head-on along x at relative speed 6."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    a = _ball(rng, (0.32, 0.5, 0.5), radius, ppc, dx)
    b = _ball(rng, (0.68, 0.5, 0.5), radius, ppc, dx)
    pos = np.concatenate([a, b])
    vel = np.zeros_like(pos)
    vel[: a.shape[0], 0] = speed / 2
    vel[a.shape[0]:, 0] = -speed / 2
    return _scene(f"two_snowballs3d_{W}_ppc{ppc}", 3, W, dt, steps, pos, vel, ppc, dict(seed=seed))


# Poisson-disk samples per unit area at minimum distance r: about 0.675 / r^2
# for the device sampler (measured on a 2D ball: 6361 samples of r = 0.2739
# on an area of 706.9).
POISSON_DENSITY_2D = 0.675


def batch_scene_2d(index: int, seed: int = 1004, steps: int = 500, side=(64, 256), count=(2000, 64000),
                   fill_max: float = 0.35, sampler: str = "uniform") -> Scene:
    """Scene `index` of the batched workload: a square grid of side drawn
    log-uniformly in [64, 256] cells, 1-4 non-overlapping snow blocks at 4-8
    particles per cell holding a particle count drawn log-uniformly in
    [2k, 64k] (capped at fill_max of the domain), E ~ U(1e5, 2e5),
    nu ~ U(0.15, 0.3); dt scales with the cell size (1e-4 at 128 cells).
    Seed: seed + index. sampler "uniform" draws the particles with numpy;
    "poisson" fills the blocks on the GPU with the Poisson-disk sampler at the
    same mean density (the volume per particle is the blocks' area over the
    count, so the mass of the scene is unchanged)."""
    rng = np.random.Generator(np.random.PCG64(seed + index))
    W = int(round(np.exp(rng.uniform(np.log(side[0]), np.log(side[1])))))
    dx = 1.0 / W
    nblocks = int(rng.integers(1, 5))
    ppc = int(rng.integers(4, 9))
    youngs = float(rng.uniform(1e5, 2e5))
    nu = float(rng.uniform(0.15, 0.3))
    hi_count = min(count[1], fill_max * W * W * ppc)
    target = float(np.exp(rng.uniform(np.log(count[0]), np.log(hi_count))))
    area = target / (W * W * ppc)  # fraction of the unit square
    shares = rng.dirichlet(np.ones(nblocks)) * area
    lo_wall, hi_wall = (MARGIN + 2) * dx, 1.0 - (MARGIN + 2) * dx
    boxes = []
    for _ in range(1000):  # place every block, restarting the layout when one does not fit
        boxes = []
        for a in sorted(shares, reverse=True):
            s_ = float(np.sqrt(a))
            for _ in range(200):
                c = rng.uniform(lo_wall + s_ / 2, hi_wall - s_ / 2, 2)
                lo, hi = c - s_ / 2, c + s_ / 2
                if all(np.any(hi <= b_lo) or np.any(lo >= b_hi) for b_lo, b_hi in boxes):
                    boxes.append((lo, hi))
                    break
            else:
                break
        if len(boxes) == nblocks:
            break
    else:
        raise RuntimeError("could not place the blocks without overlap")
    ppc_eff = ppc
    if sampler == "poisson":
        from .sampling import box, sample_shapes
        md = float(np.sqrt(POISSON_DENSITY_2D / ppc))  # cells
        shapes = [box(((lo + hi) / (2 * dx)).tolist(), ((hi - lo) / (2 * dx)).tolist()) for lo, hi in boxes]
        grid_pos, _ = sample_shapes(2, shapes, md, seed + index)
        pos = grid_pos.astype(np.float64) * dx
        area_cells = sum(float(np.prod((hi - lo) / dx)) for lo, hi in boxes)
        ppc_eff = pos.shape[0] / area_cells
    elif sampler == "uniform":
        pos = np.concatenate([_box(rng, lo, hi, ppc, dx) for lo, hi in boxes])
    else:
        raise ValueError(f"unknown sampler {sampler!r}")
    vel = np.array([0.0, -1.0]) + rng.uniform(-0.1, 0.1, pos.shape)
    dt = 1e-4 * 128.0 / W
    return _scene(f"batch2d_{index}_{W}_ppc{ppc}", 2, W, dt, steps, pos, vel, ppc_eff,
                  dict(seed=seed + index, blocks=nblocks, sampler=sampler), youngs=youngs, nu=nu)


def batch_scenes_2d(nscenes: int = 256, seed: int = 1004, steps: int = 500, sampler: str = "uniform") -> list:
    """The batched workload: `nscenes` independent 2D scenes (batch_scene_2d)."""
    return [batch_scene_2d(i, seed=seed, steps=steps, sampler=sampler) for i in range(nscenes)]


def workload(name: str) -> Scene:
    """The named workloads: c1..c5 with the sizes stated for them."""
    if name == "c1":
        return snow_blocks_2d()
    if name == "c1_22k":
        return snow_blocks_2d(ppc=20)
    if name == "c2":
        return random_blocks_2d()
    if name == "c2_1m":
        return random_blocks_2d(ppc=27)
    if name == "c3":
        return snowball_on_slab_3d()
    if name == "c5":
        return two_snowballs_3d()
    raise KeyError(name)


# The reference's default scene, in its own units (src/shared/Parameters.h:30-80):
# a 200 x 100 (x 100) grid, border margin 2, two snowballs of radius 15 at
# (50, 45[, 50]) and (150, 55[, 50]) thrown at each other at 40 cells/s,
# dt 1e-3, gravity -9.81, friction 0.3, theta_c 2e-2, theta_s 6e-3, xi 10,
# nu 0.2, E 1.4e5, RHO 400; NUM_PARTICLES 3000 sets min_dist.
REFERENCE_DEFAULT = dict(width=200, height=100, depth=100, margin=2, radius=15.0, num_particles=3000,
                         centers=((50.0, 45.0, 50.0), (150.0, 55.0, 50.0)), velocities=((40.0, 0.0, 0.0), (-40.0, 0.0, 0.0)),
                         delta_time=1e-3, gravity=-9.81, friction=0.3, theta_c=2.0e-2, theta_s=6.0e-3, xi=10.0,
                         nu=0.2, youngs=1.4e5, rho=400.0)


def reference_snowballs(dim: int = 2, seed: int = 1, steps: int = 6600, rounds: int = 30, sampler=None) -> Scene:
    """The reference's two-snowball scene with particles from the device
    Poisson-disk sampler (needs a GPU). Per snowball, as
    src/gpu/GPUSolver.cpp:99-155: min_dist = radius / NUM_PARTICLES^(1/dim),
    vol = (2 pi r^2 in 2D | 4/3 pi r^3 in 3D) / samples, mass = vol RHO / 100.
    The default 6600 steps are the reference's 200 frames at 30 frames/s.
    `sampler(dim, shapes, min_dist, seed, rounds)` replaces the device sampler
    (a restatement with the same output, for fixtures made without a GPU).
    """
    from .sampling import ball, sample_shapes

    sample_shapes = sampler or sample_shapes

    R = REFERENCE_DEFAULT
    r = R["radius"]
    n_ref = float(R["num_particles"])
    md = np.float32(r) / (np.sqrt(np.float32(n_ref)) if dim == 2 else np.cbrt(np.float32(n_ref)))
    pos, vel, vol, mass, counts = [], [], [], [], []
    for k, (c, v) in enumerate(zip(R["centers"], R["velocities"])):
        p, _ = sample_shapes(dim, [ball(c[:dim], r)], float(md), seed + 7919 * k, rounds)
        n = p.shape[0]
        f, pi, rf = np.float32, np.float32(3.1415926), np.float32(r)  # Shapes.h:8 PI, float arithmetic
        v_p = (f(2) * pi * rf * rf if dim == 2 else (f(4) / f(3)) * pi * rf * rf * rf) / f(n)
        pos.append(p)
        vel.append(np.tile(np.asarray(v[:dim], np.float32), (n, 1)))
        vol.append(np.full(n, v_p, np.float32))
        mass.append(np.full(n, v_p * np.float32(R["rho"]) / np.float32(100.0), np.float32))
        counts.append(n)
    return Scene(
        name=f"reference_snowballs{dim}d", dim=dim, width=R["width"], height=R["height"],
        depth=R["depth"] if dim == 3 else 0, border_margin=R["margin"], delta_time=R["delta_time"],
        gravity=R["gravity"], friction=R["friction"], theta_c=R["theta_c"], theta_s=R["theta_s"], xi=R["xi"],
        nu=R["nu"], youngs=R["youngs"], rho=R["rho"], steps=steps,
        position=np.ascontiguousarray(np.concatenate(pos)), velocity=np.ascontiguousarray(np.concatenate(vel)),
        volume=np.concatenate(vol), mass=np.concatenate(mass),
        info=dict(seed=seed, min_dist=float(md), per_ball=counts, sampler="device poisson-disk"),
    )
