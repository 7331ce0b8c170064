"""Generate the golden fixtures from the reference's own CPU code.

Runs oracle/_ref/refcpu_driver (src/cpu/Grid.cpp + src/cpu/Particles.cpp of the
reference, compiled unmodified by oracle/build_oracle.py) on small seeded
scenes and stores the particle state after selected steps, together with the
scene itself, as compressed .npz files in this directory.

    python tests/golden/make_golden.py [case ...]

Needs the reference tree (to build the driver); the fixtures it writes are
committed so that tests run without it.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

from mpm_snow_sim2d_b200 import scenes  # noqa: E402
from oracle import oracle as O  # noqa: E402
from oracle.build_oracle import build_refcpu  # noqa: E402

def _reference_default_2d():
    """The reference's default 2D scene (src/shared/Parameters.h:30-80) with the
    particles the device sampler draws for seed 11, here from its bit-exact CPU
    restatement (oracle/sample_ref.py)."""
    from oracle import sample_ref

    def sampler(dim, shapes, md, seed, rounds):
        full = [dict(kind=s["kind"], center=tuple(s["center"]) + (0.0,) * (3 - len(s["center"])),
                     radius=s["radius"], half=tuple(s["half"]) + (0.0,) * (3 - len(s["half"]))) for s in shapes]
        return sample_ref.sample_shapes(dim, full, md, seed, rounds)

    return scenes.reference_snowballs(2, seed=11, sampler=sampler)


CASES = {
    # the reference's own default scene: two snowballs thrown at each other, 12,686
    # particles, dt 1e-3; they meet near step 875
    "refcpu_reference_default2d": dict(scene=_reference_default_2d, dumps=(1, 500, 1000)),
    # three falling blocks, 1 particle per cell (1106 particles), 1000 steps of dt 1e-4
    "refcpu_blocks2d_ppc1": dict(scene=lambda: scenes.snow_blocks_2d(ppc=1, seed=2001), dumps=(1, 10, 100, 1000)),
    # one block driven into the floor: wall separation, Coulomb friction and plastic flow
    "refcpu_impact2d": dict(scene=lambda: scenes.impact_2d(seed=2002), dumps=(1, 50, 200, 400)),
}


def save_case(name: str, scene, dumps) -> Path:
    nsteps = max(dumps)
    out, info = O.run_refcpu(scene, nsteps, dump_every=1)
    by_step = {s: d for s, d in out}
    arrays = dict(
        position0=scene.position, velocity0=scene.velocity, volume=scene.volume, mass=scene.mass,
        knobs=np.array([scene.width, scene.height, scene.border_margin, scene.delta_time, scene.gravity,
                        scene.friction, scene.theta_c, scene.theta_s, scene.xi, scene.nu, scene.youngs,
                        scene.rho], np.float64),
        steps=np.array(dumps, np.int32),
    )
    for s in dumps:
        d = by_step[s]
        for k, v in d.items():
            arrays[f"s{s}_{k}"] = v.astype(np.float32)
    path = HERE / f"{name}.npz"
    np.savez_compressed(path, **arrays)
    print(f"{path.name}: {scene.count} particles, steps {dumps}, {path.stat().st_size} bytes, "
          f"refcpu {info['loop_seconds']:.2f} s")
    return path


def main(names=None) -> None:
    if build_refcpu() is None:
        raise SystemExit("the reference tree is needed to build oracle/_ref/refcpu_driver")
    for name, case in CASES.items():
        if names and name not in names:
            continue
        save_case(name, case["scene"](), case["dumps"])


if __name__ == "__main__":
    main(sys.argv[1:])
