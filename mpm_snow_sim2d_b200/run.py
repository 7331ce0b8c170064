"""Run a named workload for a number of steps through the C ABI.

    python -m mpm_snow_sim2d_b200.run c3 --steps 4

Prints the particle count, the device status word and the wall time; used for
profiling captures and quick checks. Workloads: see scenes.workload().
"""
from __future__ import annotations

import argparse
import time

from . import Solver, scenes


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--sort-period", type=int, default=0)
    args = ap.parse_args(argv)
    scene = scenes.workload(args.workload)
    with Solver.from_scene(scene, sort_period=args.sort_period) as s:
        t0 = time.perf_counter()
        s.Step(args.steps)
        pos = s.GetParticlePositions()  # synchronises
        dt = time.perf_counter() - t0
        print(f"{scene.name}: {scene.count} particles, {args.steps} steps, status {s.status()}, "
              f"{dt * 1e3:.1f} ms, first position {pos[0].tolist()}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
