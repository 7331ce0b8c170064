"""Run a named workload for a number of steps through the C ABI.

    python -m mpm_snow_sim2d_b200.run c3 --steps 4
    python -m mpm_snow_sim2d_b200.run impact64 --steps 100 --plasticity mlp
    python -m mpm_snow_sim2d_b200.run c4 --scenes 64 --steps 10 --batch-threads 1024
    python -m mpm_snow_sim2d_b200.run c1 --steps 1000 --frames frames/
    python -m mpm_snow_sim2d_b200.run c3 --steps 4 --formulation quadratic
    python -m mpm_snow_sim2d_b200.run reference2d --steps 6600 --frames frames/

Prints the particle count, the device status word and the wall time; used for
profiling captures and quick checks. Workloads: see scenes.workload(); "impact64" is the training set-up of the
learned return map (a 6 m/s snowball impact on a slab, 64^3); "c4" the first
`--scenes` scenes of the batched workload, run as one batch; "reference2d" /
"reference3d" the reference's default two-snowball scene (scenes.reference_snowballs).
"""
from __future__ import annotations

import argparse
import time

from . import Solver, _lib, scenes


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("workload")
    ap.add_argument("--steps", type=int, default=4)
    ap.add_argument("--sort-period", type=int, default=0)
    ap.add_argument("--plasticity", choices=["exact", "mlp"], default="exact")
    ap.add_argument("--formulation", choices=["mls", "classic", "quadratic"], default=None,
                    help="override the scene's formulation (quadratic: 3^d-node stencil)")
    ap.add_argument("--frames", default=None, help="write a PNG frame every --frame-steps steps to this directory")
    ap.add_argument("--frame-steps", type=int, default=0,
                    help="steps per frame (0: 1 / (SAVE_FPS dt), SAVE_FPS = 30 as in Parameters.h:69)")
    ap.add_argument("--scenes", type=int, default=256, help="c4: scenes in the batch")
    ap.add_argument("--batch-threads", type=int, default=1024, help="c4: threads per CTA")
    args = ap.parse_args(argv)
    if args.workload == "c4":
        from .batch import Batch
        scs = scenes.batch_scenes_2d(args.scenes)
        with Batch(scs) as b:
            b.set_config(threads=args.batch_threads, particles_per_cta=16384)
            t0 = time.perf_counter()
            b.step(args.steps)
            flags = 0
            for k in range(len(scs)):
                flags |= b.status(k)  # synchronises
            dt = time.perf_counter() - t0
            print(f"c4: {len(scs)} scenes, {b.total_particles} particles, {args.steps} steps, status {flags}, "
                  f"{dt * 1e3:.1f} ms, config {b.config}")
        return 0
    if args.workload == "impact64":
        from .mlp_train import impact_scene
        scene = impact_scene(6.0, seed=777002, W=64, steps=args.steps)
    elif args.workload in ("reference2d", "reference3d"):
        # the reference's default two-snowball scene, sampled on the device
        scene = scenes.reference_snowballs(2 if args.workload == "reference2d" else 3)
    else:
        scene = scenes.workload(args.workload)
    if args.formulation:
        scene = scene.with_(formulation={"mls": _lib.FORMULATION_MLS, "classic": _lib.FORMULATION_CLASSIC,
                                         "quadratic": _lib.FORMULATION_MLS_QUADRATIC}[args.formulation])
    with Solver.from_scene(scene, sort_period=args.sort_period) as s:
        if args.plasticity == "mlp":
            from .mlp import DEFAULT_WEIGHTS, Mlp
            net = Mlp.load(DEFAULT_WEIGHTS)
            s.set_plasticity(_lib.PLASTIC_MLP, net, 1e-3)
        t0 = time.perf_counter()
        if args.frames:
            # Simulate + Visualize + saveFrame (src/main.cpp:163-205) without a window
            from pathlib import Path
            from .image import write_png
            out = Path(args.frames)
            out.mkdir(parents=True, exist_ok=True)
            per = args.frame_steps or max(1, round(1.0 / (30.0 * scene.delta_time)))
            done, frame = 0, 0
            while done < args.steps:
                k = min(per, args.steps - done)
                s.Step(k)
                done += k
                write_png(out / f"frame_{frame}.png", s.render())
                frame += 1
        else:
            s.Step(args.steps)
        pos = s.GetParticlePositions()  # synchronises
        dt = time.perf_counter() - t0
        print(f"{scene.name}: {scene.count} particles, {args.steps} steps, status {s.status()}, "
              f"{dt * 1e3:.1f} ms, first position {pos[0].tolist()}")
        if args.plasticity == "mlp":
            print("learned return map: accepted %d, fell back %d" % s.mlp_stats())
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
