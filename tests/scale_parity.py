#!/usr/bin/env python3
"""Parity at the workloads' full sizes: the CUDA solver against the FP64 oracle
after the stated step counts (3D snowball on slab, 128^3, 1.65M particles,
1000 steps; 2D eight blocks, 512^2, 2000 steps), next to the reference's own
FP32 arithmetic (the oracle's FP32 instantiation, which reproduces the
reference's GLSL shaders bit for bit, tests/test_shader_pin.py).

The oracle runs take tens of minutes on the host cores and the GPU run
seconds, so the three parts can run on different machines; the solver is
bit-deterministic, so its final state can also be written in pieces:

    python tests/scale_parity.py oracle  --workload c3 --steps 1000 --threads 8 --out DIR
    python tests/scale_parity.py gpu     --workload c3 --steps 1000 --fields position,velocity --out DIR
    python tests/scale_parity.py compare --workload c3 --steps 1000 --oracle DIR --gpu DIR [DIR ...]

or, with the oracle's files copied to the GPU machine, in one go:

    python tests/scale_parity.py gpu --workload c3 --steps 1000 --compare-with DIR --json report.json

Reported: relative L2 over all particles of x, v, B (normalised by |v|), F_E
and J_p, overall and split into particles inside the wall-contact band (a
stencil node within two cells of a wall plane: the nodes where the predictive
wall response, src/gpu/shaders/3d/grid_update.glsl:54, can flip between FP32
and FP64) and the free particles elsewhere.
"""
from __future__ import annotations

import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

FIELDS = ("position", "velocity", "affine_b", "elastic_f", "plastic_det")


def _scene(name):
    from mpm_snow_sim2d_b200 import scenes
    return scenes.workload(name)


def run_oracle(args):
    from oracle import oracle as O
    sc = _scene(args.workload)
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    for tag, fp32 in (("fp64", False), ("fp32", True)):
        st = O.initial_state(sc, np.float32 if fp32 else np.float64)
        t0 = time.time()
        O.run_oracle(sc, st, args.steps, fp32=fp32, threads=args.threads)
        np.savez(out / f"{args.workload}_{args.steps}_{tag}.npz", position=st.position, velocity=st.velocity,
                 affine_b=st.affine_b, elastic_f=st.elastic_f, plastic_det=st.plastic_det)
        print(f"{tag}: {time.time() - t0:.0f} s", flush=True)


def run_gpu(args):
    from mpm_snow_sim2d_b200 import Solver
    sc = _scene(args.workload)
    t0 = time.time()
    with Solver.from_scene(sc) as s:
        s.Step(args.steps)
        st = s.get_state()
        flags = s.status()
    gpu_s = time.time() - t0
    if args.compare_with:
        # compare on this machine against the oracle's files; keep only the report
        od = Path(args.compare_with)
        ref = dict(np.load(od / f"{args.workload}_{args.steps}_fp64.npz"))
        r32 = dict(np.load(od / f"{args.workload}_{args.steps}_fp32.npz"))
        res = report(sc, args.steps, {f: getattr(st, f) for f in FIELDS}, flags, ref, r32)
        res["gpu_wall_s"] = round(gpu_s, 2)
        print(json.dumps(res, indent=1))
        if args.json:
            Path(args.json).write_text(json.dumps(res, indent=1))
        return
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    fields = args.fields.split(",")
    np.savez(out / f"{args.workload}_{args.steps}_gpu_{'_'.join(fields)}.npz", flags=np.uint32(flags),
             **{f: getattr(st, f) for f in fields})
    print(json.dumps({"workload": args.workload, "steps": args.steps, "flags": flags, "fields": fields}))


def contact_band(scene, position):
    """Particles with a cubic-stencil node (floor(x) - 1 .. floor(x) + 2)
    within two cells of a wall plane (x = m and x = extent - m)."""
    d = scene.dim
    ext = np.array([scene.width, scene.height, scene.depth][:d], np.float64)
    m = float(scene.border_margin)
    p = np.asarray(position, np.float64)
    near = np.zeros(p.shape[0], bool)
    for k in range(d):
        near |= (p[:, k] < m + 4.0) | (p[:, k] >= ext[k] - m - 4.0)
    return near


def errors(a, ref, mask=None):
    """Relative L2 of each field both states hold (an oracle file may carry a
    subset); B relative to |v| of `ref`."""
    from conftest import rel_l2
    sel = (lambda x: np.asarray(x)[mask]) if mask is not None else (lambda x: np.asarray(x))
    out = {}
    for f, key in (("position", "x"), ("velocity", "v"), ("elastic_f", "F"), ("plastic_det", "Jp")):
        if f in a and f in ref:
            out[key] = rel_l2(sel(a[f]), sel(ref[f]))
    if "affine_b" in a and "affine_b" in ref and "velocity" in ref:
        vnorm = np.linalg.norm(sel(ref["velocity"]).astype(np.float64))
        out["B"] = float(np.linalg.norm((sel(a["affine_b"]).astype(np.float64) - sel(ref["affine_b"])).ravel())
                         / max(vnorm, 1e-30))
    return out


def compare(args):
    sc = _scene(args.workload)
    od = Path(args.oracle)
    ref = dict(np.load(od / f"{args.workload}_{args.steps}_fp64.npz"))
    r32 = dict(np.load(od / f"{args.workload}_{args.steps}_fp32.npz"))
    gpu, flags = {}, 0
    for d in args.gpu:
        for f in Path(d).glob(f"{args.workload}_{args.steps}_gpu_*.npz"):
            z = np.load(f)
            flags |= int(z["flags"])
            gpu.update({k: z[k] for k in z.files if k != "flags"})
    missing = [f for f in FIELDS if f not in gpu]
    if missing:
        raise SystemExit(f"GPU fields missing: {missing}")
    res = report(sc, args.steps, gpu, flags, ref, r32)
    print(json.dumps(res, indent=1))
    if args.json:
        Path(args.json).write_text(json.dumps(res, indent=1))


def report(sc, steps, gpu, flags, ref, r32):
    band = contact_band(sc, ref["position"])
    res = {"workload": sc.name, "particles": sc.count, "steps": steps, "gpu_status_flags": int(flags),
           "contact_particles": int(band.sum()), "free_particles": int((~band).sum())}
    for name, a, base in (("gpu_vs_fp64", gpu, ref), ("reference_fp32_vs_fp64", r32, ref),
                          ("gpu_vs_reference_fp32", gpu, r32)):
        res[name] = {"all": errors(a, base), "contact": errors(a, base, band), "free": errors(a, base, ~band)}
    return res


def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    for name in ("oracle", "gpu", "compare"):
        p = sub.add_parser(name)
        p.add_argument("--workload", default="c3")
        p.add_argument("--steps", type=int, default=1000)
        if name == "oracle":
            p.add_argument("--threads", type=int, default=8)
            p.add_argument("--out", required=True)
        elif name == "gpu":
            p.add_argument("--fields", default=",".join(FIELDS))
            p.add_argument("--out", help="write the final state's fields here")
            p.add_argument("--compare-with", help="oracle directory: compare on this machine, write only the report")
            p.add_argument("--json")
        else:
            p.add_argument("--oracle", required=True)
            p.add_argument("--gpu", nargs="+", required=True)
            p.add_argument("--json")
    args = ap.parse_args()
    {"oracle": run_oracle, "gpu": run_gpu, "compare": compare}[args.cmd](args)


if __name__ == "__main__":
    main()
