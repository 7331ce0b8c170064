#!/usr/bin/env python3
"""Benchmark: particle-updates/s of the MLS-MPM step (P2G + grid update + G2P
with plasticity) on B200, through the solver's C ABI.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c3] [--impl ours|reference]

One JSON line on rank 0. A step is one P2G -> grid -> G2P pass over every
particle of the workload (default: the 3D snowball-on-slab scene, 128^3 grid,
8 particles per cell, 1.65M particles; its ~0.3 GB of particle and grid state
is larger than the 126 MB L2, so no flush is needed between steps).

* value     device time (CUDA events on the solver's stream) for K steps with
            state resident in HBM; max over ranks; N ranks run independent
            replicas (the path does not shard across GPUs here). The K-step
            loop is repeated until 200 ms have passed (so that the clock
            sampler sees the timed region); value is the median repetition.
* e2e       the same metric through the public C ABI with host buffers: every
            step uploads the particle state from pinned host memory
            (mpm_set_state), steps, and reads the state back (mpm_get_state).
* roofline  the dominant kernel's algorithmic bytes / its CUDA-event duration,
            against MEASURED_PEAKS.json's HBM copy bandwidth; `traffic` is the
            DRAM bytes per launch of that kernel from the ncu summary committed
            under profiles/ (a "bench-traffic:" line), named in traffic_source.
* cpu_baseline  the oracle's FP32 OpenMP port of the reference MLS step on the
            host cores, a bounded number of steps of the same scene.

--impl reference times the reference's CPU implementation of this step on the
host cores (rank 0 only): the oracle's FP32 restatement of the reference
shaders with OpenMP, since the reference's own CPU path (src/cpu) is 2D only;
for 2D workloads the reference's compiled src/cpu runs instead, one solver
per core.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "particle-updates/s (P2G+grid+G2P), plain vs MLP-plasticity, 1 B200, % HBM peak"
UNIT = "particle-updates/s"
STAGE_KERNEL = {"p2g": "k_p2g_warp", "g2p": "k_g2p_gather", "g2p2g": "k_g2p2g", "grid_update": "k_grid_marked",
                "return_map": "k_g2p_plastic"}


def profile_traffic(workload: str, stage: str):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum) of a
    stage's kernel on a workload, from the ncu summaries under profiles/: lines
    `bench-traffic: <kernel> <workload> <bytes per launch>`. (None, None) when
    no summary holds one."""
    kernel = STAGE_KERNEL.get(stage)
    for f in sorted((ROOT / "profiles").glob("*.md")):
        for line in f.read_text().splitlines():
            parts = line.strip().strip("`").split()
            if len(parts) == 4 and parts[0] == "bench-traffic:" and parts[1] == kernel and parts[2] == workload:
                return float(parts[3]), f"profiles/{f.name}"
    return None, None

# Algorithmic bytes (minimal FP32 SoA state, uniform mass/volume).
# Per particle-step: P2G reads x, v, B, F_E, J_p; G2P reads x, F_E, J_p and
# writes x, v, B, F_E, J_p.   Per active node: accumulator clear + read
# 8(d+1) each, node velocities write 8d, G2P read 8d.
def bytes_per_particle(d):
    p2g = 4 * (2 * d + 2 * d * d + 1)
    g2p = 4 * (d + d * d + 1) + 4 * (2 * d + 2 * d * d + 1)
    return p2g, g2p


def bytes_per_node(d):
    grid = 8 * (d + 1) * 2 + 8 * d
    g2p = 8 * d
    return grid, g2p


WORKLOADS = {
    "c3": "3D snowball (r 0.12, v -3) on a 0.1 slab, 128^3 grid, 8 ppc, dt 5e-5",
    "c2": "2D 8 random blocks, 512^2 grid, 8 ppc, dt 2.5e-5",
    "c2_1m": "2D 8 random blocks, 512^2 grid, 27 ppc (~1M particles), dt 2.5e-5",
    "c1": "2D 3 blocks, 128^2 grid, 4 ppc, dt 1e-4",
    "c5": "3D two snowballs (r 0.15, relative speed 6), 256^3 grid, 8 ppc, dt 5e-5",
}


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(value: float) -> float:
    """The largest of every rank's value (the job's time is its slowest rank's);
    the value itself when not distributed. NCCL reduces on the GPU, gloo on the CPU."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(value)
    device = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_rate(world: int, units_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job throughput: every rank's units over the slowest rank's time."""
    return world * units_per_rank * steps / seconds


def make_scene(name):
    from mpm_snow_sim2d_b200 import scenes
    return scenes.workload(name)


def kernel_launches(steps, sorts, auto_period):
    """Kernels the tiled 3D/2D MLS step enqueues over `steps` steps with `sorts`
    re-binning sorts: four every step (fused transfer: grid update, the fused
    G2P + next P2G, the queued particles' return map and their P2G; split
    transfer: P2G, grid update, G2P gather, return map), the four sort kernels
    (count, scan, bucket, per-tile sort) per sort, and with the auto period the
    velocity maximum that picks each period's length."""
    return 4 * steps + (5 if auto_period else 4) * sorts


def active_nodes_initial(scene) -> int:
    """Grid nodes inside some particle's stencil at the scene's initial
    positions (the cubic stencil int(x) - 1 .. int(x) + 2 per axis)."""
    d = scene.dim
    ext = [scene.width, scene.height, scene.depth][:d]
    nx = [e + 1 for e in ext]
    base = np.floor(np.clip(scene.position.astype(np.float64), -8, None)).astype(np.int64) - 1
    marks = np.zeros(int(np.prod(nx)), bool)
    offs = np.stack(np.meshgrid(*([np.arange(4)] * d), indexing="ij"), -1).reshape(-1, d)
    for o in offs:
        g = base + o
        ok = np.all((g >= 0) & (g <= np.array(ext)), axis=1)
        g = g[ok]
        idx = g[:, 0] + nx[0] * g[:, 1] + (nx[0] * nx[1] * g[:, 2] if d == 3 else 0)
        marks[idx] = True
    return int(marks.sum())


def config_of(args, scene, world) -> dict:
    """The workload description both arms print."""
    return {"workload": f"{args.workload}: {WORKLOADS[args.workload]}", "particles": scene.count,
            "nodes": scene.nodes, "active_nodes_initial": active_nodes_initial(scene), "plasticity": "exact",
            "l2": "inputs larger than L2 (no flush)", "parallelism": f"replicas x{world}"}


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def mlp_vs_plain(args, torch, stream):
    """The learned return map against the exact one on the same seeded inputs:
    per-stage device time over the whole run (G2P = gather + return map), and
    the relative L2 error of x, v, F_E, J_p at several horizons. A control run
    of the exact solver from initial velocities perturbed by 1e-6 (relative)
    shows how much any per-step difference of that size grows in this scene."""
    from mpm_snow_sim2d_b200 import Solver, _lib
    from mpm_snow_sim2d_b200.mlp import DEFAULT_WEIGHTS, MIXED_WEIGHTS, Mlp
    scene = make_scene(args.mlp_workload)
    # colliding-snowball workloads take the weights trained with collisions
    weights = args.mlp_weights or (MIXED_WEIGHTS if args.mlp_workload == "c5" else DEFAULT_WEIGHTS)
    net = Mlp.load(weights)
    rng = np.random.Generator(np.random.PCG64(99))
    solvers = {}
    for mode in ("exact", "mlp", "control"):
        s = Solver.from_scene(scene)
        s.set_stream(stream.cuda_stream)
        if mode == "mlp":
            s.set_plasticity(_lib.PLASTIC_MLP, net, args.mlp_tolerance)
        if mode == "control":
            v0 = s.get_state().velocity
            s.set_state(velocity=v0 * (1.0 + 1e-6 * rng.standard_normal(v0.shape)).astype(np.float32))
        solvers[mode] = s
    stages = {m: {} for m in solvers}
    horizons, done, errs = sorted({h for h in (10, 100, 300, args.mlp_steps) if h <= args.mlp_steps}), 0, {}
    for h in horizons:
        st = {}
        for mode, s in solvers.items():
            for k, v in s.step_profiled(h - done).items():
                stages[mode][k] = stages[mode].get(k, 0.0) + v
            st[mode] = s.get_state()
        done = h
        errs[h] = {}
        for name, other in (("mlp", "mlp"), ("control", "control")):
            a, b = st[other], st["exact"]
            errs[h][name] = {"F_E": rel_l2(a.elastic_f, b.elastic_f), "x": rel_l2(a.position, b.position),
                             "v": rel_l2(a.velocity, b.velocity), "J_p": rel_l2(a.plastic_det, b.plastic_det)}
    res = {}
    for mode in ("exact", "mlp"):
        s = solvers[mode]
        r = {"stages_ms": {k: v / args.mlp_steps for k, v in stages[mode].items()},
             "ms_per_step": sum(stages[mode].values()) / args.mlp_steps, "status_flags": s.status()}
        if mode == "mlp":
            acc, rej = s.mlp_stats()
            r.update(accepted=acc, fell_back=rej, accepted_frac=acc / max(acc + rej, 1))
        res[mode] = r
    for s in solvers.values():
        s.close()
    # G2P = the gather (with the fused transfer: the fused kernel, which also
    # does the next step's P2G) + the return map of the queued particles
    g2p = lambda r: r["stages_ms"].get("g2p", r["stages_ms"].get("g2p2g", 0.0)) + r["stages_ms"]["return_map"]
    return {
        "workload": f"{args.mlp_workload}: {WORKLOADS[args.mlp_workload]}", "particles": scene.count,
        "steps": args.mlp_steps, "tolerance": args.mlp_tolerance, "weights": Path(weights).name,
        "plain": res["exact"], "mlp": res["mlp"],
        "g2p_speedup": g2p(res["exact"]) / g2p(res["mlp"]),
        "return_map_speedup": res["exact"]["stages_ms"]["return_map"] / res["mlp"]["stages_ms"]["return_map"],
        "step_speedup": res["exact"]["ms_per_step"] / res["mlp"]["ms_per_step"],
        "rel_l2_vs_plain": {str(h): e["mlp"] for h, e in errs.items()},
        "control_rel_l2_vs_plain": {str(h): e["control"] for h, e in errs.items()},
        "timing": "CUDA events between stages every step (no graph replay), whole run",
    }


def batched_scenes(args, torch):
    """The batched workload: 256 independent 2D scenes (grid sides 64-256,
    2k-64k particles each) advanced `batch_steps` steps in one call after the
    autotuner picked the launch configuration. Scene-step latency from the
    device timestamps each scene records at the end of each of its steps;
    batch-step latency from CUDA events around single-step calls. For
    comparison, the single-scene solver is timed on a sample of the same
    scenes, one after another."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    from mpm_snow_sim2d_b200.batch import Batch
    scs = scenes.batch_scenes_2d(args.batch_scenes, steps=args.batch_steps)
    n = sum(s.count for s in scs)
    stream = torch.cuda.Stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed(fn):
        e0.record(stream)
        fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1)

    with Batch(scs) as b:
        b.set_stream(stream.cuda_stream)
        cfg, tune_ms = b.tune(4)
        b.step(args.warmup)
        torch.cuda.synchronize()
        ms = timed(lambda: b.step(args.batch_steps))
        t = b.step_times().astype(np.int64)
        scene_step_us = np.diff(t, axis=1).ravel() / 1e3
        flags = 0
        for k in range(len(scs)):
            flags |= b.status(k)
        one = [timed(lambda: b.step(1)) for _ in range(args.batch_latency_calls)]
    # the single-scene solver on every 16th scene, back to back
    sample = scs[:: max(1, len(scs) // 16)]
    seq_ms, seq_steps = 0.0, 100
    for sc in sample:
        with Solver.from_scene(sc) as s:
            s.set_stream(stream.cuda_stream)
            s.Step(5)
            seq_ms += timed(lambda: s.Step(seq_steps))
    seq_scene_step_ms = seq_ms / (len(sample) * seq_steps)
    seq_total_s = seq_scene_step_ms * len(scs) * args.batch_steps / 1e3
    p2g_b, g2p_b = bytes_per_particle(2)
    peak, peak_src = load_peaks()
    gbs = n * args.batch_steps * (p2g_b + g2p_b) / (ms / 1e3) / 1e9
    return {
        "workload": f"{len(scs)} independent 2D scenes, grid sides log-uniform 64-256, 1-4 blocks at 4-8 ppc, "
                    f"2k-64k particles each, E ~ U(1e5, 2e5), nu ~ U(0.15, 0.3)",
        "scenes": len(scs), "particles": n, "steps": args.batch_steps, "ms": ms,
        "scenes_per_s": len(scs) / (ms / 1e3),
        "scene_steps_per_s": len(scs) * args.batch_steps / (ms / 1e3),
        "particle_updates_per_s": n * args.batch_steps / (ms / 1e3),
        "scene_step_latency_us": {"p50": float(np.percentile(scene_step_us, 50)),
                                  "p99": float(np.percentile(scene_step_us, 99))},
        "batch_step_latency_ms": {"p50": float(np.percentile(one, 50)), "p99": float(np.percentile(one, 99)),
                                  "calls": len(one)},
        "config": cfg, "tuner_trial_ms": tune_ms,
        "hbm": {"algorithmic_bytes_per_particle_step": p2g_b + g2p_b, "achieved_gbs": gbs, "peak": peak,
                "frac": gbs / peak, "peak_source": peak_src},
        "sequential_single_solver": {"sample_scenes": len(sample), "ms_per_scene_step": seq_scene_step_ms,
                                     "estimated_total_s": seq_total_s,
                                     "batch_speedup": seq_total_s / (ms / 1e3)},
        "status_flags": flags,
        "timing": "CUDA events on the batch's stream; one CUDA graph per call",
    }


def quadratic_variant(args, torch, scene, bytes_per_step_fn):
    """The same workload on the quadratic stencil (3^d nodes, D^-1 = 4):
    device time per step with CUDA events on the solver's stream."""
    from mpm_snow_sim2d_b200 import Solver
    stream = torch.cuda.Stream()
    sc = scene.with_(formulation=2)
    with Solver.from_scene(sc, sort_period=args.sort_period) as q:
        q.set_stream(stream.cuda_stream)
        q.Step(args.warmup)
        m, _ = q.rasterize()
        active = int((m > 0).sum())
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        q.Step(args.quad_steps)
        e1.record(stream)
        e1.synchronize()
        ms = e0.elapsed_time(e1) / args.quad_steps
        stages = {k: v / args.quad_steps for k, v in q.step_profiled(args.quad_steps).items()}
        flags = q.status()
    step_bytes = bytes_per_step_fn(active)
    return {"formulation": "MLS quadratic (3^d nodes, D^-1 = 4)", "steps": args.quad_steps, "ms_per_step": ms,
            "value": scene.count / (ms / 1e3), "unit": UNIT, "stages_ms": stages, "active_nodes": active,
            "step_achieved_gbs": step_bytes / (ms / 1e3) / 1e9, "status_flags": flags}


def cpu_port_time(scene, target_s=12.0, max_steps=20):
    """FP32 OpenMP port of the reference MLS step on all host cores."""
    from oracle import oracle as O
    threads = O.lib().orc_max_threads()
    st = O.initial_state(scene, np.float32)
    t0 = time.perf_counter()
    O.run_oracle(scene, st, 1, fp32=True, threads=threads)
    one = time.perf_counter() - t0
    steps = int(max(1, min(max_steps, target_s / max(one, 1e-6))))
    t0 = time.perf_counter()
    O.run_oracle(scene, st, steps, fp32=True, threads=threads)
    dt = time.perf_counter() - t0
    return dict(value=scene.count * steps / dt, unit=UNIT, cores=threads, kind="port",
                sample=f"{steps} full steps of the {scene.name} scene ({scene.count} particles), FP32, "
                       f"{threads} OpenMP threads, after 1 untimed step")


def refcpu_time(scene, steps, replicas):
    from oracle import oracle as O
    _, info = O.run_refcpu(scene, steps, replicas=replicas)
    return scene.count * steps * replicas / info["loop_seconds"], info


def reference_cpu_leg(steps, c2_steps=0):
    """The reference's own CPU path (src/cpu compiled unmodified) on the 2D
    three-block workload (128^2, 4 ppc): `steps` steps on one core, then one
    independent single-threaded solver per host core at once; with c2_steps,
    the same for a window of that many steps of the 512^2 eight-block
    workload."""
    from mpm_snow_sim2d_b200 import scenes
    from oracle import oracle as O
    if not O.refcpu_available():
        return {"unavailable": "oracle/_ref/refcpu_driver is not built"}
    cores = os.cpu_count() or 1

    def leg(name, n_steps):
        scene = scenes.workload(name)
        one, info1 = refcpu_time(scene, n_steps, 1)
        many, infon = refcpu_time(scene, n_steps, cores)
        return {"workload": f"{name}: {WORKLOADS[name]}", "particles": scene.count, "steps": n_steps, "unit": UNIT,
                "one_core": one, "all_cores": many, "cores": cores, "kind": "reference",
                "sample": f"{n_steps} steps per solver; the reference's src/cpu (CLASSIC APIC, single-threaded) "
                          f"compiled unmodified; all_cores = {cores} independent solvers at once",
                "loop_seconds": {"one_core": info1.get("loop_seconds"), "all_cores": infon.get("loop_seconds")}}

    out = leg("c1", steps)
    if c2_steps > 0:
        out["c2_window"] = leg("c2", c2_steps)
    return out


def run_reference_arm(args):
    world, rank, _ = dist_setup()
    if rank != 0:
        return
    scene = make_scene(args.workload)
    from oracle import oracle as O
    if scene.dim == 2 and O.refcpu_available():
        cores = os.cpu_count() or 1
        for _ in range(args.warmup and 1):
            refcpu_time(scene, 1, 1)
        rate, info = refcpu_time(scene, args.steps, cores)
        kind, sample = "reference", (f"{args.steps} steps of the {scene.name} scene, reference src/cpu compiled "
                                      f"unmodified, {cores} independent single-threaded solvers")
        value = rate
    else:
        threads = O.lib().orc_max_threads()
        st = O.initial_state(scene, np.float32)
        O.run_oracle(scene, st, 1, fp32=True, threads=threads)  # untimed warm-up step
        done, spent = 0, 0.0
        while done < args.steps and spent < args.budget_s:
            t0 = time.perf_counter()
            O.run_oracle(scene, st, 1, fp32=True, threads=threads)
            spent += time.perf_counter() - t0
            done += 1
        value = scene.count * done / spent
        cores, kind = threads, "port"
        sample = (f"{done} of {args.steps} full steps of the {scene.name} scene ({scene.count} particles), capped at "
                  f"{args.budget_s:.0f} s: FP32 restatement of the reference MLS step (src/gpu/shaders/"
                  f"{scene.dim}d) with {threads} OpenMP threads; the reference's own CPU path is 2D only")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded scene)",
        "config": config_of(args, scene, args.gpus),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=10)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--budget-s", type=float, default=60.0, help="CPU time cap of the reference arm")
    ap.add_argument("--sort-period", type=int, default=0, help="steps between particle re-sorts (0: solver default)")
    ap.add_argument("--mlp-workload", default="c5", choices=sorted(WORKLOADS))
    ap.add_argument("--mlp-steps", type=int, default=1000)
    ap.add_argument("--mlp-tolerance", type=float, default=1e-3)
    ap.add_argument("--mlp-weights", default=None, help="network weights (.npz) for the learned return map "
                    "(default: the shipped ones for the workload: collisions for c5, impacts otherwise)")
    ap.add_argument("--no-mlp", action="store_true", help="skip the learned-plasticity comparison")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched-scenes measurement")
    ap.add_argument("--batch-scenes", type=int, default=256)
    ap.add_argument("--batch-steps", type=int, default=500)
    ap.add_argument("--batch-latency-calls", type=int, default=50)
    ap.add_argument("--quad-steps", type=int, default=500, help="timed steps of the quadratic-stencil line (0: skip)")
    ap.add_argument("--refcpu-steps", type=int, default=1000,
                    help="steps of the reference's compiled src/cpu on the 2D three-block workload (0: skip)")
    ap.add_argument("--refcpu-c2-steps", type=int, default=20,
                    help="a window of steps of the same on the 512^2 eight-block workload (0: skip)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)

    if args.impl == "reference":
        run_reference_arm(args)
        return

    import torch
    import torch.distributed as dist
    from mpm_snow_sim2d_b200 import Solver
    from mpm_snow_sim2d_b200.build import build

    world, rank, local = dist_setup()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    if rank == 0:
        build()
    if world > 1:
        dist.barrier()
    device = torch.cuda.current_device()

    scene = make_scene(args.workload)
    d = scene.dim
    stream = torch.cuda.Stream()
    solver = Solver.from_scene(scene, sort_period=args.sort_period)
    solver.set_stream(stream.cuda_stream)

    # warm-up, then active-node count (untimed P2G-only pass)
    solver.Step(args.warmup)
    torch.cuda.synchronize()
    m, _ = solver.rasterize()
    active = int((m > 0).sum())

    # ---- timed region: K steps, state resident in HBM, repeated until the
    # repetitions span 200 ms (every rank runs the same count); value from the
    # median repetition ----
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    def timed_k_steps():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        solver.Step(args.steps)
        e1.record(stream)
        e1.synchronize()
        torch.cuda.synchronize()
        return max_over_ranks(e0.elapsed_time(e1))

    sorts0, _ = solver.sort_stats()
    reps_ms = []
    with ClockSampler(device) as clocks:
        reps_ms.append(timed_k_steps())
        reps = int(max_over_ranks(float(max(1, -(-200.0 // max(reps_ms[0], 1e-3))))))
        while len(reps_ms) < reps:
            reps_ms.append(timed_k_steps())
    ms = float(np.median(reps_ms))
    flags = solver.status()
    sorts1, period_end = solver.sort_stats()
    timed_sorts = (sorts1 - sorts0) / len(reps_ms)
    value = job_rate(world, scene.count, args.steps, ms / 1e3)

    # ---- per-stage device time (events between kernels), for the roofline ----
    stages = solver.step_profiled(args.steps)
    stage_avg = {k: v / args.steps for k, v in stages.items()}

    # ---- e2e: host state in (pinned), step, host state out, through the C ABI ----
    import ctypes as C
    from mpm_snow_sim2d_b200._lib import MpmStateHost, check
    n = scene.count
    pin = lambda *shape: torch.empty(shape, dtype=torch.float32, pin_memory=True)
    host_in = [pin(n, d), pin(n, d), pin(n, d, d), pin(n, d, d), pin(n)]
    host_out = [pin(n, d), pin(n, d), pin(n, d, d), pin(n, d, d), pin(n)]
    st0 = solver.get_state()
    for t_, a in zip(host_in, (st0.position, st0.velocity, st0.affine_b, st0.elastic_f, st0.plastic_det)):
        t_.numpy()[...] = a
    fp = lambda t_: C.cast(C.c_void_p(t_.data_ptr()), C.POINTER(C.c_float))
    hin = MpmStateHost(n, *[fp(t_) for t_ in host_in])
    hout = MpmStateHost(n, *[fp(t_) for t_ in host_out])
    lib = solver._lib
    bytes_state = sum(t_.numel() * 4 for t_ in host_in)
    ke = max(1, args.e2e_steps)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(ke):
        check(lib.mpm_set_state(solver._h, C.byref(hin)), solver._h)
        check(lib.mpm_step(solver._h, 1), solver._h)
        check(lib.mpm_get_state(solver._h, C.byref(hout)), solver._h)
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = job_rate(world, n, ke, e2e_s)

    # ---- roofline of the dominant kernel ----
    # Algorithmic bytes per launch: the split transfer's P2G reads x, v, B, F_E,
    # J_p and its G2P reads x, F_E, J_p, writes x, v, B, F_E, J_p and reads
    # the active nodes' velocities; the fused kernel does the G2P of a step and
    # the P2G of the next, so it carries both particle terms (its P2G takes
    # x, v, B, F_E, J_p from registers: its DRAM traffic is below this count).
    peak, peak_src = load_peaks()
    p2g_b, g2p_b = bytes_per_particle(d)
    grid_b, g2p_nb = bytes_per_node(d)
    if "g2p2g" in stage_avg:
        alg = {"g2p2g": n * (p2g_b + g2p_b) + active * g2p_nb, "grid_update": active * grid_b}
    else:
        alg = {"p2g": n * p2g_b, "grid_update": active * grid_b, "g2p": n * g2p_b + active * g2p_nb}
    dom = max(alg, key=lambda k: stage_avg.get(k, 0.0))
    achieved = alg[dom] / (stage_avg[dom] / 1e3) / 1e9
    step_bytes = sum(alg.values())
    step_ms = ms / args.steps
    traffic, traffic_src = profile_traffic(args.workload, dom)
    roofline = {"bound": "hbm", "kernel": STAGE_KERNEL[dom], "stage": dom, "achieved": achieved, "peak": peak,
                "unit": "GB/s", "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                "peak_source": peak_src, "algorithmic_bytes_per_launch": alg[dom],
                "kernel_ms": stage_avg[dom], "timing": "CUDA events on the solver's stream around the stage, every step",
                "step": {"algorithmic_bytes": step_bytes, "achieved_gbs": step_bytes / (step_ms / 1e3) / 1e9,
                         "frac": step_bytes / (step_ms / 1e3) / 1e9 / peak}}

    mlp = None
    if world == 1 and not args.no_mlp and d == 3:
        try:
            mlp = mlp_vs_plain(args, torch, stream)
        except Exception as e:  # reported next to the headline, never required for it
            mlp = {"error": str(e)}

    quad = None
    if world == 1 and args.quad_steps > 0:
        try:
            quad = quadratic_variant(args, torch, scene, lambda act: n * (p2g_b + g2p_b) + act * (grid_b + g2p_nb))
            quad["step_frac"] = quad["step_achieved_gbs"] / peak
        except Exception as e:  # reported next to the headline, never required for it
            quad = {"error": str(e)}

    batch = None
    if world == 1 and not args.no_batch:
        try:
            batch = batched_scenes(args, torch)
        except Exception as e:  # reported next to the headline, never required for it
            batch = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            cpu = cpu_port_time(scene)
        except Exception as e:  # the CPU baseline is reported, never required
            cpu = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": f"failed: {e}"}

    refcpu_leg = None
    if rank == 0 and world == 1 and args.refcpu_steps > 0:
        try:
            refcpu_leg = reference_cpu_leg(args.refcpu_steps, args.refcpu_c2_steps)
        except Exception as e:  # reported, never required
            refcpu_leg = {"error": str(e)}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": f"synthetic (seeded {scene.name} scene, {scene.count} particles)",
            "config": config_of(args, scene, world),
            "sort_period": (f"auto ({timed_sorts:g} sorts per {args.steps} timed steps, last period {period_end})"
                            if args.sort_period <= 0 else args.sort_period),
            "active_nodes": active, "timed_repetitions": len(reps_ms),
            "repetition_ms": reps_ms,
            "roofline": roofline,
            "stages_ms": stage_avg,
            "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": bytes_state,
                    "d2h_bytes_per_step": bytes_state, "steps": ke},
            "gpu_launches": int(round(kernel_launches(args.steps, timed_sorts, args.sort_period <= 0))),
            "clocks": clocks.summary(),
            "status_flags": flags,
            "cpu_baseline": cpu,
            "reference_cpu_2d": refcpu_leg,
            "mlp_vs_plain": mlp,
            "quadratic": quad,
            "batched": batch,
        }
        print(json.dumps(line), flush=True)
    solver.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
