"""Train the learned plasticity surrogate on pairs logged by the plain solver.

    python -m mpm_snow_sim2d_b200.mlp_train [--pairs 50000000] [--steps 60000] [--batch 16384] [--lr 4e-3] [--out PATH]
        [--save-pairs DIR | --load-pairs DIR]

Data: seeded snowball-on-slab impacts (the 3D workload's set-up, 64^3 grid so
that contact starts at once) with impact speeds drawn from U(1, 8) m/s, 1000 steps
each; every step logs the exact return map (F_hat, J_p) -> (F_E', J_p') of
each particle whose trial F left the elastic band (mpm_pair_log_*), and a
uniform subset of each 10-step window is kept. Training: the library's
own GPU kernels (BF16 tensor-core forward/backward, AdamW). Writes the FP32
parameters and the feature normalisation to an .npz.
"""
from __future__ import annotations

import argparse
import time

import numpy as np

from . import Solver, _lib, scenes
from .mlp import DEFAULT_WEIGHTS, Mlp, features, normalization, targets


def impact_scene(speed: float, seed: int, W: int = 64, steps: int = 200):
    """A snowball launched at `speed` m/s into a slab, touching it at the start."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    radius = rng.uniform(0.1, 0.16)
    slab = 0.1
    m = scenes.MARGIN * dx
    top = m + slab
    cy = top + radius + 0.5 * dx
    ang = rng.uniform(-0.5, 0.5)
    ball = scenes._ball(rng, (rng.uniform(0.35, 0.65), cy, rng.uniform(0.35, 0.65)), radius, 8, dx)
    box = scenes._box(rng, (m, m, m), (1.0 - m, top, 1.0 - m), 8, dx)
    pos = np.concatenate([ball, box])
    vel = np.zeros_like(pos)
    vel[: ball.shape[0], 0] = speed * np.sin(ang)
    vel[: ball.shape[0], 1] = -speed * np.cos(ang)
    return scenes._scene(f"impact_v{speed:.2f}", 3, W, 5e-5, steps, pos, vel, 8, dict(seed=seed))


def collision_scene(speed: float, seed: int, W: int = 256, steps: int = 1000):
    """Two snowballs of radius U(0.12, 0.16) thrown at each other at relative
    speed `speed` m/s along a random direction near the x axis, a few cells
    apart at the start (the two-snowball workload's set-up with other sizes,
    speeds and seeds)."""
    dx = 1.0 / W
    rng = np.random.Generator(np.random.PCG64(seed))
    r = rng.uniform(0.12, 0.16)
    gap = rng.uniform(2.0, 6.0) * dx
    th, ph = rng.uniform(-0.3, 0.3), rng.uniform(-0.3, 0.3)
    u = np.array([np.cos(th) * np.cos(ph), np.sin(th), np.cos(th) * np.sin(ph)])
    c = np.array([0.5, rng.uniform(0.4, 0.6), 0.5])
    ca, cb = c - u * (r + gap / 2), c + u * (r + gap / 2)
    a = scenes._ball(rng, tuple(ca), r, 8, dx)
    b = scenes._ball(rng, tuple(cb), r, 8, dx)
    pos = np.concatenate([a, b])
    vel = np.zeros_like(pos)
    vel[: a.shape[0]] = u * speed / 2
    vel[a.shape[0]:] = -u * speed / 2
    return scenes._scene(f"collide_v{speed:.2f}", 3, W, 5e-5, steps, pos, vel, 8, dict(seed=seed))


def collect_pairs(n_pairs: int, seed: int = 7, W: int = 64, steps: int = 1000, per_scene: int = 1_000_000,
                  every: int = 10, verbose: bool = True, kind: str = "impact") -> np.ndarray:
    """Exact return-map pairs from seeded impacts (kind "impact": snowball on
    slab) or collisions (kind "collision": two snowballs), spread over each
    whole run: the log holds every out-of-band particle of `every` steps, and
    each read keeps a uniform random subset of per_scene / (steps / every)
    rows."""
    rng = np.random.Generator(np.random.PCG64(seed))
    chunks, total, k = [], 0, 0
    reads = max(1, steps // every)
    while total < n_pairs:
        speed = float(rng.uniform(1.0, 8.0))
        if kind == "collision":
            sc = collision_scene(speed, seed * 1000 + k, W=W, steps=steps)
        else:
            sc = impact_scene(speed, seed * 1000 + k, W=W, steps=steps)
        keep = max(1, min(per_scene, n_pairs - total) // reads)
        log_cap = every * sc.count
        taken = []
        with Solver.from_scene(sc) as s:
            s.pair_log_enable(log_cap)
            for _ in range(reads):
                s.Step(every)
                got = s.pair_log_read(log_cap)
                if got.shape[0] > keep:
                    got = got[rng.choice(got.shape[0], keep, replace=False)]
                if got.shape[0]:
                    taken.append(got)
            s.pair_log_enable(0)
        p = np.concatenate(taken) if taken else np.empty((0, 20), np.float32)
        p = p[np.isfinite(p).all(1) & (p[:, 9] > 0) & (p[:, 19] > 0)]
        chunks.append(p)
        total += p.shape[0]
        k += 1
        if verbose:
            print(f"scene {k}: speed {speed:.2f} m/s, {sc.count} particles, {p.shape[0]} pairs (total {total})",
                  flush=True)
    return np.concatenate(chunks)[:n_pairs]


PAIR_LAYOUT = "F_hat[9] J_p F_E'[9] J_p'"  # one row of the pair log (float32)


def save_pair_shards(pairs: np.ndarray, directory, shard_rows: int = 1_000_000) -> list:
    """Write logged pairs as .npy shards of at most `shard_rows` rows (float32,
    (rows, 20)) plus index.json (row count, shard names, layout)."""
    import json
    from pathlib import Path
    d = Path(directory)
    d.mkdir(parents=True, exist_ok=True)
    pairs = np.ascontiguousarray(pairs, np.float32)
    if pairs.ndim != 2 or pairs.shape[1] != 20:
        raise ValueError("pairs must be (n, 20)")
    names = []
    for k, lo in enumerate(range(0, pairs.shape[0], shard_rows)):
        name = f"pairs_{k:05d}.npy"
        np.save(d / name, pairs[lo:lo + shard_rows])
        names.append(name)
    (d / "index.json").write_text(json.dumps({"rows": int(pairs.shape[0]), "shards": names, "layout": PAIR_LAYOUT,
                                              "dtype": "float32"}, indent=1))
    return names


def load_pair_shards(directory) -> np.ndarray:
    """All rows of a shard directory written by save_pair_shards, in order."""
    import json
    from pathlib import Path
    d = Path(directory)
    idx = json.loads((d / "index.json").read_text())
    if idx.get("layout") != PAIR_LAYOUT:
        raise ValueError(f"unknown pair layout {idx.get('layout')!r}")
    parts = [np.load(d / name, mmap_mode="r") for name in idx["shards"]]
    out = np.concatenate(parts) if parts else np.empty((0, 20), np.float32)
    if out.shape[0] != idx["rows"] or (out.ndim == 2 and out.shape[1] != 20):
        raise ValueError("pair shards do not match their index")
    return np.ascontiguousarray(out, np.float32)


def evaluate(mlp: Mlp, pairs: np.ndarray):
    """Relative error of the predicted F_E' against the exact one, per pair."""
    pred = mlp.predict(pairs)
    F_pred = pairs[:, :9].astype(np.float64) + pred[:, :9]
    F_true = pairs[:, 10:19].astype(np.float64)
    err = np.linalg.norm(F_pred - F_true, axis=1) / np.linalg.norm(F_true, axis=1)
    base = np.linalg.norm(pairs[:, :9] - F_true, axis=1) / np.linalg.norm(F_true, axis=1)
    return err, base


def train(pairs: np.ndarray, steps: int = 4000, batch: int = 8192, lr: float = 2e-3, seed: int = 0,
          holdout: float = 0.02):
    rng = np.random.Generator(np.random.PCG64(seed))
    perm = rng.permutation(pairs.shape[0])
    n_hold = max(1, int(holdout * pairs.shape[0]))
    test, tr = pairs[perm[:n_hold]], pairs[perm[n_hold:]]
    mlp = Mlp(seed)
    mlp.set_normalization(*normalization(tr))
    mlp.load_pairs(tr)
    t0 = time.perf_counter()
    loss = mlp.train(steps, batch=batch, lr=lr, seed=seed + 1)
    dt = time.perf_counter() - t0
    err, base = evaluate(mlp, test)
    return mlp, dict(loss=loss, train_seconds=dt, heldout_rel_err_median=float(np.median(err)),
                     heldout_rel_err_p99=float(np.percentile(err, 99)),
                     identity_rel_err_median=float(np.median(base)), n_train=int(tr.shape[0]),
                     n_test=int(test.shape[0]))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--pairs", type=int, default=50_000_000)
    ap.add_argument("--steps", type=int, default=60000)
    ap.add_argument("--batch", type=int, default=16384)
    ap.add_argument("--lr", type=float, default=4e-3)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS))
    ap.add_argument("--save-pairs", default=None, help="also write the collected pairs as shards to this directory")
    ap.add_argument("--load-pairs", default=None, help="train on the shards in this directory instead of collecting")
    ap.add_argument("--collision-pairs", type=int, default=0,
                    help="pairs from colliding-snowball runs (256^3) collected in addition to the impacts")
    ap.add_argument("--collision-grid", type=int, default=256)
    args = ap.parse_args(argv)
    _lib.load()
    t0 = time.perf_counter()
    if args.load_pairs:
        pairs = load_pair_shards(args.load_pairs)
        print(f"loaded {pairs.shape[0]} pairs in {time.perf_counter() - t0:.1f} s")
    else:
        pairs = collect_pairs(args.pairs, seed=args.seed)
        if args.collision_pairs > 0:
            coll = collect_pairs(args.collision_pairs, seed=args.seed + 1000, W=args.collision_grid,
                                 kind="collision", per_scene=5_000_000)
            pairs = np.concatenate([pairs, coll])
        print(f"collected {pairs.shape[0]} pairs in {time.perf_counter() - t0:.1f} s")
        if args.save_pairs:
            save_pair_shards(pairs, args.save_pairs)
    mlp, info = train(pairs, steps=args.steps, batch=args.batch, lr=args.lr, seed=args.seed)
    print({k: v for k, v in info.items() if k != "loss"}, "loss first/last", float(info["loss"][0]),
          float(info["loss"][-1]))
    from pathlib import Path
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    mlp.save(args.out)
    print("saved", args.out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
