"""Poisson-disk sampling on the host: the CPU restatement of the device
sampler against the minimum-distance property, the reference's own Bridson
samplers (src/shared/Shapes.h, built into oracle/_ref when the reference tree
is present) and the C ABI's argument checks."""
import ctypes as C
import json
import subprocess

import numpy as np
import pytest
from scipy.spatial import cKDTree

from oracle import sample_ref
from oracle.build_oracle import POISSON

MD2 = float(np.float32(15.0) / np.sqrt(np.float32(3000.0)))   # radius / sqrt(NUM_PARTICLES), GPUSolver.cpp:142
MD3 = float(np.float32(15.0) / np.cbrt(np.float32(3000.0)))   # radius / cbrt(NUM_PARTICLES), GPUSolver.cpp:112


def _ball(c, r):
    return dict(kind=sample_ref.BALL, center=tuple(c) + (0.0,) * (3 - len(c)), radius=float(r), half=(0.0,) * 3)


def _box(c, h):
    return dict(kind=sample_ref.BOX, center=tuple(c) + (0.0,) * (3 - len(c)), radius=0.0,
                half=tuple(h) + (0.0,) * (3 - len(h)))


def _min_dist(p):
    d, _ = cKDTree(p.astype(np.float64)).query(p.astype(np.float64), k=2)
    return float(d[:, 1].min())


def _ref_count(dim, md):
    exe = POISSON[dim]
    if not exe.exists():
        pytest.skip(f"{exe.name} not built (needs the reference tree)")
    args = ["50", "45", "15", f"{md:.9g}"] if dim == 2 else ["50", "45", "50", "15", f"{md:.9g}"]
    counts = []
    for _ in range(3):  # std::random_device seeds it: a few runs
        out = json.loads(subprocess.run([str(exe)] + args, capture_output=True, text=True, check=True).stdout)
        assert out["min_dist"] >= md * (1 - 1e-5)
        counts.append(out["count"])
    return float(np.mean(counts))


def test_oracle_2d_reference_ball_properties():
    p, owner = sample_ref.sample_shapes(2, [_ball((50, 45), 15)], MD2, seed=1)
    assert _min_dist(p) >= MD2 * (1 - 1e-6)
    assert (owner == 0).all()
    assert (np.linalg.norm(p - [50, 45], axis=1) <= 15 * (1 + 1e-6)).all()
    # no hole: every probe inside the disc lies within 2 min_dist of a sample
    rng = np.random.default_rng(0)
    q = rng.uniform(-1, 1, (20000, 2))
    q = 50 + 15 * 0.98 * q[(q ** 2).sum(1) <= 1] + [0, -5]
    d, _ = cKDTree(p).query(q)
    assert d.max() < 2 * MD2


def test_oracle_against_reference_bridson_counts():
    """Same shape, same min_dist: the dart thrower packs a few percent denser
    than Bridson's k=30 sampler (its 3^dim phases visit every cell 30 times);
    the reference's scene normalises volume by the count, so the mass per ball
    is the same either way."""
    ref = _ref_count(2, MD2)
    p, _ = sample_ref.sample_shapes(2, [_ball((50, 45), 15)], MD2, seed=1)
    ratio = p.shape[0] / ref
    print(f"2D: device sampler {p.shape[0]}, reference Bridson {ref:.0f}, ratio {ratio:.3f}")
    assert 1.0 <= ratio <= 1.15


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_union_determinism_and_seed(dim):
    md = 0.9
    shapes = [_ball((4.0,) * dim, 3.0), _box((8.0,) + (4.0,) * (dim - 1), (2.0,) + (1.5,) * (dim - 1))]
    a, oa = sample_ref.sample_shapes(dim, shapes, md, seed=7, rounds=20)
    b, ob = sample_ref.sample_shapes(dim, shapes, md, seed=7, rounds=20)
    c, _ = sample_ref.sample_shapes(dim, shapes, md, seed=8, rounds=20)
    assert np.array_equal(a, b) and np.array_equal(oa, ob)
    assert a.shape != c.shape or not np.array_equal(a, c)
    assert _min_dist(a) >= md * (1 - 1e-6)
    assert set(np.unique(oa)) == {0, 1}
    # a sample belongs to the first shape that contains it
    in_ball = np.linalg.norm(a - 4.0, axis=1) <= 3.0
    assert (oa[in_ball] == 0).all() and (oa[~in_ball] == 1).all()


def test_c_abi_argument_checks():
    """Invalid arguments are refused before any device work (no GPU needed)."""
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200.build import build
    build()
    lib = _lib.load()
    sh = (_lib.MpmShape * 1)()
    sh[0].kind = _lib.SHAPE_BALL
    sh[0].radius = 1.0
    cnt = C.c_int64(-1)
    bad = [
        (4, sh, 1, 0.1, 30),     # dim
        (2, sh, 0, 0.1, 30),     # no shapes
        (2, sh, 1, 0.0, 30),     # min_dist
        (2, sh, 1, float("nan"), 30),
        (2, sh, 1, 0.1, 0),      # rounds
    ]
    for dim, shapes, n, md, rounds in bad:
        st = lib.mpm_sample_shapes(dim, shapes, n, md, 1, rounds, None, None, 0, C.byref(cnt))
        assert _lib.STATUS_NAMES[st] == "MPM_ERR_INVALID_ARGUMENT"
    sh[0].kind = 7
    assert _lib.STATUS_NAMES[lib.mpm_sample_shapes(2, sh, 1, 0.1, 1, 30, None, None, 0, C.byref(cnt))] == "MPM_ERR_INVALID_ARGUMENT"
    sh[0].kind = _lib.SHAPE_BALL
    sh[0].radius = -1.0
    assert lib.mpm_sample_shapes(2, sh, 1, 0.1, 1, 30, None, None, 0, C.byref(cnt)) != 0
    # positions required when capacity > 0
    sh[0].radius = 1.0
    assert lib.mpm_sample_shapes(2, sh, 1, 0.1, 1, 30, None, None, 5, C.byref(cnt)) != 0


def test_capacity_bound_covers_oracle():
    from mpm_snow_sim2d_b200.sampling import _capacity_bound, ball
    for dim, md in ((2, MD2), (2, 0.5), (3, 1.3)):
        shapes = [ball((50, 45, 50)[:dim], 15)]
        p, _ = sample_ref.sample_shapes(dim, [_ball((50, 45, 50)[:dim], 15)], md, seed=3, rounds=10 if dim == 3 else 30)
        assert p.shape[0] <= _capacity_bound(dim, shapes, md)
