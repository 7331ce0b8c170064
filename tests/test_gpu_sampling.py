"""Device Poisson-disk sampling (mpm_sample_shapes) against its CPU
restatement, bit for bit, and the reference's default two-snowball scene
built on it, stepped on the GPU against the FP64 oracle."""
import numpy as np
import pytest

from conftest import state_errors
from oracle import sample_ref

pytestmark = pytest.mark.gpu

MD2 = float(np.float32(15.0) / np.sqrt(np.float32(3000.0)))


def _shape(kind, c, r=0.0, h=(0.0, 0.0, 0.0)):
    return dict(kind=kind, center=tuple(c) + (0.0,) * (3 - len(c)), radius=float(r),
                half=tuple(h) + (0.0,) * (3 - len(h)))


CASES = {
    "ref_ball_2d": (2, [_shape(0, (50, 45), 15)], MD2, 1, 30),
    "union_2d": (2, [_shape(0, (20, 20), 8), _shape(1, (33, 18), h=(6, 4)), _shape(0, (26, 30), 5)], 0.4, 99, 30),
    "ball_box_3d": (3, [_shape(0, (10, 10, 10), 6), _shape(1, (19, 9, 10), h=(4, 3, 5))], 0.8, 5, 20),
}


@pytest.mark.parametrize("case", sorted(CASES))
def test_device_sampler_matches_restatement_bitwise(gpu_lib, case):
    from mpm_snow_sim2d_b200.sampling import sample_shapes
    dim, shapes, md, seed, rounds = CASES[case]
    got, owner = sample_shapes(dim, shapes, md, seed, rounds)
    ref, ref_owner = sample_ref.sample_shapes(dim, shapes, md, seed, rounds)
    print(f"{case}: {got.shape[0]} samples (restatement {ref.shape[0]})")
    assert got.shape == ref.shape
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))
    assert np.array_equal(owner, ref_owner)
    # determinism and seed dependence
    again, _ = sample_shapes(dim, shapes, md, seed, rounds)
    assert np.array_equal(again.view(np.uint32), got.view(np.uint32))
    other, _ = sample_shapes(dim, shapes, md, seed + 1, rounds)
    assert other.shape != got.shape or not np.array_equal(other, got)


def test_device_sampler_capacity_and_errors(gpu_lib):
    import ctypes as C
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200.sampling import _pack
    lib = gpu_lib
    shapes = _pack([_shape(0, (0, 0), 3)])
    pos = np.empty((10, 2), np.float32)
    cnt = C.c_int64(0)
    st = lib.mpm_sample_shapes(2, shapes, 1, 0.3, 4, 30, _lib.fptr(pos), None, 10, C.byref(cnt))
    assert _lib.STATUS_NAMES[st] == "MPM_ERR_CAPACITY" and cnt.value > 10
    full = np.empty((cnt.value, 2), np.float32)
    st = lib.mpm_sample_shapes(2, shapes, 1, 0.3, 4, 30, _lib.fptr(full), None, cnt.value, C.byref(cnt))
    assert st == 0 and np.array_equal(full[:10], pos)
    # a background grid beyond 4e8 cells is refused, not allocated
    st = lib.mpm_sample_shapes(3, _pack([_shape(1, (0, 0, 0), h=(100, 100, 100))]), 1, 0.1, 1, 1, None, None, 0,
                               C.byref(cnt))
    assert _lib.STATUS_NAMES[st] == "MPM_ERR_CAPACITY"


@pytest.mark.parametrize("dim,steps", [(2, [1, 300, 1000]), (3, [1, 100])])
def test_reference_default_scene_against_oracle(gpu_lib, oracle_mod, dim, steps):
    """The reference's own scene (two snowballs of radius 15 at +-40 cells/s on a
    200 x 100 [x 100] grid, dt 1e-3) sampled on the device, stepped through the
    C ABI and compared with the FP64 oracle; in 2D the balls meet near step 875."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.reference_snowballs(dim, seed=11)
    n1, n2 = sc.info["per_ball"]
    vol1 = float(sc.volume[:n1].sum())
    want = 2 * 3.1415926 * 15 ** 2 if dim == 2 else 4 / 3 * 3.1415926 * 15 ** 3
    assert abs(vol1 - want) / want < 1e-4
    assert (sc.velocity[:n1, 0] == 40).all() and (sc.velocity[n1:, 0] == -40).all()
    from test_gpu_parity import TIGHT, TARGET, _check, _check_vs_fp32_reference, _fp32_reference_errors, _oracle_ref
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, prev = {}, 0
    with Solver.from_scene(sc) as solver:
        for s in steps:
            solver.Step(s - prev)
            prev = s
            got[s] = solver.get_state()
        assert solver.status() & 1 == 0
    # past the collision the bar is the reference's own FP32 arithmetic's
    # distance from FP64 (x1.5, never looser than 1e-4)
    r32 = _fp32_reference_errors(oracle_mod, sc, steps)
    _check_vs_fp32_reference(state_errors(got[1], ref[1], dim), r32[1], f"{dim}D step 1", TIGHT)
    for s in steps[1:]:
        _check_vs_fp32_reference(state_errors(got[s], ref[s], dim), r32[s], f"{dim}D step {s}", TARGET)


def test_reference_default_scene_matches_golden_fixture(gpu_lib):
    """The fixture refcpu_reference_default2d was made without a GPU from the
    sampler's CPU restatement; the device must draw the same particles."""
    from golden_io import load_case
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.reference_snowballs(2, seed=11)
    golden, _ = load_case("refcpu_reference_default2d")
    assert np.array_equal(sc.position.view(np.uint32), golden.position.view(np.uint32))
    assert np.array_equal(sc.volume, golden.volume) and np.array_equal(sc.velocity, golden.velocity)


def test_batch_scenes_with_device_sampling(gpu_lib):
    """The batched workload's blocks filled by the device Poisson-disk sampler:
    the same blocks and mean density as the uniform draw, the same mass per
    scene, at least min_dist between particles; the batch steps them cleanly."""
    from scipy.spatial import cKDTree
    from mpm_snow_sim2d_b200 import scenes
    from mpm_snow_sim2d_b200.batch import Batch
    pois = [scenes.batch_scene_2d(i, steps=50, sampler="poisson") for i in range(4)]
    unif = [scenes.batch_scene_2d(i, steps=50) for i in range(4)]
    for p, u in zip(pois, unif):
        assert (p.width, p.info["blocks"]) == (u.width, u.info["blocks"])
        ratio = p.count / u.count
        assert 0.85 < ratio < 1.15, ratio
        assert abs(float(p.mass.astype(np.float64).sum()) / float(u.mass.astype(np.float64).sum()) - 1) < 1e-3
        md = float(np.sqrt(scenes.POISSON_DENSITY_2D / int(u.name.split("ppc")[1])))
        d, _ = cKDTree(p.position.astype(np.float64)).query(p.position.astype(np.float64), k=2)
        assert d[:, 1].min() >= md * (1 - 1e-5)
        again = scenes.batch_scene_2d(0, steps=50, sampler="poisson")
    assert np.array_equal(again.position, pois[0].position)
    with Batch(pois) as b:
        b.step(50)
        assert all(b.status(k) & 1 == 0 for k in range(len(pois)))
