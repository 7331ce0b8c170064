"""GPU parity: the CUDA solver, called through the C ABI, against the FP64
oracle (MLS, 2D and 3D) and against the reference's own CPU code (CLASSIC,
golden fixtures), plus determinism, conservation and the API contract.

Tolerances are relative L2 norms over all particles (B normalised by the
velocity norm, see conftest.state_errors). The workload target is 1e-4 after
1000 steps; short horizons are held much tighter."""
import numpy as np
import pytest

from conftest import state_errors
from golden_io import load_case

pytestmark = pytest.mark.gpu


def _oracle_ref(O, scene, steps, formulation=None):
    st = O.initial_state(scene)
    out, prev = {}, 0
    for s in steps:
        O.run_oracle(scene, st, s - prev, formulation=formulation)
        prev = s
        out[s] = dict(position=st.position.copy(), velocity=st.velocity.copy(), affine_b=st.affine_b.copy(),
                      elastic_f=st.elastic_f.copy(), plastic_det=st.plastic_det.copy())
    return out


def _gpu_run(scene, steps, **kw):
    from mpm_snow_sim2d_b200 import Solver
    out, prev = {}, 0
    with Solver.from_scene(scene, **kw) as s:
        for st in steps:
            s.Step(st - prev)
            prev = st
            out[st] = s.get_state()
        flags = s.status()
    return out, flags


def _check(errs, tol, label):
    print(f"{label}: " + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    for k, v in errs.items():
        assert v <= tol[k], f"{label}: {k} rel-L2 {v:.3e} > {tol[k]:.1e} (all: { {a: f'{b:.2e}' for a, b in errs.items()} })"


TIGHT = dict(x=1e-6, v=1e-5, B=1e-5, F=1e-6, Jp=1e-6)
TARGET = dict(x=1e-4, v=1e-4, B=1e-4, F=1e-4, Jp=1e-4)


def _fp32_reference_errors(O, scene, steps):
    """Distance of the reference step evaluated in FP32 (the oracle's float
    instantiation, same operation order as the shaders) from FP64."""
    a, b = O.initial_state(scene), O.initial_state(scene, np.float32)
    out, prev = {}, 0
    for s in steps:
        O.run_oracle(scene, a, s - prev)
        O.run_oracle(scene, b, s - prev, fp32=True)
        prev = s

        class S:
            position, velocity, affine_b, elastic_f, plastic_det = b.position, b.velocity, b.affine_b, b.elastic_f, b.plastic_det
        out[s] = state_errors(S, dict(position=a.position, velocity=a.velocity, affine_b=a.affine_b,
                                      elastic_f=a.elastic_f, plastic_det=a.plastic_det), scene.dim)
    return out


def _check_vs_fp32_reference(errs, ref32, label, floor=TARGET):
    """After contact, velocities approach zero and relative errors grow: the bar
    is twice the reference's own FP32 arithmetic's distance from FP64 (the
    oracle's FP32 instantiation reproduces the reference's shaders bit for
    bit, tests/test_shader_pin.py), never tighter than `floor`. Two FP32
    implementations that sum in different orders land on different sides of
    wall-contact and clamping branches for a few particles, which moves these
    distances by tens of percent either way (the same factor 2 bounds the
    CLASSIC path against the reference's compiled CPU code)."""
    tol = {k: max(floor[k], 2.0 * ref32[k]) for k in errs}
    _check(errs, tol, label)


def test_mls_2d_blocks_1000_steps(gpu_lib, oracle_mod):
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.snow_blocks_2d()          # the 128^2 three-block workload, 4425 particles
    steps = [1, 10, 100, 1000]
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, flags = _gpu_run(sc, steps)
    assert flags & 1 == 0
    r32 = _fp32_reference_errors(oracle_mod, sc, [1])
    _check_vs_fp32_reference(state_errors(got[1], ref[1], 2), r32[1], "step 1", TIGHT)
    for s in (100, 1000):
        _check(state_errors(got[s], ref[s], 2), TARGET, f"step {s}")


def test_mls_2d_impact(gpu_lib, oracle_mod):
    """Contact, friction and plastic flow (J_p leaves 1)."""
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.impact_2d()
    steps = [1, 100, 400]
    ref = _oracle_ref(oracle_mod, sc, steps)
    assert ref[400]["plastic_det"].min() < 0.99
    got, flags = _gpu_run(sc, steps)
    r32 = _fp32_reference_errors(oracle_mod, sc, [1, 100, 400])
    _check_vs_fp32_reference(state_errors(got[1], ref[1], 2), r32[1], "step 1", TIGHT)
    _check_vs_fp32_reference(state_errors(got[100], ref[100], 2), r32[100], "step 100")
    _check_vs_fp32_reference(state_errors(got[400], ref[400], 2), r32[400], "step 400")


def test_mls_3d_impact(gpu_lib, oracle_mod):
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.impact_3d()
    steps = [1, 100, 300]
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, flags = _gpu_run(sc, steps)
    assert flags & 1 == 0
    r32 = _fp32_reference_errors(oracle_mod, sc, [1, 100, 300])
    _check_vs_fp32_reference(state_errors(got[1], ref[1], 3), r32[1], "step 1", TIGHT)
    _check_vs_fp32_reference(state_errors(got[100], ref[100], 3), r32[100], "step 100")
    _check_vs_fp32_reference(state_errors(got[300], ref[300], 3), r32[300], "step 300")


def test_mls_3d_snowball_slab_1000_steps(gpu_lib, oracle_mod):
    """The snowball-on-slab workload at reduced resolution (32^3, 1 ppc)."""
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.snowball_on_slab_3d(W=32, ppc=1)
    steps = [1, 1000]
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, _ = _gpu_run(sc, steps)
    r32 = _fp32_reference_errors(oracle_mod, sc, [1, 1000])
    _check_vs_fp32_reference(state_errors(got[1], ref[1], 3), r32[1], "step 1", TIGHT)
    # the slab rests on the floor: the wall-contact branch (grid_update.glsl:54)
    # flips for a few nodes between FP32 and FP64, which the reference's own FP32
    # arithmetic shows too (its velocity error here is ~2.4e-4).
    _check_vs_fp32_reference(state_errors(got[1000], ref[1000], 3), r32[1000], "step 1000")


# Floor of the GPU's FP64 distance per case. On the reference's default scene
# the two balls fly freely for ~875 steps, F stays within ~4e-7 of I, and the
# relative F distance after 500 steps is FP32 rounding accumulated in F (GPU
# 4.4e-6, the reference's own FP32 code 1.0e-6): both far inside the 1e-4 bar.
CLASSIC_FLOOR = {"refcpu_reference_default2d": 1e-5}


@pytest.mark.parametrize("case", ["refcpu_blocks2d_ppc1", "refcpu_impact2d", "refcpu_reference_default2d"])
def test_classic_matches_reference_cpu(gpu_lib, oracle_mod, case):
    """CLASSIC formulation vs the reference's compiled src/cpu (golden fixtures).
    Both are FP32 with different operation order; each is held to the FP64
    oracle, and to the reference within the sum of their FP64 distances."""
    from mpm_snow_sim2d_b200._lib import FORMULATION_CLASSIC
    scene, dumps = load_case(case)
    steps = sorted(dumps)
    got, _ = _gpu_run(scene, steps, formulation=FORMULATION_CLASSIC)
    f64 = _oracle_ref(oracle_mod, scene, steps, formulation=oracle_mod.CLASSIC)
    for s in steps:
        ref = dict(dumps[s])
        e_gpu = state_errors(got[s], f64[s], 2)

        class R:  # reference dump as a state
            position, velocity, affine_b, elastic_f = ref["position"], ref["velocity"], ref["affine_b"], ref["elastic_f"]
            plastic_det = np.linalg.det(ref["plastic_f"].astype(np.float64))
        e_ref = state_errors(R, f64[s], 2)
        e_pair = state_errors(got[s], dict(ref, plastic_det=R.plastic_det), 2)
        print(f"{case} step {s}: gpu-fp64 " + ", ".join(f"{k} {v:.2e}" for k, v in e_gpu.items()) +
              " | reference-fp64 " + ", ".join(f"{k} {v:.2e}" for k, v in e_ref.items()))
        floor = CLASSIC_FLOOR.get(case, 2e-6)
        for k in e_gpu:
            assert e_gpu[k] <= max(2.0 * e_ref[k], floor), f"step {s} {k}: gpu {e_gpu[k]:.2e} vs reference {e_ref[k]:.2e}"
            assert e_pair[k] <= 2.0 * (e_gpu[k] + e_ref[k]) + 1e-6, f"step {s} {k}: {e_pair[k]:.2e}"
        if s == 1:
            _check(e_pair, dict(x=1e-6, v=1e-5, B=1e-5, F=1e-6, Jp=1e-6), "step 1 vs reference")


@pytest.mark.parametrize("case", ["impact3d", "dense3d", "dense2d"])
def test_run_to_run_bitwise_determinism(gpu_lib, case):
    """Bit-identical grid sums and particle state across runs. dense3d has
    ~1000 particles per 4^3 tile (counting sort and, above 1024, the bitonic
    network in shared memory); dense2d has >4032 particles per 8^2 tile (sorted
    in global memory)."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = {"impact3d": lambda: scenes.impact_3d(),
          "dense3d": lambda: scenes.snowball_on_slab_3d(W=32, ppc=16),
          "dense2d": lambda: scenes.impact_2d(W=16, ppc=1000)}[case]()
    outs = []
    for _ in range(2):
        with Solver.from_scene(sc) as s:
            s.Step(40)
            m, p, raw = s.rasterize(raw=True)
            st = s.get_state()
            outs.append((raw, st))
    (r0, s0), (r1, s1) = outs
    assert np.array_equal(r0, r1)
    for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_det"):
        assert np.array_equal(getattr(s0, f), getattr(s1, f)), f


@pytest.mark.parametrize("dim", [2, 3])
def test_p2g_conservation(gpu_lib, dim):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.impact_2d() if dim == 2 else scenes.impact_3d()
    with Solver.from_scene(sc) as s:
        s.Step(60)
        st = s.get_state()
        m, p = s.rasterize()
    total = float(sc.mass.astype(np.float64).sum())
    # FP32 B-spline weights sum to 1 within a few ulps (as in the reference)
    assert abs(m.sum() - total) <= 1e-6 * total
    mom = (sc.mass.astype(np.float64)[:, None] * st.velocity.astype(np.float64)).sum(0)
    scale = (sc.mass.astype(np.float64)[:, None] * np.abs(st.velocity)).sum()
    assert np.all(np.abs(p.sum(0) - mom) <= 1e-5 * scale)


def test_rest_state_stays_at_rest(gpu_lib):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.snow_blocks_2d().with_(gravity=0.0)
    sc = sc.with_(velocity=np.zeros_like(sc.velocity))
    with Solver.from_scene(sc) as s:
        s.Step(50)
        st = s.get_state()
    assert np.array_equal(st.position, sc.position)
    assert not np.any(st.velocity)
    assert np.array_equal(st.elastic_f, np.broadcast_to(np.eye(2, dtype=np.float32), st.elastic_f.shape))


def test_free_fall_is_exact(gpu_lib):
    """Uniform fall, no wall in reach: v = v0 + g t, x quadratic in t."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.snow_blocks_2d(steps=100)
    sc = sc.with_(velocity=np.tile(np.float32([0.0, -50.0]), (sc.count, 1)))
    with Solver.from_scene(sc) as s:
        s.Step(100)
        st = s.get_state()
    t = 100 * sc.delta_time
    v_exp = -50.0 + sc.gravity * t
    inner = np.median(st.velocity[:, 1])
    assert abs(inner - v_exp) < 1e-4 * abs(v_exp)
    dy = np.median(st.position[:, 1] - sc.position[:, 1])
    y_exp = sum((-50.0 + sc.gravity * sc.delta_time * (k + 1)) * sc.delta_time for k in range(100))
    assert abs(dy - y_exp) < 1e-3 * abs(y_exp)


def test_positions_state_checkpoint_roundtrip(gpu_lib, tmp_path):
    from mpm_snow_sim2d_b200 import MpmError, Solver, scenes
    sc = scenes.impact_2d()
    with Solver.from_scene(sc) as a:
        a.Step(30)
        a.save(tmp_path / "ck.bin")
        pos = a.GetParticlePositions()
        a.Step(20)
        end = a.get_state()
    assert pos.shape == (sc.count, 2)
    with Solver.from_scene(sc) as b:
        b.load(tmp_path / "ck.bin")
        assert b.step_count == 30
        assert np.array_equal(b.GetParticlePositions(), pos)
        b.Step(20)
        again = b.get_state()
    for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_det"):
        assert np.array_equal(getattr(end, f), getattr(again, f)), f
    # a checkpoint from another configuration is refused
    other = scenes.impact_2d(W=64)
    with Solver.from_scene(other) as c:
        with pytest.raises(MpmError) as ei:
            c.load(tmp_path / "ck.bin")
        assert ei.value.status == 8
    # a truncated file is refused without touching the state
    raw = (tmp_path / "ck.bin").read_bytes()
    (tmp_path / "bad.bin").write_bytes(raw[: len(raw) // 2])
    with Solver.from_scene(sc) as d:
        with pytest.raises(MpmError) as ei:
            d.load(tmp_path / "bad.bin")
        assert ei.value.status == 7


def test_api_errors_and_flags(gpu_lib):
    import ctypes as C
    from mpm_snow_sim2d_b200 import MpmError, Solver, scenes
    lib = gpu_lib
    sc = scenes.impact_2d()
    with Solver.from_scene(sc) as s:
        small = np.empty(3, np.float32)
        rc = lib.mpm_get_positions(s._h, small.ctypes.data_as(C.POINTER(C.c_float)), 3)
        assert rc == 11 and b"capacity" in lib.mpm_last_error(s._h)
        with pytest.raises(MpmError):
            s.Step(-1)
        assert s.status() & 1 == 0
        # a NaN injected into the state is reported through the status word, no trap
        st = s.get_state()
        st.position[5] = np.nan
        s.set_state(position=st.position)
        s.Step(1)
        assert s.status() & 1
    with pytest.raises(MpmError) as ei:
        Solver.from_scene(sc.with_(position=np.full_like(sc.position, np.nan)))
    assert ei.value.status == 1


def test_set_stream_and_external_events(gpu_lib):
    import torch
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.impact_2d()
    stream = torch.cuda.Stream()
    with Solver.from_scene(sc) as s:
        s.set_stream(stream.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        s.Step(10)
        e1.record(stream)
        e1.synchronize()
        assert e0.elapsed_time(e1) > 0
        assert s.step_count == 10


@pytest.mark.parametrize("dim", [2, 3])
def test_stale_tile_order_matches_oracle(gpu_lib, oracle_mod, dim):
    """Particles drift away from the tile order of the last sort: with the
    re-sort disabled, drifters beyond the one-cell margin take the
    per-particle path and results still match the oracle."""
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.impact_2d(steps=150) if dim == 2 else scenes.impact_3d(steps=150)
    steps = [150]
    ref = _oracle_ref(oracle_mod, sc, steps)
    r32 = _fp32_reference_errors(oracle_mod, sc, steps)
    got, flags = _gpu_run(sc, steps, sort_period=100000)
    assert flags & 1 == 0
    _check_vs_fp32_reference(state_errors(got[150], ref[150], dim), r32[150], "step 150")


def test_auto_sort_period(gpu_lib):
    """sort_period 0: each period is the longest of {4, 6, 8, 12, 16, 24, 32}
    steps over which the fastest particle moves at most a quarter cell."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    slow = scenes.snow_blocks_2d(steps=100).with_(gravity=0.0)
    slow = slow.with_(velocity=np.tile(np.float32([0.0, -50.0]), (slow.count, 1)))  # 0.005 cells/step
    with Solver.from_scene(slow) as s:
        s.Step(64)
        sorts, period = s.sort_stats()
    assert period == 32 and sorts == 2
    mid = slow.with_(velocity=np.tile(np.float32([0.0, -180.0]), (slow.count, 1)))  # 0.018: 12 steps, 0.22 cells
    with Solver.from_scene(mid) as s:
        s.Step(48)
        sorts, period = s.sort_stats()
    assert period == 12 and sorts == 4
    fast = scenes.impact_2d()  # up to ~4.1 m/s on a 128 grid, dt 1e-4: ~0.052 cells/step
    with Solver.from_scene(fast) as s:
        s.Step(40)
        sorts, period = s.sort_stats()
    assert period == 4 and sorts == 10
    # a fixed period is kept as given
    with Solver.from_scene(fast, sort_period=16) as s:
        s.Step(40)
        sorts, period = s.sort_stats()
    assert period == 16 and sorts == 3
