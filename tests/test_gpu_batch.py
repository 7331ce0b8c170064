"""Batched 2D scenes on the GPU, through the C ABI (mpm_batch_*): scenes of a
mixed batch (grids of 64 to 256 cells, clusters of 1 to 8 CTAs) against the
FP64 oracle and the single-scene solver; a scene's result independent of its
cluster size and of the other scenes (bitwise); determinism; the autotuner;
state round trips; errors."""
import ctypes as C

import numpy as np
import pytest

from conftest import state_errors
from test_gpu_parity import TARGET, _check, _check_vs_fp32_reference, _fp32_reference_errors

pytestmark = pytest.mark.gpu


def _mixed_scenes(k=8, steps=100):
    """k scenes of the batched workload spanning its grid sizes."""
    from mpm_snow_sim2d_b200 import scenes
    pool = [scenes.batch_scene_2d(i, steps=steps) for i in range(48)]
    pool.sort(key=lambda s: s.width)
    idx = np.linspace(0, len(pool) - 1, k).round().astype(int)
    return [pool[i] for i in idx]


def _states(b, k):
    return [b.get_state(s) for s in range(k)]


def _as_ref(st):
    return dict(position=st.position, velocity=st.velocity, affine_b=st.affine_b, elastic_f=st.elastic_f,
                plastic_det=st.plastic_det)


def _equal(a, b):
    return all(np.array_equal(getattr(a, f), getattr(b, f))
               for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_det"))


def test_batch_scenes_match_oracle_and_single_solver(gpu_lib, oracle_mod):
    from mpm_snow_sim2d_b200 import Solver
    from mpm_snow_sim2d_b200.batch import Batch
    scs = _mixed_scenes()
    assert min(s.width for s in scs) < 100 and max(s.width for s in scs) > 200
    with Batch(scs) as b:
        b.step(100)
        got = _states(b, len(scs))
        flags = [b.status(s) for s in range(len(scs))]
    for s, sc in enumerate(scs):
        assert flags[s] & 3 == 0, (s, flags[s])
        with Solver.from_scene(sc) as single:
            single.Step(100)
            one = single.get_state()
        errs = state_errors(got[s], _as_ref(one), 2)
        print(f"scene {sc.name} ({sc.count} particles) vs single-scene solver:",
              {k: f"{v:.1e}" for k, v in errs.items()})
        _check(errs, TARGET, f"{sc.name} vs single-scene solver")
    # the smallest, a middle and the largest scene against the FP64 oracle
    for s in (0, len(scs) // 2, len(scs) - 1):
        sc = scs[s]
        st = oracle_mod.initial_state(sc)
        oracle_mod.run_oracle(sc, st, 100)
        ref = dict(position=st.position, velocity=st.velocity, affine_b=st.affine_b, elastic_f=st.elastic_f,
                   plastic_det=st.plastic_det)
        errs = state_errors(got[s], ref, 2)
        ref32 = _fp32_reference_errors(oracle_mod, sc, [100])[100]
        print(f"scene {sc.name} vs FP64 oracle:", {k: f"{v:.1e}" for k, v in errs.items()})
        _check_vs_fp32_reference(errs, ref32, f"{sc.name} vs FP64 oracle")


def test_scene_result_independent_of_cluster_and_partners(gpu_lib):
    """Bitwise, for each kernel width: the int64 sums are exact and every
    particle's arithmetic is its own, so neither the cluster size, nor the
    particle order, nor the other scenes change a scene's result. (Kernels of
    different widths are compiled under different register limits and may
    contract multiply-adds differently: equal within FP32 rounding.)"""
    from mpm_snow_sim2d_b200.batch import Batch
    scs = _mixed_scenes(k=6, steps=40)
    per_width = {}
    for threads in (512, 1024):
        with Batch(scs) as b:
            b.set_config(particles_per_cta=0, threads=threads)
            b.step(40)
            base = _states(b, len(scs))
        with Batch(scs) as b:
            b.set_config(particles_per_cta=1024, threads=threads)  # every scene on more CTAs
            b.step(25)
            b.step(15)
            spread = _states(b, len(scs))
        for s in range(len(scs)):
            assert _equal(base[s], spread[s]), f"scene {s} changed with its cluster size ({threads} threads)"
        with Batch([scs[-1]]) as b:  # the largest scene alone
            b.set_config(threads=threads)
            b.step(40)
            alone = b.get_state(0)
        assert _equal(alone, base[-1])
        per_width[threads] = base
    for s in range(len(scs)):
        errs = state_errors(per_width[1024][s], _as_ref(per_width[512][s]), 2)
        _check(errs, dict(x=1e-6, v=1e-5, B=1e-5, F=1e-6, Jp=1e-6), f"scene {s}, 1024 vs 512 threads")


@pytest.mark.parametrize("threads", [512, 1024])
def test_batch_determinism_and_state_roundtrip(gpu_lib, threads):
    from mpm_snow_sim2d_b200.batch import Batch
    scs = _mixed_scenes(k=4, steps=30)
    runs = []
    for rt in range(2):
        with Batch(scs) as b:
            b.set_config(threads=threads)
            b.step(10)
            if rt:
                for s in range(len(scs)):  # upload what was read: continues unchanged
                    st = b.get_state(s)
                    b.set_state(s, st.position, st.velocity, st.affine_b, st.elastic_f, st.plastic_det)
            b.step(20)
            runs.append(_states(b, len(scs)))
    for s in range(len(scs)):
        assert _equal(runs[0][s], runs[1][s]), f"scene {s}"


def test_autotuner_keeps_the_state(gpu_lib):
    from mpm_snow_sim2d_b200.batch import Batch
    scs = _mixed_scenes(k=6, steps=20)
    with Batch(scs) as b:
        before = _states(b, len(scs))
        cfg, ms = b.tune(3)
        assert cfg["threads"] in (256, 512, 1024) and ms > 0
        assert b.config == cfg
        after = _states(b, len(scs))
        b.step(20)
        got = _states(b, len(scs))
    for s in range(len(scs)):
        assert _equal(before[s], after[s]), f"scene {s}: the tuner left its trial steps behind"
    with Batch(scs) as b:  # the chosen configuration from the start: same run, bitwise
        b.set_config(**cfg)
        b.step(20)
        ref = _states(b, len(scs))
    for s in range(len(scs)):
        assert _equal(ref[s], got[s]), f"scene {s}"


def test_step_times_and_errors(gpu_lib):
    from mpm_snow_sim2d_b200 import scenes
    from mpm_snow_sim2d_b200._lib import MpmError
    from mpm_snow_sim2d_b200.batch import Batch
    scs = _mixed_scenes(k=3, steps=10)
    with Batch(scs) as b:
        b.step(10)
        t = b.step_times()
        assert t.shape == (3, 11)
        assert np.all(t > 0) and np.all(np.diff(t.astype(np.int64), axis=1) >= 0)
        with pytest.raises(MpmError) as e:
            b.set_config(threads=384)
        assert e.value.status == 1
        out = np.empty(8, np.float32)
        assert b._lib.mpm_batch_get_positions(b._h, 3, out.ctypes.data_as(C.POINTER(C.c_float)), 8) == 1
        assert b._lib.mpm_batch_get_positions(b._h, 0, out.ctypes.data_as(C.POINTER(C.c_float)), 8) == 11
    big = scenes.batch_scene_2d(0).with_(width=400, height=400)  # 401^2 nodes: beyond 8 CTAs
    with pytest.raises(MpmError) as e:
        Batch([big])
    assert e.value.status == 11
    with pytest.raises(ValueError):
        Batch([scenes.impact_3d()])
