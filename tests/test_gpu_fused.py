"""The fused transfer (G2P of a step and the next step's P2G in one kernel per
cell tile) against the split kernels and itself: same results to FP32
rounding, bit-identical resume from a checkpoint taken while particles are on
the queued-window scatter path, and pending grid sums equal to a fresh P2G of the
same state. The oracle parity tests in test_gpu_parity.py run the fused path
(the default) as well."""
import os

import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

FIELDS = ("position", "velocity", "affine_b", "elastic_f", "plastic_det")


def _run(scene, steps, transfer, box_load="gather", **kw):
    from mpm_snow_sim2d_b200 import Solver
    env = {"MPM_TRANSFER": transfer, "MPM_BOX_LOAD": box_load}
    old = {k: os.environ.get(k) for k in env}
    os.environ.update(env)
    try:
        with Solver.from_scene(scene, **kw) as s:
            s.Step(steps)
            st = s.get_state()
            flags = s.status()
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v
    return st, flags


def _scenes():
    from mpm_snow_sim2d_b200 import _lib, scenes
    quad = dict(formulation=_lib.FORMULATION_MLS_QUADRATIC)
    return {
        "impact2d": (scenes.impact_2d(), 200),
        "impact3d": (scenes.impact_3d(), 200),
        "slab3d": (scenes.snowball_on_slab_3d(W=32, ppc=4), 300),
        "blocks2d": (scenes.snow_blocks_2d(), 300),
        "impact3d_quad": (scenes.impact_3d().with_(**quad), 150),
        "impact2d_quad": (scenes.impact_2d().with_(**quad), 150),
        # two snowballs through their collision: most particles leave the
        # elastic band and take the queued-window scatter
        "collide3d": (scenes.two_snowballs_3d(W=64, ppc=2), 400),
    }


@pytest.mark.parametrize("case", ["impact2d", "impact3d", "slab3d", "blocks2d", "impact3d_quad", "impact2d_quad",
                                  "collide3d"])
def test_fused_matches_split(gpu_lib, case):
    """The two transfers differ only in how P2G groups particles before its
    int64 adds (FP32 partial sums over different runs), so they agree to a
    few FP32 roundings per step."""
    sc, steps = _scenes()[case]
    a, fa = _run(sc, steps, "fused")
    b, fb = _run(sc, steps, "split")
    assert fa & 1 == 0 and fb & 1 == 0
    errs = {f: rel_l2(getattr(a, f), getattr(b, f)) for f in ("position", "velocity", "elastic_f", "plastic_det")}
    print(case, ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert errs["position"] < 2e-6 and errs["elastic_f"] < 2e-5 and errs["plastic_det"] < 2e-5
    assert errs["velocity"] < 5e-4  # relative to near-zero velocities after contact


def test_queued_windows_bitwise(gpu_lib):
    """The queued particles' scatter groups them by the window the fused
    kernel recorded, in whatever order the windows were recorded: two runs
    through the collision (most particles queued) are bit-identical."""
    sc, steps = _scenes()["collide3d"]
    a, fa = _run(sc, steps, "fused")
    b, fb = _run(sc, steps, "fused")
    assert fa & 1 == 0 and fa == fb
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


def test_tma_pipeline_bitwise(gpu_lib):
    """The TMA pipeline hands tiles and windows to warps in whatever order they
    come free; the sums do not depend on it: two runs through the collision are
    bit-identical."""
    sc, steps = _scenes()["collide3d"]
    a, fa = _run(sc, steps, "fused", "tma")
    b, fb = _run(sc, steps, "fused", "tma")
    assert fa & (1 | 16) == 0 and fa == fb
    for f in FIELDS:
        assert np.array_equal(getattr(a, f), getattr(b, f)), f


@pytest.mark.parametrize("case", ["impact2d", "slab3d", "impact3d_quad", "impact2d_quad", "collide3d"])
def test_tma_box_load(gpu_lib, case):
    """The TMA box pipeline (k_g2p2g_pipe: node boxes by TMA tensor loads two
    stages deep, warps moving between tiles without CTA barriers, mbarrier
    waits bounded) against the staged boxes: the same windows and runs, so the
    runs agree to FP32 contraction differences between the two kernel builds,
    and no wait gives up."""
    sc, steps = _scenes()[case]
    a, fa = _run(sc, steps, "fused", "gather")
    b, fb = _run(sc, steps, "fused", "tma")
    assert fb & 16 == 0, "a TMA box load timed out"
    assert fa & 1 == 0 and fb & 1 == 0
    same = all(np.array_equal(getattr(a, f), getattr(b, f)) for f in FIELDS)
    errs = {f: rel_l2(getattr(b, f), getattr(a, f)) for f in ("position", "velocity", "elastic_f", "plastic_det")}
    print(case, "bitwise" if same else ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert errs["position"] < 1e-6 and errs["elastic_f"] < 1e-5 and errs["plastic_det"] < 1e-5


def test_fused_resume_is_bitwise(gpu_lib, tmp_path):
    """Checkpoints taken right after the first step, after a sort and while
    out-of-band particles take the queued-window scatter: the resumed run restores
    the tiles of the last sort and the pending grid sums and continues bit for
    bit."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.impact_3d(steps=200)
    for save_at in (1, 8, 45, 90, 130):
        with Solver.from_scene(sc) as a:
            a.Step(save_at)
            a.save(tmp_path / "ck.bin")
            a.Step(25)
            end = a.get_state()
        with Solver.from_scene(sc) as b:
            b.load(tmp_path / "ck.bin")
            b.Step(25)
            again = b.get_state()
        for f in FIELDS:
            assert np.array_equal(getattr(end, f), getattr(again, f)), (save_at, f)


def test_pending_sums_match_a_fresh_p2g(gpu_lib):
    """After a step the grid holds the next step's P2G; a solver given the same
    state computes it afresh with the prologue pass."""
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = scenes.impact_3d()
    with Solver.from_scene(sc) as a:
        a.Step(60)
        st = a.get_state()
        m1, p1 = a.rasterize()
        m1b, p1b = a.rasterize()  # reading the pending sums twice changes nothing
    with Solver.from_scene(sc) as b:
        b.set_state(position=st.position, velocity=st.velocity, affine_b=st.affine_b, elastic_f=st.elastic_f,
                     plastic_det=st.plastic_det)
        m2, p2 = b.rasterize()
    assert np.array_equal(m1, m1b) and np.array_equal(p1, p1b)
    assert rel_l2(m1, m2) < 1e-6
    assert rel_l2(p1, p2) < 1e-5
