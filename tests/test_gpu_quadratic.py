"""The quadratic-stencil variant (MPM_FORMULATION_MLS_QUADRATIC: 3 nodes per
axis from floor(x - 1/2), D^-1 = 4) against the FP64 quadratic restatement
in the oracle, plus the properties the cubic path is held to: determinism,
conservation, exact free fall, stale sort order."""
import numpy as np
import pytest

from conftest import state_errors
from test_gpu_parity import TARGET, TIGHT, _check, _check_vs_fp32_reference, _fp32_reference_errors, _gpu_run, _oracle_ref

pytestmark = pytest.mark.gpu
QUAD = 2


def _q(sc):
    return sc.with_(formulation=QUAD)


@pytest.mark.parametrize("case", ["impact2d", "impact3d"])
def test_quadratic_impact_against_oracle(gpu_lib, oracle_mod, case):
    from mpm_snow_sim2d_b200 import scenes
    sc = _q(scenes.impact_2d() if case == "impact2d" else scenes.impact_3d())
    dim = sc.dim
    steps = [1, 100, 300]
    ref = _oracle_ref(oracle_mod, sc, steps)
    assert ref[300]["plastic_det"].min() < 0.99  # plastic flow happened
    got, flags = _gpu_run(sc, steps)
    assert flags & 1 == 0
    r32 = _fp32_reference_errors(oracle_mod, sc, steps)
    _check_vs_fp32_reference(state_errors(got[1], ref[1], dim), r32[1], f"quad {case} step 1", TIGHT)
    for s in steps[1:]:
        _check_vs_fp32_reference(state_errors(got[s], ref[s], dim), r32[s], f"quad {case} step {s}")


def test_quadratic_2d_blocks_1000_steps(gpu_lib, oracle_mod):
    from mpm_snow_sim2d_b200 import scenes
    sc = _q(scenes.snow_blocks_2d())
    steps = [1, 1000]
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, flags = _gpu_run(sc, steps)
    assert flags & 1 == 0
    _check(state_errors(got[1], ref[1], 2), TIGHT, "quad blocks step 1")
    _check(state_errors(got[1000], ref[1000], 2), TARGET, "quad blocks step 1000")


def test_quadratic_3d_snowball_slab_1000_steps(gpu_lib, oracle_mod):
    from mpm_snow_sim2d_b200 import scenes
    sc = _q(scenes.snowball_on_slab_3d(W=32, ppc=1))
    steps = [1, 1000]
    ref = _oracle_ref(oracle_mod, sc, steps)
    got, _ = _gpu_run(sc, steps)
    r32 = _fp32_reference_errors(oracle_mod, sc, steps)
    _check_vs_fp32_reference(state_errors(got[1], ref[1], 3), r32[1], "quad slab step 1", TIGHT)
    _check_vs_fp32_reference(state_errors(got[1000], ref[1000], 3), r32[1000], "quad slab step 1000")


@pytest.mark.parametrize("case", ["impact3d", "dense2d"])
def test_quadratic_bitwise_determinism(gpu_lib, case):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = _q({"impact3d": lambda: scenes.impact_3d(), "dense2d": lambda: scenes.impact_2d(W=16, ppc=1000)}[case]())
    outs = []
    for _ in range(2):
        with Solver.from_scene(sc) as s:
            s.Step(40)
            _, _, raw = s.rasterize(raw=True)
            outs.append((raw, s.get_state()))
    (r0, s0), (r1, s1) = outs
    assert np.array_equal(r0, r1)
    for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_det"):
        assert np.array_equal(getattr(s0, f), getattr(s1, f)), f


@pytest.mark.parametrize("dim", [2, 3])
def test_quadratic_p2g_conservation(gpu_lib, dim):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = _q(scenes.impact_2d() if dim == 2 else scenes.impact_3d())
    with Solver.from_scene(sc) as s:
        s.Step(60)
        st = s.get_state()
        m, p = s.rasterize()
    total = float(sc.mass.astype(np.float64).sum())
    assert abs(m.sum() - total) <= 1e-6 * total
    mom = (sc.mass.astype(np.float64)[:, None] * st.velocity.astype(np.float64)).sum(0)
    scale = (sc.mass.astype(np.float64)[:, None] * np.abs(st.velocity)).sum()
    assert np.all(np.abs(p.sum(0) - mom) <= 1e-5 * scale)


def test_quadratic_free_fall_is_exact(gpu_lib):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = _q(scenes.snow_blocks_2d(steps=100))
    sc = sc.with_(velocity=np.tile(np.float32([0.0, -50.0]), (sc.count, 1)))
    with Solver.from_scene(sc) as s:
        s.Step(100)
        st = s.get_state()
    t = 100 * sc.delta_time
    v_exp = -50.0 + sc.gravity * t
    assert abs(np.median(st.velocity[:, 1]) - v_exp) < 1e-4 * abs(v_exp)
    dy = np.median(st.position[:, 1] - sc.position[:, 1])
    y_exp = sum((-50.0 + sc.gravity * sc.delta_time * (k + 1)) * sc.delta_time for k in range(100))
    assert abs(dy - y_exp) < 1e-3 * abs(y_exp)


def test_quadratic_rejects_learned_return_map(gpu_lib):
    """The surrogate was trained on the cubic step's return maps."""
    from mpm_snow_sim2d_b200 import MpmError, Solver, _lib, scenes
    from mpm_snow_sim2d_b200.mlp import DEFAULT_WEIGHTS, Mlp
    sc = _q(scenes.impact_3d())
    net = Mlp.load(DEFAULT_WEIGHTS)
    with Solver.from_scene(sc) as s:
        with pytest.raises(MpmError) as ei:
            s.set_plasticity(_lib.PLASTIC_MLP, net, 1e-3)
        assert ei.value.status == 10


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("form,dinv", [(0, 3.0), (QUAD, 4.0)])
def test_affine_field_transfers_exactly(gpu_lib, dim, form, dinv):
    """One APIC step carries v = v0 + M x exactly and returns B = M / D^-1
    (3 cubic, 4 quadratic): checks each stencil's weights and factor on the
    device independently of the oracle."""
    from mpm_snow_sim2d_b200 import Solver
    from test_oracle_quadratic import affine_scene
    sc, M, v0 = affine_scene(dim)
    sc = sc.with_(formulation=form)
    x0 = sc.position.astype(np.float64)
    with Solver.from_scene(sc) as s:
        s.set_state(affine_b=np.broadcast_to((M / dinv).astype(np.float32), (sc.count, dim, dim)).copy())
        s.Step(1)
        st = s.get_state()
    v_exp = v0 + x0 @ M.T
    err_v = np.abs(st.velocity - v_exp).max() / np.abs(v_exp).max()
    err_b = np.abs(st.affine_b - M / dinv).max() / np.abs(M / dinv).max()
    print(f"dim {dim} form {form}: v {err_v:.2e}, B {err_b:.2e}")
    assert err_v < 2e-6 and err_b < 1e-4  # B: sums of |v| ~ 100 terms cancelling to |B| ~ 0.5
