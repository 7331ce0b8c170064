"""The FP64 quadratic-stencil restatement (formulation QUAD = 2) on its own:
the transfer identities that distinguish it from the cubic stencil. With
gravity off, F = I (zero stress) and walls out of reach, one step of APIC
transfers an affine velocity field v(x) = v0 + M x exactly and returns
B = M / D^-1, with D^-1 = 4 on the quadratic stencil and 3 on the cubic."""
import numpy as np
import pytest

from oracle import oracle as O

MLS, QUAD = 0, 2


def affine_scene(dim, seed=5):
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.impact_2d() if dim == 2 else scenes.impact_3d()
    rng = np.random.default_rng(seed)
    c = np.float32(sc.width / 2)
    pos = (c + rng.uniform(-4, 4, (300, dim))).astype(np.float32)
    M = rng.uniform(-2, 2, (dim, dim))
    v0 = rng.uniform(-3, 3, dim)
    vel = (v0 + pos.astype(np.float64) @ M.T).astype(np.float32)
    # heavy particles: no stencil node falls under the grid's 1e-6 mass cut
    # (grid_update.glsl:90), which would drop its velocity from the sums
    sc = sc.with_(position=pos, velocity=vel, volume=sc.volume[:300], mass=np.full(300, 1e6, np.float32),
                  gravity=0.0)
    return sc, M, v0


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("form,dinv", [(MLS, 3.0), (QUAD, 4.0)])
def test_affine_field_transfers_exactly(oracle_mod, dim, form, dinv):
    sc, M, v0 = affine_scene(dim)
    st = O.initial_state(sc.with_(formulation=form))
    st.velocity[:] = v0 + st.position @ M.T      # exact in FP64
    st.affine_b[:] = M / dinv
    x0 = st.position.copy()
    O.run_oracle(sc.with_(formulation=form), st, 1)
    assert np.allclose(st.velocity, v0 + x0 @ M.T, rtol=0, atol=1e-9)
    assert np.allclose(st.affine_b, np.broadcast_to(M / dinv, st.affine_b.shape), rtol=0, atol=1e-9)
    # and the other factor does not reproduce it
    other = O.initial_state(sc.with_(formulation=form))
    other.velocity[:] = v0 + other.position @ M.T
    other.affine_b[:] = M / (7.0 - dinv)
    O.run_oracle(sc.with_(formulation=form), other, 1)
    assert not np.allclose(other.velocity, v0 + x0 @ M.T, rtol=0, atol=1e-6)


@pytest.mark.parametrize("dim", [2, 3])
def test_quadratic_free_fall_and_rest(oracle_mod, dim):
    from mpm_snow_sim2d_b200 import scenes
    sc = (scenes.snow_blocks_2d(steps=50) if dim == 2 else scenes.impact_3d()).with_(formulation=QUAD)
    sc = sc.with_(velocity=np.zeros_like(sc.velocity), mass=np.full(sc.count, 1e6, np.float32))  # no mass cut
    st = O.initial_state(sc.with_(gravity=0.0))
    O.run_oracle(sc.with_(gravity=0.0), st, 20)
    assert np.array_equal(st.position, sc.position.astype(np.float64)) or np.abs(st.position - sc.position).max() < 1e-12
    assert np.abs(st.velocity).max() < 1e-12
    # free fall of blocks far from the walls: v = g t exactly
    if dim == 2:
        st = O.initial_state(sc)
        O.run_oracle(sc, st, 20)
        v_exp = sc.gravity * sc.delta_time * 20
        assert np.allclose(st.velocity[:, 1], v_exp, rtol=1e-12)
        assert np.abs(st.velocity[:, 0]).max() < 1e-12


def test_oracle_rejects_unknown_formulation(oracle_mod):
    from mpm_snow_sim2d_b200 import scenes
    sc = scenes.impact_2d()
    st = O.initial_state(sc)
    with pytest.raises(RuntimeError):
        O.run_oracle(sc, st, 1, formulation=3)
