"""Status flags raised by conditions injected on the host (no GPU fault).

The reference meets a non-finite stress by printing and spinning forever
(src/cpu/Particles.cpp:50-61) and has no other runtime checks. Here kernels
raise bits of a device status word and never trap; mpm_check_status turns the
word into an error code. Each condition below is reached through the public
API with ordinary in-bounds inputs: a particle given a speed far above the
fixed-point design cap (16 cells per step), a material whose Young's modulus
makes the stress leave the fixed-point range, and particles whose stencil
reaches outside the grid."""
import numpy as np
import pytest

from mpm_snow_sim2d_b200 import _lib

pytestmark = pytest.mark.gpu

OVERFLOW = _lib.FLAG_FIXED_POINT_OVERFLOW
OUTSIDE = _lib.FLAG_PARTICLE_OUT_OF_DOMAIN


def _scene(dim):
    from mpm_snow_sim2d_b200 import scenes
    return scenes.impact_2d(steps=10) if dim == 2 else scenes.impact_3d(steps=10)


@pytest.mark.parametrize("dim", [2, 3])
def test_speed_above_cap_raises_overflow(gpu_lib, dim):
    from mpm_snow_sim2d_b200 import Solver
    sc = _scene(dim)
    with Solver.from_scene(sc) as s:
        s.Step(2)
        assert s.status() == 0 and s.check_status() == 0
        st = s.get_state()
        # 2000 cells per step: the nodes it reaches exceed the cap whatever the
        # neighbouring masses (at most ~30 particles share a node here)
        st.velocity[0, 0] = np.float32(2000.0 / sc.delta_time)
        s.set_state(velocity=st.velocity)
        s.Step(1)
        flags = s.status()
        assert flags & OVERFLOW, f"flags {flags:#x}"
        rc = s.check_status()
        assert rc in (4, 5), rc  # overflow, or NaN if the wrapped sums also went non-finite
        if not flags & 1:
            assert rc == 5
        assert "overflow" in s.last_error()


@pytest.mark.parametrize("dim", [2, 3])
def test_absurd_youngs_modulus_raises_overflow(gpu_lib, dim):
    from mpm_snow_sim2d_b200 import Solver
    sc = _scene(dim).with_(youngs=1e37)
    with Solver.from_scene(sc) as s:
        s.Step(5)
        flags = s.status()
        assert flags & OVERFLOW, f"flags {flags:#x}"
        assert s.check_status() in (4, 5)


@pytest.mark.parametrize("dim", [2, 3])
def test_stencil_outside_grid_raises_out_of_domain(gpu_lib, dim):
    from mpm_snow_sim2d_b200 import Solver
    sc = _scene(dim)
    pos = sc.position.copy()
    pos[:4] = np.float32(0.5)  # cell 0: the cubic stencil starts at node -1
    with Solver.from_scene(sc.with_(position=pos)) as s:
        s.Step(1)
        flags = s.status()
        assert flags & OUTSIDE, f"flags {flags:#x}"
        assert not flags & (1 | OVERFLOW)
        assert s.check_status() == 12
        assert "outside the grid" in s.last_error()
        # the particles stay finite and inside the clamped index range
        st = s.get_state()
        assert np.isfinite(st.position).all()
