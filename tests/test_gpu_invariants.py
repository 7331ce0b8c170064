"""The step's invariants on the device (cubic and quadratic stencils): the
return map's volume bookkeeping and APIC's angular momentum, as checked on
the FP64 oracle in tests/test_oracle_invariants.py, here at FP32 tolerance."""
import numpy as np
import pytest

from test_oracle_invariants import STENCILS, angular_momentum_z, rotating_disc, spin_b

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("form,dinv", STENCILS)
@pytest.mark.parametrize("dim", [2, 3])
def test_volume_bookkeeping_on_device(gpu_lib, form, dinv, dim):
    from mpm_snow_sim2d_b200 import Solver, scenes
    sc = (scenes.impact_2d() if dim == 2 else scenes.impact_3d()).with_(formulation=form)
    with Solver.from_scene(sc) as s:
        s.Step(150)
        a = s.get_state()
        s.Step(1)
        b = s.get_state()
    assert b.plastic_det.min() < 0.95
    J0 = np.linalg.det(a.elastic_f.astype(np.float64)) * a.plastic_det
    J1 = np.linalg.det(b.elastic_f.astype(np.float64)) * b.plastic_det
    G = np.linalg.det(np.eye(dim) + sc.delta_time * dinv * b.affine_b.astype(np.float64))
    err = np.abs(J1 - G * J0).max() / np.abs(J0).max()
    print(f"dim {dim} form {form}: volume bookkeeping {err:.2e}")
    assert err < 2e-5


@pytest.mark.parametrize("form,dinv", STENCILS)
def test_rigid_rotation_keeps_angular_momentum_on_device(gpu_lib, form, dinv):
    from mpm_snow_sim2d_b200 import Solver
    sc, omega = rotating_disc()
    sc = sc.with_(formulation=form)
    m = sc.mass.astype(np.float64)
    B0 = np.broadcast_to(spin_b(2, omega, dinv), (sc.count, 2, 2)).astype(np.float32).copy()
    with Solver.from_scene(sc) as s:
        s.set_state(affine_b=B0)
        a = s.get_state()
        s.Step(100)
        b = s.get_state()
    f64 = lambda st: (st.position.astype(np.float64), st.velocity.astype(np.float64), st.affine_b.astype(np.float64))
    L0 = angular_momentum_z(*f64(a), m)
    L1 = angular_momentum_z(*f64(b), m)
    print(f"form {form}: L0 {L0:.6e} L1 {L1:.6e} rel {abs(L1 - L0) / abs(L0):.2e}")
    assert abs(L1 - L0) < 2e-5 * abs(L0)
