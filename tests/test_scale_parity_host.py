"""Host logic of tests/scale_parity.py (the full-size parity report): the
contact band, the per-field errors over the fields both states hold, and the
report's contact / free split."""
import numpy as np

import scale_parity as S
from mpm_snow_sim2d_b200 import scenes


def _state(rng, n, dim):
    return {"position": rng.uniform(0, 1, (n, dim)).astype(np.float64),
            "velocity": rng.standard_normal((n, dim)),
            "affine_b": rng.standard_normal((n, dim * dim)),
            "elastic_f": np.tile(np.eye(dim).ravel(), (n, 1)) + 0.01 * rng.standard_normal((n, dim * dim)),
            "plastic_det": 1.0 + 0.01 * rng.standard_normal(n)}


def test_contact_band_is_the_cubic_stencil_reach():
    """A cubic stencil spans floor(x) - 1 .. floor(x) + 2: a node within two
    cells of the wall plane at m means x < m + 4, and at extent - m means
    x >= extent - m - 4."""
    sc = scenes.impact_2d()
    m, W, H = float(sc.border_margin), float(sc.width), float(sc.height)
    mid = H / 2
    pts = np.array([[m + 3.99, mid], [m + 4.0, mid], [W - m - 4.0, mid], [W - m - 4.01, mid],
                    [W / 2, m + 3.5], [W / 2, H - m - 3.0], [W / 2, mid]])
    assert S.contact_band(sc, pts).tolist() == [True, False, True, False, True, True, False]


def test_errors_cover_the_fields_both_states_hold():
    rng = np.random.default_rng(3)
    ref = _state(rng, 500, 3)
    got = {k: v + 1e-6 * np.abs(v).max() * rng.standard_normal(v.shape) for k, v in ref.items()}
    full = S.errors(got, ref)
    assert set(full) == {"x", "v", "F", "Jp", "B"} and all(0 < e < 1e-4 for e in full.values())
    part = S.errors({k: got[k] for k in ("position", "elastic_f")}, ref)
    assert set(part) == {"x", "F"} and part["x"] == full["x"] and part["F"] == full["F"]
    # B needs the velocity of the state compared against
    assert "B" not in S.errors(got, {k: v for k, v in ref.items() if k != "velocity"})
    assert S.errors(ref, ref)["x"] == 0.0


def test_report_splits_contact_and_free():
    sc = scenes.impact_2d()
    rng = np.random.default_rng(4)
    n = 400
    ref = _state(rng, n, 2)
    ref["position"] = rng.uniform(0, sc.width, (n, 2))
    r32 = {k: v.astype(np.float32) for k, v in ref.items()}
    gpu = {k: v.copy() for k, v in ref.items()}
    band = S.contact_band(sc, ref["position"])
    gpu["position"][band] += 1e-3  # only the contact band differs
    res = S.report(sc, 10, gpu, 0, ref, r32)
    assert res["contact_particles"] == int(band.sum()) and res["free_particles"] == n - int(band.sum())
    assert res["gpu_vs_fp64"]["free"]["x"] == 0.0 and res["gpu_vs_fp64"]["contact"]["x"] > 0.0
    assert res["reference_fp32_vs_fp64"]["all"]["x"] < 1e-6
