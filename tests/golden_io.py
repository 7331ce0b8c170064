"""Load the golden fixtures written by tests/golden/make_golden.py."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from mpm_snow_sim2d_b200.scenes import Scene

GOLDEN = Path(__file__).resolve().parent / "golden"


def load_case(name: str):
    z = np.load(GOLDEN / f"{name}.npz")
    k = z["knobs"]
    pos = z["position0"]
    scene = Scene(
        name=name, dim=2, width=int(k[0]), height=int(k[1]), depth=0, border_margin=int(k[2]),
        delta_time=float(np.float32(k[3])), gravity=float(np.float32(k[4])), friction=float(np.float32(k[5])),
        theta_c=float(np.float32(k[6])), theta_s=float(np.float32(k[7])), xi=float(np.float32(k[8])),
        nu=float(np.float32(k[9])), youngs=float(np.float32(k[10])), rho=float(np.float32(k[11])),
        steps=int(z["steps"].max()), position=pos, velocity=z["velocity0"], volume=z["volume"], mass=z["mass"])
    dumps = {}
    for s in z["steps"].tolist():
        dumps[s] = {f: z[f"s{s}_{f}"] for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_f")}
    return scene, dumps
