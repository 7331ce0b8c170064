import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA B200 (sm_100a) device")
    config.addinivalue_line("markers", "slow: long-running check")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle as O
    from oracle.build_oracle import build_oracle
    build_oracle()
    return O


@pytest.fixture(scope="session")
def gpu_lib():
    """The CUDA library, built in-tree; GPU tests fail loudly without it."""
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200.build import build
    build()
    if not has_gpu():
        pytest.fail("GPU test selected but no CUDA device is visible")
    return _lib.load()


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (den if den > 0 else 1.0))


def state_errors(gpu_state, ref, dim):
    """Relative L2 errors of a solver state against an oracle / reference state.

    B is normalised by the velocity norm: it is a velocity times a cell offset
    whose terms cancel, so its own norm is dominated by rounding of O(|v|)
    terms."""
    vnorm = np.linalg.norm(np.asarray(ref["velocity"], np.float64))
    jp_ref = ref["plastic_det"] if "plastic_det" in ref else np.linalg.det(ref["plastic_f"])
    return dict(
        x=rel_l2(gpu_state.position, ref["position"]),
        v=rel_l2(gpu_state.velocity, ref["velocity"]),
        B=float(np.linalg.norm((np.asarray(gpu_state.affine_b, np.float64) - ref["affine_b"]).ravel()) / max(vnorm, 1e-30)),
        F=rel_l2(gpu_state.elastic_f, ref["elastic_f"]),
        Jp=rel_l2(gpu_state.plastic_det, jp_ref),
    )
