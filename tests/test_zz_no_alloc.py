"""mpm_mlp_predict_noalloc through the C ABI: same outputs as mpm_mlp_predict
on two calls in a row, and the capacity limit. Collected last so that it also
runs after every other GPU test in the same process."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _rows(n, seed):
    rng = np.random.default_rng(seed)
    F = np.eye(3)[None] + 0.02 * rng.standard_normal((n, 3, 3))
    rows = np.zeros((n, 20), np.float32)
    rows[:, :9] = F.reshape(n, 9)
    rows[:, 9] = rng.uniform(0.5, 1.0, n)
    return rows


def test_noalloc_predict_matches_predict(gpu_lib):
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200._lib import fptr
    from mpm_snow_sim2d_b200.mlp import DEFAULT_WEIGHTS, Mlp
    lib = _lib.load()
    net = Mlp.load(DEFAULT_WEIGHTS)
    for call, n in enumerate((5000, 777)):
        rows = _rows(n, seed=call)
        ref = net.predict(rows)
        out = np.full((n, 10), np.nan, np.float32)
        st = lib.mpm_mlp_predict_noalloc(net._h, fptr(rows), n, 20, fptr(out))
        assert st == 0, lib.mpm_mlp_last_error(net._h)
        # same kernel and inputs: equal up to 1e-6 of the output scale
        np.testing.assert_allclose(out, ref, rtol=0, atol=1e-6 * float(np.abs(ref).max()))
    n = 65537
    rows = np.zeros((n, 10), np.float32)
    rows[:, 9] = 1.0
    out = np.empty((n, 10), np.float32)
    st = lib.mpm_mlp_predict_noalloc(net._h, fptr(rows), n, 10, fptr(out))
    assert st == 11  # MPM_ERR_CAPACITY
    assert b"65536" in lib.mpm_mlp_last_error(net._h)
    net.close()
