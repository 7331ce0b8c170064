"""Batched scenes, host side (no GPU): the seeded batched workload and the
C ABI's argument checks and no-device path."""
import ctypes as C

import numpy as np
import pytest

from conftest import has_gpu


def test_batched_workload_follows_its_ranges():
    from mpm_snow_sim2d_b200 import scenes
    scs = scenes.batch_scenes_2d()
    assert len(scs) == 256
    W = np.array([s.width for s in scs])
    n = np.array([s.count for s in scs])
    assert W.min() >= 64 and W.max() <= 256 and len(set(W.tolist())) > 50
    assert n.min() >= 1900 and n.max() <= 64500
    assert 2.5e6 < n.sum() < 6e6
    for s in scs:
        assert s.dim == 2 and s.height == s.width
        assert 1e5 <= s.youngs <= 2e5 and 0.15 <= s.nu <= 0.3
        assert 4 <= s.info["ppc"] <= 8 and 1 <= s.info["blocks"] <= 4
        assert np.isclose(s.delta_time, 1e-4 * 128 / s.width)
        m = s.border_margin
        assert s.position.min() >= m and s.position.max() <= s.width - m
    again = scenes.batch_scene_2d(17)
    assert np.array_equal(again.position, scs[17].position)


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_batch_create_without_device():
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200._lib import MpmParams, MpmParticlesInit
    lib = _lib.load()
    p = (MpmParams * 1)()
    lib.mpm_params_default(C.byref(p[0]), 2)
    init = (MpmParticlesInit * 1)(MpmParticlesInit(0, None, None, None, None))
    h = C.c_void_p()
    assert lib.mpm_batch_create(p, init, 1, C.byref(h)) == 6
    assert not h.value


def test_batch_create_rejects_bad_arguments():
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200._lib import MpmParams, MpmParticlesInit
    lib = _lib.load()
    p = (MpmParams * 1)()
    lib.mpm_params_default(C.byref(p[0]), 3)
    init = (MpmParticlesInit * 1)(MpmParticlesInit(0, None, None, None, None))
    h = C.c_void_p()
    assert lib.mpm_batch_create(p, init, 0, C.byref(h)) == 1       # no scenes
    assert lib.mpm_batch_create(p, init, 1, C.byref(h)) == 10      # 3D: unsupported
    lib.mpm_params_default(C.byref(p[0]), 2)
    p[0].formulation = 1
    assert lib.mpm_batch_create(p, init, 1, C.byref(h)) == 10      # CLASSIC: unsupported
    assert not h.value
