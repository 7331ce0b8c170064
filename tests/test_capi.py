"""CPU-side checks of the C ABI: the library loads, exports every function that
include/mpm/mpm.h declares, and host-only entry points behave (no kernel runs)."""
import ctypes as C
import re
from pathlib import Path

import pytest

from conftest import ROOT, has_gpu

HEADERS = sorted((ROOT / "include" / "mpm").glob("*.h"))


def declared_functions():
    names = []
    for h in HEADERS:
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][A-Za-z0-9_\s\*]*?\b(mpm_[a-z0-9_]+)\s*\(", text, flags=re.M)
    return sorted(set(names))


@pytest.fixture(scope="module")
def lib():
    from mpm_snow_sim2d_b200 import _lib
    from mpm_snow_sim2d_b200.build import build
    build()
    return _lib.load()


def test_header_declares_the_boundary():
    names = declared_functions()
    for required in ("mpm_create", "mpm_step", "mpm_get_positions", "mpm_destroy", "mpm_get_state"):
        assert required in names


def test_library_exports_every_declared_symbol(lib):
    from mpm_snow_sim2d_b200 import _lib
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing
    # and the Python binding covers all of them
    assert set(declared_functions()) <= set(_lib.SIGNATURES), set(declared_functions()) - set(_lib.SIGNATURES)


def test_params_default_mirrors_parameters_h(lib):
    from mpm_snow_sim2d_b200._lib import MpmParams
    p = MpmParams()
    lib.mpm_params_default(C.byref(p), 2)
    assert (p.width, p.height, p.border_margin) == (200, 100, 2)
    assert abs(p.delta_time - 1e-3) < 1e-9 and abs(p.gravity + 9.81) < 1e-6 and abs(p.friction - 0.3) < 1e-7
    assert abs(p.theta_c - 2e-2) < 1e-9 and abs(p.theta_s - 6e-3) < 1e-9 and p.xi == 10.0
    assert abs(p.nu - 0.2) < 1e-7 and p.youngs == 1.4e5 and p.rho == 400.0
    assert C.sizeof(MpmParams) == 96


def test_status_strings(lib):
    assert lib.mpm_status_string(0) == b"ok"
    assert b"sm_100" in lib.mpm_status_string(6)
    assert lib.mpm_status_string(999) == b"unknown status"


def test_create_rejects_bad_arguments(lib):
    from mpm_snow_sim2d_b200._lib import MpmParams, MpmParticlesInit
    p = MpmParams()
    lib.mpm_params_default(C.byref(p), 2)
    h = C.c_void_p()
    init = MpmParticlesInit(0, None, None, None, None)
    bad = MpmParams.from_buffer_copy(p)
    bad.dim = 4
    assert lib.mpm_create(C.byref(bad), C.byref(init), C.byref(h)) == 1
    bad = MpmParams.from_buffer_copy(p)
    bad.delta_time = 0.0
    assert lib.mpm_create(C.byref(bad), C.byref(init), C.byref(h)) == 1
    bad = MpmParams.from_buffer_copy(p)
    bad.dim, bad.formulation = 3, 1
    assert lib.mpm_create(C.byref(bad), C.byref(init), C.byref(h)) == 10
    bad = MpmParams.from_buffer_copy(p)
    bad.formulation = 3  # unknown (0 MLS, 1 CLASSIC, 2 quadratic)
    assert lib.mpm_create(C.byref(bad), C.byref(init), C.byref(h)) == 1
    bad = MpmParams.from_buffer_copy(p)
    bad.dim, bad.width, bad.height, bad.depth = 3, 2_000_001, 10, 10  # past the 3D per-axis cap
    assert lib.mpm_create(C.byref(bad), C.byref(init), C.byref(h)) == 1
    assert lib.mpm_create(C.byref(p), None, C.byref(h)) == 1


@pytest.mark.skipif(has_gpu(), reason="checks the no-device path")
def test_no_device_means_no_solver(lib):
    """The product path has no CPU fallback: without a GPU, create fails."""
    from mpm_snow_sim2d_b200._lib import MpmParams, MpmParticlesInit
    p = MpmParams()
    lib.mpm_params_default(C.byref(p), 2)
    h = C.c_void_p()
    init = MpmParticlesInit(0, None, None, None, None)
    assert lib.mpm_create(C.byref(p), C.byref(init), C.byref(h)) == 6
    assert not h.value
