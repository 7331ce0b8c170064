"""The MLS restatement in oracle/mpm_oracle.cpp pinned to the reference's own
GPU code: the GLSL compute shaders of src/gpu/shaders/{2d,3d}, turned into C++
by a text shim (oracle/shader/glsl_cpp.py) and run on the CPU against the
reference's vendored glm (oracle/shader/shader_runner.cpp). The oracle's FP32
instantiation reproduces them bit for bit — function by function (svd,
B-spline weights, wall response) and over whole runs of steps — so its FP64
instantiation is the reference's algorithm evaluated in double."""
import ctypes as C

import numpy as np
import pytest

from mpm_snow_sim2d_b200 import scenes


@pytest.fixture(scope="module")
def sr():
    from oracle import shader_ref
    if not shader_ref.available():
        pytest.skip("the reference's shaders are not built (no reference tree and no earlier build)")
    return shader_ref


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _matrices(rng, dim, n):
    """Near identity (the elastic regime), strongly stretched, and nearly
    singular matrices, both orientations."""
    out = []
    for k in range(n):
        kind = k % 3
        if kind == 0:
            M = np.eye(dim) + 0.05 * rng.standard_normal((dim, dim))
        elif kind == 1:
            M = rng.standard_normal((dim, dim)) * rng.uniform(0.2, 3.0)
        else:
            U, _, Vt = np.linalg.svd(rng.standard_normal((dim, dim)))
            s = np.sort(rng.uniform(0.5, 1.5, dim))[::-1]
            s[-1] = 10.0 ** rng.uniform(-4, -1)
            M = U @ np.diag(s) @ Vt
        out.append(M.astype(np.float32))
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_svd_bitwise(sr, oracle_mod, dim):
    L = oracle_mod.lib()
    rng = np.random.default_rng(dim)
    for M in _matrices(rng, dim, 3000):
        U1, S1, V1 = sr.svd(dim, M)
        U2, V2 = np.empty((dim, dim), np.float32), np.empty((dim, dim), np.float32)
        S2 = np.empty(dim, np.float32)
        L.orc_svd_f32(dim, oracle_mod.MLS, _fp(M), _fp(U2), _fp(S2), _fp(V2))
        assert np.array_equal(S1, S2) and np.array_equal(U1, U2) and np.array_equal(V1, V2), M
        # the FP64 instantiation is the same algorithm in double: same factors
        # to FP32 rounding where the matrix is well conditioned (M^T M squares
        # the condition number, so FP32 loses digits of small singular values)
        Md = M.astype(np.float64)
        Ud, Vd, Sd = np.empty((dim, dim)), np.empty((dim, dim)), np.empty(dim)
        L.orc_svd_f64(dim, oracle_mod.MLS, _dp(Md), _dp(Ud), _dp(Sd), _dp(Vd))
        if np.abs(Sd).min() > 0.3 * np.abs(Sd).max():
            np.testing.assert_allclose(S1, Sd, rtol=2e-5, atol=1e-6)
            np.testing.assert_allclose(U1 * S1 @ V1.T, Md, atol=3e-5 * max(1.0, np.abs(Md).max()))


def test_bspline_bitwise(sr, oracle_mod):
    L = oracle_mod.lib()
    rng = np.random.default_rng(5)
    xs = np.concatenate([rng.uniform(-2.5, 2.5, 20000), [-2, -1, 0, 1, 2, -1.9999999, 0.9999999, 1.0000001]])
    for x in xs.astype(np.float32):
        for dim in (2, 3):
            n1, d1 = sr.bspline(dim, x)
            n2, d2 = C.c_float(), C.c_float()
            L.orc_bspline_f32(float(x), C.byref(n2), C.byref(d2))
            assert (n1, d1) == (n2.value, d2.value), x
            n3, d3 = C.c_double(), C.c_double()
            L.orc_bspline_f64(float(x), C.byref(n3), C.byref(d3))
            assert abs(n1 - n3.value) <= 2e-7 and abs(d1 - d3.value) <= 5e-7


@pytest.mark.parametrize("dim", [2, 3])
def test_wall_response_bitwise(sr, oracle_mod, dim):
    """Every wall plane, edge and corner of the grid, speeds from creeping to
    far beyond a cell per step."""
    L = oracle_mod.lib()
    sc = scenes.impact_2d() if dim == 2 else scenes.impact_3d()
    p = oracle_mod.params_of(sc)
    ext = [sc.width, sc.height, sc.depth][:dim]
    rng = np.random.default_rng(11 + dim)
    for _ in range(6000):
        loc = np.array([rng.choice([0, 1, 2, 3, 4, 5, e - 5, e - 4, e - 3, e - 2, e - 1, e, int(rng.integers(0, e + 1))])
                        for e in ext], np.float32)
        vel = (rng.standard_normal(dim) * rng.choice([1e-4, 1.0, 30.0, 3e3])).astype(np.float32)
        vc1, vf1 = sr.collide(sc, loc, vel)
        vc2, vf2 = np.empty(dim, np.float32), np.empty(dim, np.float32)
        L.orc_collide_f32(C.byref(p), _fp(loc), _fp(vel), _fp(vc2), _fp(vf2))
        assert np.array_equal(vc1, vc2) and np.array_equal(vf1, vf2), (loc, vel)


@pytest.mark.parametrize("case", ["impact2d", "blocks2d", "impact3d"])
def test_step_bitwise(sr, oracle_mod, case):
    """Whole steps: the reference's p2g, grid_update, g2p and reset shaders in
    dispatch order against the oracle's FP32 instantiation (single-threaded,
    particles in the same order), through impact, wall contact and plastic
    flow."""
    O = oracle_mod
    sc, steps = {"impact2d": (scenes.impact_2d(), 300), "blocks2d": (scenes.snow_blocks_2d(), 150),
                 "impact3d": (scenes.impact_3d(), 25)}[case]
    a, b = O.initial_state(sc, np.float32), O.initial_state(sc, np.float32)
    sr.run_shader(sc, a, steps)
    O.run_oracle(sc, b, steps, fp32=True)
    for f in ("position", "velocity", "affine_b", "elastic_f", "plastic_f"):
        assert np.array_equal(getattr(a, f), getattr(b, f)), f
    assert np.isfinite(a.position).all()
