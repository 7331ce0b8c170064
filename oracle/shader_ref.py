"""TEST INFRASTRUCTURE — the reference's GLSL shaders executed on the CPU.

Only tests/ use this module. oracle/_ref/libshader_ref.so is built by
oracle/build_oracle.py from the reference's own src/gpu/shaders/{2d,3d}/*.glsl
(turned into C++ by oracle/shader/glsl_cpp.py, run by
oracle/shader/shader_runner.cpp); it pins the MLS restatement of
oracle/mpm_oracle.cpp to the reference's shader code. Like oracle/_ref's other
builds it travels with the repository to machines without the reference tree.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from .build_oracle import SHADER_LIB, build_shader_ref


class SrParams(C.Structure):
    _fields_ = [("dim", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32),
                ("border_margin", C.c_float), ("delta_time", C.c_float), ("gravity", C.c_float),
                ("friction", C.c_float), ("theta_c", C.c_float), ("theta_s", C.c_float), ("xi", C.c_float),
                ("mu", C.c_float), ("lambda_", C.c_float)]


_lib = None


def available() -> bool:
    return build_shader_ref() is not None


def lib():
    global _lib
    if _lib is None:
        path = build_shader_ref()
        if path is None:
            raise FileNotFoundError("oracle/_ref/libshader_ref.so is not built (needs the reference tree once)")
        L = C.CDLL(str(path))
        fp = C.POINTER(C.c_float)
        L.sr_run.argtypes = [C.POINTER(SrParams), C.c_int64] + [fp] * 7 + [C.c_int32]
        L.sr_svd.argtypes = [C.c_int32, fp, fp, fp, fp]
        L.sr_svd.restype = None
        L.sr_bspline.argtypes = [C.c_int32, C.c_float, fp, fp]
        L.sr_bspline.restype = None
        L.sr_collide.argtypes = [C.POINTER(SrParams), fp, fp, fp, fp]
        L.sr_collide.restype = None
        _lib = L
    return _lib


def params_of(scene) -> SrParams:
    """Uniforms as GPUSolver sets them; MU and LAMBDA from E and nu as
    src/shared/Parameters.h:82-84 (evaluated in double, stored as float)."""
    p = SrParams()
    p.dim, p.width, p.height = scene.dim, scene.width, scene.height
    p.depth = scene.depth if scene.dim == 3 else 0
    p.border_margin = float(scene.border_margin)
    p.delta_time, p.gravity, p.friction = scene.delta_time, scene.gravity, scene.friction
    p.theta_c, p.theta_s, p.xi = scene.theta_c, scene.theta_s, scene.xi
    E, nu = float(scene.youngs), float(scene.nu)
    p.mu = E / (2.0 * (1.0 + nu))
    p.lambda_ = (E * nu) / ((1.0 + nu) * (1.0 - 2.0 * nu))
    return p


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def run_shader(scene, state, nsteps: int):
    """Advance an FP32 oracle.OracleState in place by nsteps of the shaders."""
    arrs = [state.position, state.velocity, state.affine_b, state.elastic_f, state.plastic_f, state.mass, state.volume]
    assert all(a.dtype == np.float32 and a.flags.c_contiguous for a in arrs)
    p = params_of(scene)
    rc = lib().sr_run(C.byref(p), state.position.shape[0], *map(_fp, arrs), int(nsteps))
    if rc != 0:
        raise RuntimeError(f"sr_run failed ({rc})")
    return state


def svd(dim: int, M: np.ndarray):
    M = np.ascontiguousarray(M, np.float32)
    U = np.empty((dim, dim), np.float32)
    V = np.empty((dim, dim), np.float32)
    S = np.empty(dim, np.float32)
    lib().sr_svd(dim, _fp(M), _fp(U), _fp(S), _fp(V))
    return U, S, V


def bspline(dim: int, x: float):
    n, dn = C.c_float(), C.c_float()
    lib().sr_bspline(dim, float(x), C.byref(n), C.byref(dn))
    return n.value, dn.value


def collide(scene, loc, vel):
    p = params_of(scene)
    d = scene.dim
    loc = np.ascontiguousarray(loc, np.float32)
    vel = np.ascontiguousarray(vel, np.float32)
    vc = np.empty(d, np.float32)
    vf = np.empty(d, np.float32)
    lib().sr_collide(C.byref(p), _fp(loc), _fp(vel), _fp(vc), _fp(vf))
    return vc, vf
