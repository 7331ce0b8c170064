"""Python host mirror of the reference's solver interface.

``Solver`` keeps the names and behaviour of the reference's compile-time
``Solver`` alias (src/main.cpp:23-29):

    solver = Solver(params, particles)   # GPUSolver()   src/gpu/GPUSolver.cpp:7-51
    solver.Step()                        # Step()        src/gpu/GPUSolver.cpp:63-80
    pos = solver.GetParticlePositions()  # GetParticlePositions()  :276-295

and forwards every call to the C ABI of libmpm_b200.so (include/mpm/mpm.h).
Errors surface as ``MpmError`` carrying the ``mpm_status`` code (the reference
threw std::runtime_error / std::string, src/gpu/GPUSolver.cpp:39-49).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib
from ._lib import MpmParams, MpmParticlesInit, MpmStateHost, check, fptr


def params_from_scene(scene, *, formulation=None, boundary=None, sort_period=0) -> MpmParams:
    p = MpmParams()
    _lib.load().mpm_params_default(C.byref(p), scene.dim)
    p.dim = scene.dim
    p.width, p.height, p.depth = scene.width, scene.height, scene.depth if scene.dim == 3 else 0
    p.border_margin = scene.border_margin
    p.formulation = scene.formulation if formulation is None else formulation
    p.boundary = scene.boundary if boundary is None else boundary
    p.sort_period = sort_period
    p.delta_time = scene.delta_time
    p.gravity = scene.gravity
    p.friction = scene.friction
    p.theta_c, p.theta_s, p.xi = scene.theta_c, scene.theta_s, scene.xi
    p.nu, p.youngs, p.rho = scene.nu, scene.youngs, scene.rho
    return p


@dataclass
class State:
    position: np.ndarray
    velocity: np.ndarray
    affine_b: np.ndarray
    elastic_f: np.ndarray
    plastic_det: np.ndarray


def _f32(a, shape=None):
    if a is None:
        return None
    a = np.ascontiguousarray(a, dtype=np.float32)
    if shape is not None and a.shape != shape:
        a = a.reshape(shape)
    return a


class Solver:
    """One snow scene on the current CUDA device (B200, sm_100a)."""

    def __init__(self, params: MpmParams, position, volume, velocity=None, mass=None):
        lib = _lib.load()
        self._lib = lib
        self.dim = int(params.dim)
        pos = _f32(position)
        n = pos.shape[0] if pos.ndim == 2 else pos.size // self.dim
        self._keep = [pos.reshape(n, self.dim), _f32(volume).reshape(n),
                      None if velocity is None else _f32(velocity).reshape(n, self.dim),
                      None if mass is None else _f32(mass).reshape(n)]
        init = MpmParticlesInit(n, fptr(self._keep[0]), fptr(self._keep[2]), fptr(self._keep[1]),
                                fptr(self._keep[3]))
        self.params = params
        handle = C.c_void_p()
        check(lib.mpm_create(C.byref(params), C.byref(init), C.byref(handle)))
        self._h = handle
        self.count = n

    @classmethod
    def from_scene(cls, scene, **kw) -> "Solver":
        return cls(params_from_scene(scene, **kw), scene.position, scene.volume, scene.velocity, scene.mass)

    # -- reference interface -------------------------------------------------
    def Step(self, nsteps: int = 1) -> None:
        check(self._lib.mpm_step(self._h, int(nsteps)), self._h)

    def GetParticlePositions(self) -> np.ndarray:
        out = np.empty((self.count, self.dim), np.float32)
        check(self._lib.mpm_get_positions(self._h, fptr(out), out.size), self._h)
        return out

    # -- state, diagnostics, checkpoints --------------------------------------
    def get_state(self) -> State:
        n, d = self.count, self.dim
        st = State(np.empty((n, d), np.float32), np.empty((n, d), np.float32), np.empty((n, d, d), np.float32),
                   np.empty((n, d, d), np.float32), np.empty(n, np.float32))
        h = MpmStateHost(n, fptr(st.position), fptr(st.velocity), fptr(st.affine_b), fptr(st.elastic_f),
                         fptr(st.plastic_det))
        check(self._lib.mpm_get_state(self._h, C.byref(h)), self._h)
        return st

    def set_state(self, position=None, velocity=None, affine_b=None, elastic_f=None, plastic_det=None) -> None:
        n, d = self.count, self.dim
        arrs = [_f32(position, (n, d)), _f32(velocity, (n, d)), _f32(affine_b, (n, d, d)),
                _f32(elastic_f, (n, d, d)), _f32(plastic_det, (n,))]
        h = MpmStateHost(n, *[fptr(a) for a in arrs])
        check(self._lib.mpm_set_state(self._h, C.byref(h)), self._h)

    @property
    def nodes(self) -> int:
        p = self.params
        n = (p.width + 1) * (p.height + 1)
        return n * (p.depth + 1) if self.dim == 3 else n

    def rasterize(self, raw: bool = False):
        """P2G only (Grid::RasterizeToGrid): node mass (nodes,), momentum (nodes, dim)."""
        nodes = self.nodes
        m = np.empty(nodes, np.float64)
        p = np.empty((nodes, self.dim), np.float64)
        r = np.empty((1 + self.dim, nodes), np.int64) if raw else None
        check(self._lib.mpm_rasterize(self._h, m.ctypes.data_as(C.POINTER(C.c_double)),
                                      p.ctypes.data_as(C.POINTER(C.c_double)),
                                      r.ctypes.data_as(C.POINTER(C.c_int64)) if raw else None, nodes), self._h)
        return (m, p, r) if raw else (m, p)

    def status(self) -> int:
        f = C.c_uint32()
        check(self._lib.mpm_get_status(self._h, C.byref(f)), self._h)
        return int(f.value)

    def check_status(self) -> int:
        """The status word as an mpm_status code (0 when no error flag is set);
        last_error() names the flags."""
        return int(self._lib.mpm_check_status(self._h))

    def last_error(self) -> str:
        raw = self._lib.mpm_last_error(self._h)
        return raw.decode() if raw else ""

    def set_stream(self, cuda_stream_handle: int) -> None:
        check(self._lib.mpm_set_stream(self._h, C.c_void_p(cuda_stream_handle)), self._h)

    def save(self, path) -> None:
        check(self._lib.mpm_save_state(self._h, str(path).encode()), self._h)

    def load(self, path) -> None:
        check(self._lib.mpm_load_state(self._h, str(path).encode()), self._h)

    @property
    def step_count(self) -> int:
        s = C.c_int64()
        check(self._lib.mpm_get_step(self._h, C.byref(s)), self._h)
        return int(s.value)

    def sort_stats(self):
        """(sorts run so far, current sort period in steps)."""
        n, k = C.c_int64(), C.c_int32()
        check(self._lib.mpm_get_sort_stats(self._h, C.byref(n), C.byref(k)), self._h)
        return int(n.value), int(k.value)

    def fixed_point(self):
        a, b = C.c_int32(), C.c_int32()
        check(self._lib.mpm_get_fixed_point(self._h, C.byref(a), C.byref(b)), self._h)
        return int(a.value), int(b.value)

    def step_profiled(self, nsteps: int = 1) -> dict:
        """Run nsteps with CUDA events between stages; device ms per stage."""
        n = int(self._lib.mpm_stage_count(self._h))
        ms = (C.c_double * n)()
        check(self._lib.mpm_step_profiled(self._h, int(nsteps), ms, n), self._h)
        return {self._lib.mpm_stage_name(self._h, k).decode(): float(ms[k]) for k in range(n)}

    # -- headless frames (Visualize + saveFrame) -------------------------------
    def render(self, **kw) -> np.ndarray:
        """(height, width, 3) uint8 frame of the current state; keywords
        override mpm_render_params_default (width, height, point_size,
        camera_angle, camera_elevation, camera_distance, fov_degrees)."""
        p = _lib.MpmRenderParams()
        self._lib.mpm_render_params_default(C.byref(p))
        for k, v in kw.items():
            setattr(p, k, v)
        out = np.empty((p.height, p.width, 3), np.uint8)
        check(self._lib.mpm_render(self._h, C.byref(p), out.ctypes.data_as(C.POINTER(C.c_uint8)), out.nbytes),
              self._h)
        return out

    # -- learned plasticity ---------------------------------------------------
    def set_plasticity(self, mode: int, mlp=None, tolerance: float = 1e-3) -> None:
        """_lib.PLASTIC_EXACT, or _lib.PLASTIC_MLP with an Mlp (kept alive by the caller)."""
        self._mlp_ref = mlp
        check(self._lib.mpm_set_plasticity(self._h, int(mode), mlp._h if mlp is not None else None,
                                           float(tolerance)), self._h)

    def mlp_stats(self):
        a, r = C.c_uint64(), C.c_uint64()
        check(self._lib.mpm_get_mlp_stats(self._h, C.byref(a), C.byref(r)), self._h)
        return int(a.value), int(r.value)

    def pair_log_enable(self, capacity: int) -> None:
        check(self._lib.mpm_pair_log_enable(self._h, int(capacity)), self._h)

    def pair_log_read(self, cap: int) -> np.ndarray:
        out = np.empty((cap, 20), np.float32)
        n = C.c_int64()
        check(self._lib.mpm_pair_log_read(self._h, fptr(out), cap, C.byref(n)), self._h)
        return out[: n.value].copy()

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mpm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
