"""TEST INFRASTRUCTURE — Python access to the oracles.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the product path (mpm_snow_sim2d_b200) never imports it.

* ``run_oracle``: the project's CPU restatement (liboracle_mpm.so) of the
  reference step — FP64 (the oracle) or FP32 with OpenMP (the CPU baseline).
* ``run_refcpu``: the reference's own CPU path (oracle/_ref/refcpu_driver,
  compiled from src/cpu unmodified) on the same particles, in a subprocess with
  a timeout (the reference spins forever on a NaN stress,
  src/cpu/Particles.cpp:50-61).
"""
from __future__ import annotations

import ctypes as C
import json
import os
import struct
import subprocess
import tempfile
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .build_oracle import ORACLE_LIB, REFCPU, build_oracle

MLS, CLASSIC = 0, 1


class OrcParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32),
        ("border_margin", C.c_int32), ("formulation", C.c_int32), ("boundary", C.c_int32),
        ("reserved", C.c_int32),
        ("delta_time", C.c_double), ("gravity", C.c_double), ("friction", C.c_double),
        ("theta_c", C.c_double), ("theta_s", C.c_double), ("xi", C.c_double), ("nu", C.c_double),
        ("youngs", C.c_double),
    ]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not ORACLE_LIB.exists():
            build_oracle()
        L = C.CDLL(str(ORACLE_LIB))
        dp, fp = C.POINTER(C.c_double), C.POINTER(C.c_float)
        L.orc_step_f64.argtypes = [C.POINTER(OrcParams), C.c_int64] + [dp] * 7 + [C.c_int32]
        L.orc_step_f32.argtypes = [C.POINTER(OrcParams), C.c_int64] + [fp] * 7 + [C.c_int32, C.c_int32]
        L.orc_step_f64_mt.argtypes = [C.POINTER(OrcParams), C.c_int64] + [dp] * 7 + [C.c_int32, C.c_int32]
        L.orc_bspline_f64.argtypes = [C.c_double, dp, dp]
        L.orc_svd_f64.argtypes = [C.c_int32, C.c_int32, dp, dp, dp, dp]
        L.orc_svd_f64.restype = None
        L.orc_stress_f64.argtypes = [C.POINTER(OrcParams), dp, dp, dp]
        L.orc_stress_f64.restype = None
        L.orc_collide_f64.argtypes = [C.POINTER(OrcParams), dp, dp, dp, dp]
        L.orc_collide_f64.restype = None
        fp = C.POINTER(C.c_float)
        L.orc_bspline_f32.argtypes = [C.c_float, fp, fp]
        L.orc_bspline_f32.restype = None
        L.orc_svd_f32.argtypes = [C.c_int32, C.c_int32, fp, fp, fp, fp]
        L.orc_svd_f32.restype = None
        L.orc_collide_f32.argtypes = [C.POINTER(OrcParams), fp, fp, fp, fp]
        L.orc_collide_f32.restype = None
        L.orc_p2g_f64.argtypes = [C.POINTER(OrcParams), C.c_int64] + [dp] * 9
        L.orc_max_threads.restype = C.c_int
        _lib = L
    return _lib


def params_of(scene, formulation=None, boundary=None) -> OrcParams:
    p = OrcParams()
    p.dim, p.width, p.height = scene.dim, scene.width, scene.height
    p.depth = scene.depth if scene.dim == 3 else 0
    p.border_margin = scene.border_margin
    p.formulation = scene.formulation if formulation is None else formulation
    p.boundary = scene.boundary if boundary is None else boundary
    p.delta_time, p.gravity, p.friction = scene.delta_time, scene.gravity, scene.friction
    p.theta_c, p.theta_s, p.xi = scene.theta_c, scene.theta_s, scene.xi
    p.nu, p.youngs = scene.nu, scene.youngs
    return p


@dataclass
class OracleState:
    position: np.ndarray   # (n, d)
    velocity: np.ndarray   # (n, d)
    affine_b: np.ndarray   # (n, d, d)
    elastic_f: np.ndarray  # (n, d, d)
    plastic_f: np.ndarray  # (n, d, d) full F_P as the reference stores it
    mass: np.ndarray
    volume: np.ndarray

    @property
    def plastic_det(self) -> np.ndarray:
        return np.linalg.det(self.plastic_f)

    def copy(self) -> "OracleState":
        return OracleState(*(a.copy() for a in (self.position, self.velocity, self.affine_b, self.elastic_f,
                                                 self.plastic_f, self.mass, self.volume)))


def initial_state(scene, dtype=np.float64) -> OracleState:
    n, d = scene.count, scene.dim
    eye = np.ascontiguousarray(np.broadcast_to(np.eye(d, dtype=dtype), (n, d, d)))
    return OracleState(
        np.array(scene.position, dtype, order="C"), np.array(scene.velocity, dtype, order="C"),
        np.zeros((n, d, d), dtype), eye.copy(), eye.copy(), np.array(scene.mass, dtype, order="C"),
        np.array(scene.volume, dtype, order="C"))


def run_oracle(scene, state: OracleState, nsteps: int, *, formulation=None, boundary=None,
               fp32: bool = False, threads: int = 1) -> OracleState:
    """Advance `state` in place by nsteps with the CPU restatement."""
    L = lib()
    p = params_of(scene, formulation, boundary)
    n = state.position.shape[0]
    if fp32:
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_float))
        arrs = [state.position, state.velocity, state.affine_b, state.elastic_f, state.plastic_f, state.mass, state.volume]
        assert all(a.dtype == np.float32 and a.flags.c_contiguous for a in arrs)
        rc = L.orc_step_f32(C.byref(p), n, *map(ptr, arrs), nsteps, threads)
    else:
        ptr = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        arrs = [state.position, state.velocity, state.affine_b, state.elastic_f, state.plastic_f, state.mass, state.volume]
        assert all(a.dtype == np.float64 and a.flags.c_contiguous for a in arrs)
        rc = (L.orc_step_f64(C.byref(p), n, *map(ptr, arrs), nsteps) if threads <= 1
              else L.orc_step_f64_mt(C.byref(p), n, *map(ptr, arrs), nsteps, threads))
    if rc != 0:
        raise RuntimeError(f"oracle step failed with code {rc}")
    return state


# ---------------------------------------------------------------------------
# The reference's own CPU path.

def refcpu_available() -> bool:
    return REFCPU.exists() and os.access(REFCPU, os.X_OK)


def write_refcpu_input(path, scene, nsteps: int, dump_every: int = 0) -> None:
    assert scene.dim == 2, "the reference CPU path is 2D only"
    with open(path, "wb") as f:
        f.write(b"RCPU")
        f.write(struct.pack("<i", 1))
        f.write(struct.pack("<5i", scene.width, scene.height, scene.border_margin, nsteps, dump_every))
        f.write(struct.pack("<9f", scene.delta_time, scene.gravity, scene.friction, scene.theta_c, scene.theta_s,
                            scene.xi, scene.nu, scene.youngs, scene.rho))
        f.write(struct.pack("<q", scene.count))
        f.write(np.ascontiguousarray(scene.position, np.float32).tobytes())
        f.write(np.ascontiguousarray(scene.velocity, np.float32).tobytes())
        f.write(np.ascontiguousarray(scene.volume, np.float32).tobytes())


def read_refcpu_output(path, n: int):
    """List of (step, dict(position, velocity, affine_b, elastic_f, plastic_f))."""
    raw = Path(path).read_bytes()
    out, off = [], 0
    rec = 4 + 4 * n * (2 + 2 + 4 + 4 + 4)
    while off + rec <= len(raw):
        step = struct.unpack_from("<i", raw, off)[0]
        a = np.frombuffer(raw, np.float32, n * 16, off + 4)
        o = 0
        def take(k, shape):
            nonlocal o
            v = a[o:o + k].reshape(shape).copy()
            o += k
            return v
        out.append((step, dict(position=take(2 * n, (n, 2)), velocity=take(2 * n, (n, 2)),
                               affine_b=take(4 * n, (n, 2, 2)), elastic_f=take(4 * n, (n, 2, 2)),
                               plastic_f=take(4 * n, (n, 2, 2)))))
        off += rec
    return out


def run_refcpu(scene, nsteps: int, dump_every: int = 0, replicas: int = 1, timeout: int = 600):
    """Run the reference CPU path; returns (dumps, info json)."""
    if not refcpu_available():
        raise FileNotFoundError(f"{REFCPU} is not built")
    with tempfile.TemporaryDirectory() as td:
        fin, fout = Path(td) / "in.bin", Path(td) / "out.bin"
        write_refcpu_input(fin, scene, nsteps, dump_every)
        res = subprocess.run([str(REFCPU), str(fin), str(fout), "--replicas", str(replicas), "--timeout", str(timeout)],
                             capture_output=True, text=True, timeout=timeout + 30)
        if res.returncode != 0:
            raise RuntimeError(f"refcpu_driver exited {res.returncode}: {res.stderr.strip()}")
        info = json.loads(res.stdout.strip().splitlines()[-1])
        return read_refcpu_output(fout, scene.count), info
