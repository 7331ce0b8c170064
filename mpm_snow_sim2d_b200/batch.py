"""Batched 2D scenes: Python host mirror of mpm_batch_* (include/mpm/mpm.h).

    batch = Batch(scenes.batch_scenes_2d())   # 256 independent scenes
    batch.tune(4)                            # project autotuner (threads, CTAs per scene)
    batch.step(500)                          # one CUDA graph: a persistent launch per cluster size
    pos = batch.positions(17)                # scene 17, (n, 2) float32

Each scene is what mpm_create would make of it (same constants, fixed-point
scales and per-particle arithmetic); the batch only changes where the grid
lives (the shared memory of a CTA cluster) and how scenes share the GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import MpmBatchConfig, MpmError, MpmParticlesInit, MpmStateHost, fptr
from .solver import State, _f32, params_from_scene


class Batch:
    def __init__(self, scenes):
        lib = _lib.load()
        self._lib = lib
        self.scenes = list(scenes)
        k = len(self.scenes)
        params = (_lib.MpmParams * k)()
        inits = (MpmParticlesInit * k)()
        self._keep = []
        for s, sc in enumerate(self.scenes):
            if sc.dim != 2:
                raise ValueError("batched scenes are 2D")
            params[s] = params_from_scene(sc)
            pos, vel = _f32(sc.position).reshape(-1, 2), _f32(sc.velocity).reshape(-1, 2)
            vol, mass = _f32(sc.volume).reshape(-1), _f32(sc.mass).reshape(-1)
            self._keep += [pos, vel, vol, mass]
            inits[s] = MpmParticlesInit(pos.shape[0], fptr(pos), fptr(vel), fptr(vol), fptr(mass))
        h = C.c_void_p()
        st = lib.mpm_batch_create(params, inits, k, C.byref(h))
        if st != 0:
            raise MpmError(st, lib.mpm_status_string(st).decode())
        self._h = h
        self.counts = [sc.count for sc in self.scenes]

    def _check(self, st):
        if st != 0:
            detail = self._lib.mpm_batch_last_error(self._h)
            raise MpmError(st, (detail or b"").decode() or self._lib.mpm_status_string(st).decode())

    @property
    def total_particles(self) -> int:
        n, t = C.c_int32(), C.c_int64()
        self._check(self._lib.mpm_batch_info(self._h, C.byref(n), C.byref(t)))
        return int(t.value)

    def step(self, nsteps: int = 1) -> None:
        self._check(self._lib.mpm_batch_step(self._h, int(nsteps)))

    def set_stream(self, cuda_stream) -> None:
        self._check(self._lib.mpm_batch_set_stream(self._h, C.c_void_p(cuda_stream)))

    def positions(self, scene: int) -> np.ndarray:
        out = np.empty((self.counts[scene], 2), np.float32)
        self._check(self._lib.mpm_batch_get_positions(self._h, int(scene), fptr(out), out.size))
        return out

    def get_state(self, scene: int) -> State:
        n = self.counts[scene]
        st = State(np.empty((n, 2), np.float32), np.empty((n, 2), np.float32), np.empty((n, 2, 2), np.float32),
                   np.empty((n, 2, 2), np.float32), np.empty(n, np.float32))
        h = MpmStateHost(n, fptr(st.position), fptr(st.velocity), fptr(st.affine_b), fptr(st.elastic_f),
                         fptr(st.plastic_det))
        self._check(self._lib.mpm_batch_get_state(self._h, int(scene), C.byref(h)))
        return st

    def set_state(self, scene: int, position=None, velocity=None, affine_b=None, elastic_f=None,
                  plastic_det=None) -> None:
        n = self.counts[scene]
        arrs = [_f32(position, (n, 2)), _f32(velocity, (n, 2)), _f32(affine_b, (n, 2, 2)),
                _f32(elastic_f, (n, 2, 2)), _f32(plastic_det, (n,))]
        h = MpmStateHost(n, *[fptr(a) for a in arrs])
        self._check(self._lib.mpm_batch_set_state(self._h, int(scene), C.byref(h)))

    def status(self, scene: int) -> int:
        f = C.c_uint32()
        self._check(self._lib.mpm_batch_get_status(self._h, int(scene), C.byref(f)))
        return int(f.value)

    def step_times(self) -> np.ndarray:
        """Device timestamps (ns) of the last step call: (scenes, nsteps + 1),
        each scene's start then the end of each of its steps."""
        ns = C.c_int32()
        # a call without a buffer reports the step count
        self._lib.mpm_batch_step_times(self._h, None, 0, C.byref(ns))
        steps = int(ns.value)
        out = np.zeros((len(self.scenes), steps + 1), np.uint64)
        if steps:
            self._check(self._lib.mpm_batch_step_times(
                self._h, out.ctypes.data_as(C.POINTER(C.c_uint64)), out.size, C.byref(ns)))
        return out

    @property
    def config(self) -> dict:
        c = MpmBatchConfig()
        self._check(self._lib.mpm_batch_get_config(self._h, C.byref(c)))
        return dict(threads=c.threads, particles_per_cta=c.particles_per_cta, max_cluster=c.max_cluster,
                    sort_period=c.sort_period)

    def set_config(self, threads=None, particles_per_cta=None, max_cluster=None, sort_period=None) -> None:
        c = MpmBatchConfig()
        self._check(self._lib.mpm_batch_get_config(self._h, C.byref(c)))
        if threads is not None:
            c.threads = threads
        if particles_per_cta is not None:
            c.particles_per_cta = particles_per_cta
        if max_cluster is not None:
            c.max_cluster = max_cluster
        if sort_period is not None:
            c.sort_period = sort_period
        self._check(self._lib.mpm_batch_set_config(self._h, C.byref(c)))

    def tune(self, trial_steps: int = 4):
        """Run the autotuner; returns (chosen config, its trial time in ms)."""
        c = MpmBatchConfig()
        ms = C.c_double()
        self._check(self._lib.mpm_batch_tune(self._h, int(trial_steps), C.byref(c), C.byref(ms)))
        return dict(threads=c.threads, particles_per_cta=c.particles_per_cta, max_cluster=c.max_cluster,
                    sort_period=c.sort_period), ms.value

    def close(self) -> None:
        if getattr(self, "_h", None):
            self._lib.mpm_batch_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
