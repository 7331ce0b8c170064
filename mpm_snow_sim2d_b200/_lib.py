"""ctypes binding of ``libmpm_b200.so`` (the C ABI in ``include/mpm/mpm.h``).

The library is loaded from the package directory. There is no fallback: if it
is missing or fails to load, every call raises.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libmpm_b200.so"

# mpm_status
OK = 0
STATUS_NAMES = {
    0: "MPM_OK", 1: "MPM_ERR_INVALID_ARGUMENT", 2: "MPM_ERR_CUDA", 3: "MPM_ERR_OUT_OF_MEMORY",
    4: "MPM_ERR_NAN_STATE", 5: "MPM_ERR_FIXED_POINT_OVERFLOW", 6: "MPM_ERR_NO_DEVICE", 7: "MPM_ERR_IO",
    8: "MPM_ERR_STATE_MISMATCH", 9: "MPM_ERR_TIMEOUT", 10: "MPM_ERR_UNSUPPORTED", 11: "MPM_ERR_CAPACITY",
    12: "MPM_ERR_PARTICLE_OUT_OF_DOMAIN",
}
FLAG_NAN_STATE = 1 << 0
FLAG_FIXED_POINT_OVERFLOW = 1 << 1
FLAG_PARTICLE_OUT_OF_DOMAIN = 1 << 2
FLAG_SVD_FP64_FALLBACK = 1 << 3
FLAG_TIMEOUT = 1 << 4

FORMULATION_MLS = 0
FORMULATION_CLASSIC = 1
FORMULATION_MLS_QUADRATIC = 2
BOUNDARY_FRICTION = 0
BOUNDARY_STICKY = 1
PLASTIC_EXACT = 0
PLASTIC_MLP = 1


class MpmParams(C.Structure):
    _fields_ = [
        ("dim", C.c_int32), ("width", C.c_int32), ("height", C.c_int32), ("depth", C.c_int32),
        ("border_margin", C.c_int32), ("formulation", C.c_int32), ("boundary", C.c_int32),
        ("sort_period", C.c_int32),
        ("delta_time", C.c_float), ("gravity", C.c_float), ("friction", C.c_float),
        ("theta_c", C.c_float), ("theta_s", C.c_float), ("xi", C.c_float), ("nu", C.c_float),
        ("youngs", C.c_float), ("rho", C.c_float),
        ("fixed_point_log2_mass", C.c_int32), ("fixed_point_log2_momentum", C.c_int32),
        ("reserved", C.c_int32 * 5),
    ]


class MpmParticlesInit(C.Structure):
    _fields_ = [
        ("count", C.c_int64),
        ("position", C.POINTER(C.c_float)), ("velocity", C.POINTER(C.c_float)),
        ("volume", C.POINTER(C.c_float)), ("mass", C.POINTER(C.c_float)),
    ]


class MpmStateHost(C.Structure):
    _fields_ = [
        ("count", C.c_int64),
        ("position", C.POINTER(C.c_float)), ("velocity", C.POINTER(C.c_float)),
        ("affine_b", C.POINTER(C.c_float)), ("elastic_f", C.POINTER(C.c_float)),
        ("plastic_det", C.POINTER(C.c_float)),
    ]


class MpmShape(C.Structure):
    _fields_ = [("kind", C.c_int32), ("center", C.c_float * 3), ("radius", C.c_float), ("half", C.c_float * 3)]


SHAPE_BALL = 0
SHAPE_BOX = 1


class MpmRenderParams(C.Structure):
    _fields_ = [("width", C.c_int32), ("height", C.c_int32), ("point_size", C.c_float), ("camera_angle", C.c_float),
                ("camera_elevation", C.c_float), ("camera_distance", C.c_float), ("fov_degrees", C.c_float),
                ("reserved", C.c_int32 * 5)]


class MpmBatchConfig(C.Structure):
    _fields_ = [("threads", C.c_int32), ("particles_per_cta", C.c_int32), ("max_cluster", C.c_int32),
                ("sort_period", C.c_int32), ("reserved", C.c_int32 * 4)]


# Every symbol include/mpm/mpm.h declares, with its ctypes signature.
_P = C.c_void_p
SIGNATURES = {
    "mpm_params_default": (None, [C.POINTER(MpmParams), C.c_int32]),
    "mpm_create": (C.c_int, [C.POINTER(MpmParams), C.POINTER(MpmParticlesInit), C.POINTER(_P)]),
    "mpm_destroy": (C.c_int, [_P]),
    "mpm_step": (C.c_int, [_P, C.c_int32]),
    "mpm_get_positions": (C.c_int, [_P, C.POINTER(C.c_float), C.c_size_t]),
    "mpm_get_info": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "mpm_get_state": (C.c_int, [_P, C.POINTER(MpmStateHost)]),
    "mpm_set_state": (C.c_int, [_P, C.POINTER(MpmStateHost)]),
    "mpm_rasterize": (C.c_int, [_P, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_int64), C.c_size_t]),
    "mpm_get_status": (C.c_int, [_P, C.POINTER(C.c_uint32)]),
    "mpm_check_status": (C.c_int, [_P]),
    "mpm_set_stream": (C.c_int, [_P, _P]),
    "mpm_save_state": (C.c_int, [_P, C.c_char_p]),
    "mpm_load_state": (C.c_int, [_P, C.c_char_p]),
    "mpm_get_step": (C.c_int, [_P, C.POINTER(C.c_int64)]),
    "mpm_last_error": (C.c_char_p, [_P]),
    "mpm_status_string": (C.c_char_p, [C.c_int]),
    "mpm_get_fixed_point": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "mpm_step_profiled": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_double), C.c_int32]),
    "mpm_stage_count": (C.c_int32, [_P]),
    "mpm_stage_name": (C.c_char_p, [_P, C.c_int32]),
    "mpm_mlp_param_count": (C.c_int32, []),
    "mpm_mlp_create": (C.c_int, [C.c_uint64, C.POINTER(_P)]),
    "mpm_mlp_destroy": (C.c_int, [_P]),
    "mpm_mlp_last_error": (C.c_char_p, [_P]),
    "mpm_mlp_set_params": (C.c_int, [_P, C.POINTER(C.c_float), C.c_size_t]),
    "mpm_mlp_get_params": (C.c_int, [_P, C.POINTER(C.c_float), C.c_size_t]),
    "mpm_mlp_set_normalization": (C.c_int, [_P] + [C.POINTER(C.c_float)] * 4),
    "mpm_mlp_load_pairs": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int64]),
    "mpm_mlp_train": (C.c_int, [_P, C.c_int32, C.c_int32, C.c_float, C.c_float, C.c_uint32, C.POINTER(C.c_float)]),
    "mpm_mlp_gradient": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float), C.POINTER(C.c_float)]),
    "mpm_mlp_predict": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int64, C.c_int32, C.POINTER(C.c_float)]),
    "mpm_mlp_predict_noalloc": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int64, C.c_int32, C.POINTER(C.c_float)]),
    "mpm_set_plasticity": (C.c_int, [_P, C.c_int32, _P, C.c_float]),
    "mpm_get_mlp_stats": (C.c_int, [_P, C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "mpm_pair_log_enable": (C.c_int, [_P, C.c_int64]),
    "mpm_pair_log_read": (C.c_int, [_P, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_int64)]),
    "mpm_get_sort_stats": (C.c_int, [_P, C.POINTER(C.c_int64), C.POINTER(C.c_int32)]),
    "mpm_sample_shapes": (C.c_int, [C.c_int32, C.POINTER(MpmShape), C.c_int32, C.c_float, C.c_uint64, C.c_int32,
                                     C.POINTER(C.c_float), C.POINTER(C.c_int32), C.c_int64, C.POINTER(C.c_int64)]),
    "mpm_render_params_default": (None, [C.POINTER(MpmRenderParams)]),
    "mpm_render": (C.c_int, [_P, C.POINTER(MpmRenderParams), C.POINTER(C.c_uint8), C.c_size_t]),
    "mpm_batch_create": (C.c_int, [C.POINTER(MpmParams), C.POINTER(MpmParticlesInit), C.c_int32, C.POINTER(_P)]),
    "mpm_batch_destroy": (C.c_int, [_P]),
    "mpm_batch_last_error": (C.c_char_p, [_P]),
    "mpm_batch_info": (C.c_int, [_P, C.POINTER(C.c_int32), C.POINTER(C.c_int64)]),
    "mpm_batch_step": (C.c_int, [_P, C.c_int32]),
    "mpm_batch_set_stream": (C.c_int, [_P, _P]),
    "mpm_batch_get_state": (C.c_int, [_P, C.c_int32, C.POINTER(MpmStateHost)]),
    "mpm_batch_set_state": (C.c_int, [_P, C.c_int32, C.POINTER(MpmStateHost)]),
    "mpm_batch_get_positions": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_float), C.c_size_t]),
    "mpm_batch_get_status": (C.c_int, [_P, C.c_int32, C.POINTER(C.c_uint32)]),
    "mpm_batch_step_times": (C.c_int, [_P, C.POINTER(C.c_uint64), C.c_size_t, C.POINTER(C.c_int32)]),
    "mpm_batch_get_config": (C.c_int, [_P, C.POINTER(MpmBatchConfig)]),
    "mpm_batch_set_config": (C.c_int, [_P, C.POINTER(MpmBatchConfig)]),
    "mpm_batch_tune": (C.c_int, [_P, C.c_int32, C.POINTER(MpmBatchConfig), C.POINTER(C.c_double)]),
}

_lib = None


def load() -> C.CDLL:
    """Load libmpm_b200.so once; raise if it is missing (no fallback path)."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH} is missing: build it with `python -m mpm_snow_sim2d_b200.build` "
            "(the solver has no CPU fallback)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class MpmError(RuntimeError):
    def __init__(self, status: int, detail: str = ""):
        self.status = status
        name = STATUS_NAMES.get(status, f"status {status}")
        super().__init__(f"{name}: {detail}" if detail else name)


def check(status: int, handle=None) -> None:
    if status != OK:
        lib = load()
        detail = ""
        if handle:
            raw = lib.mpm_last_error(handle)
            detail = raw.decode() if raw else ""
        if not detail:
            detail = lib.mpm_status_string(status).decode()
        raise MpmError(status, detail)


def fptr(a):
    """float32 contiguous numpy array -> POINTER(c_float) (None for None)."""
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_float))
