"""B200-native (sm_100a) MLS-MPM snow solver with the simulation surface of
michal-sitarz2/MPM_Snow_Sim2D (Parameters.h knobs, per-step P2G -> grid update
-> G2P with Stomakhin hardening and critical compression/stretch clamps, in
2D and 3D). The compute path is hand-written CUDA behind the C ABI in
include/mpm/mpm.h; this package is its Python host mirror.
"""
from ._lib import MpmError, MpmParams  # noqa: F401
from .solver import Solver, State, params_from_scene  # noqa: F401
from . import scenes  # noqa: F401
