"""B200-native constant-pH Monte Carlo energy engine for polyelectrolyte brushes.

The compute path is libphmc.so (CUDA, sm_100a) behind the C ABI in
include/phmc.h; this package holds its Python handle, the model containers
and the workload builders.
"""
from . import _abi
from .engine import Engine, Surrogate
from .model import ModelParams, SystemArrays, build_brush, ewald_alpha, ideal_alpha

__all__ = ["Engine", "Surrogate", "ModelParams", "SystemArrays", "build_brush", "ewald_alpha", "ideal_alpha", "_abi"]
