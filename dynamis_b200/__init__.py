"""dynamis_b200: a B200 (sm_100a) implementation of the Dynamis rigid-body step.

The step itself runs in libdynamis_cuda.so (hand-written CUDA kernels behind the C ABI of
include/dynamis_cuda.h); this package is the Python host mirror of dynamis-world's World API,
the ABI record dtypes and the seeded benchmark scenes.
"""
from . import records
from ._native import DynamisError, lib
from .world import World, default_config

__all__ = ["World", "DynamisError", "default_config", "records", "lib"]
