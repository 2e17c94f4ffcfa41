"""B200-native time step of the AWP-ODC anelastic wave solver (pmcl3d).

The compute path is libawpb200.so (hand-written sm_100a CUDA behind a C ABI,
include/awp_b200.h); this package is a thin Python mirror of that ABI.
"""
from ._lib import AwpError, FIELDS, FIELD_ID, LIB_PATH, awp_params, load
from .solver import ALIGN, NGSL, Batch, Mesh, Solver, default_params, padded_shape

__all__ = ["AwpError", "FIELDS", "FIELD_ID", "LIB_PATH", "awp_params", "load", "Batch", "Mesh", "Solver",
           "default_params", "padded_shape", "NGSL", "ALIGN"]
