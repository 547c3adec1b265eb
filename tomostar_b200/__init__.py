"""tomostar_b200 — a B200-native (sm_100a) forward engine for TomoSTAR's data-parallel hot path:
spherical eikonal travel-time fields, back-traced rays and their Jacobian rows.

The compute runs in libtomostar_cuda.so (hand-written CUDA behind a C ABI, include/tomostar_cuda.h);
this package is the host-side mirror of the reference's interfaces over that ABI.
"""
from .grid import GridDef  # noqa: F401

__all__ = ["GridDef"]
