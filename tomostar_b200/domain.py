"""The forward domain and model (Forward/ForwardDomain.cs, Forward/TravelTimeTable.cs:213-241).

`covering` is ForwardDomain.Covering (on the host); `put_resampled` is ForwardModel.FromInversionGrid
on the device, straight into a resident model that solves, tables and rays use by id.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .grid import GridDef


@dataclass
class Background:
    """VelocityModel1D's nodes (Model/VelocityModel1D.cs): depths (a repeated depth is a discontinuity),
    Vp and Vs in km/s."""

    depth_km: np.ndarray
    vp: np.ndarray
    vs: np.ndarray

    def struct(self) -> L.Background:
        arrs = [np.ascontiguousarray(a, np.float64) for a in (self.depth_km, self.vp, self.vs)]
        b = L.Background(len(arrs[0]), 0, *[a.ctypes.data_as(C.POINTER(C.c_double)) for a in arrs])
        b._keep = arrs
        return b

    @staticmethod
    def layer_mean(grid: GridDef, vp: np.ndarray, vs: np.ndarray) -> "Background":
        """ForwardDomain.LayerMean (Forward/ForwardDomain.cs:120-136): the mean of each depth level of a
        model on the inversion grid, constant below the bottom (a node 1 km above the Earth's centre)."""
        layer = grid.nx * grid.ny
        p = np.asarray(vp, np.float64).reshape(grid.nz, layer)
        s = np.asarray(vs, np.float64).reshape(grid.nz, layer)
        mp = np.array([sum(row) / layer for row in p.tolist()])  # sequential sums, as the reference's loop
        ms = np.array([sum(row) / layer for row in s.tolist()])
        depth = np.append(grid.depth(), 6371.0 - 1)
        return Background(depth, np.append(mp, mp[-1]), np.append(ms, ms[-1]))


def covering(inversion: GridDef, refinement: int, points, max_nodes: int = 12_000_000):
    """ForwardDomain.Covering: (forward GridDef, extended, coarsening factor)."""
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    g = inversion.struct()
    out = L.GridStruct()
    ext = C.c_int32()
    fac = C.c_double()
    rc = L.load().ts_domain_covering(C.byref(g), refinement, len(pts), pts.ctypes.data_as(C.POINTER(C.c_double)),
                                     max_nodes, C.byref(out), C.byref(ext), C.byref(fac))
    if rc != L.TS_OK:
        raise L.TsError(rc, L.load().ts_last_error(None).decode())
    fwd = GridDef(out.min_lon, out.max_lon, out.min_lat, out.max_lat, out.min_depth_km, out.max_depth_km, out.nx,
                  out.ny, out.nz)
    return fwd, bool(ext.value), fac.value


def put_resampled(solver, forward: GridDef, inversion: GridDef, inv_slowness, background: Background | None = None,
                  precision: int = 64) -> int:
    """ForwardModel.FromInversionGrid into a resident model; returns its id (drop it with ts_model_drop)."""
    s = np.ascontiguousarray(inv_slowness, np.float64).reshape(-1, inversion.count)
    fg, ig = forward.struct(), inversion.struct()
    bg = background.struct() if background is not None else None
    mid = C.c_int32()
    rc = L.load().ts_model_put_resampled(solver.handle, C.byref(fg), C.byref(ig),
                                         s.ctypes.data_as(C.POINTER(C.c_double)), len(s),
                                         C.byref(bg) if bg is not None else None, precision, C.byref(mid))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return mid.value


def copy_slowness(solver, model_id: int, phase: int, count: int) -> np.ndarray:
    out = np.empty(count)
    rc = L.load().ts_model_copy_slowness(solver.handle, model_id, phase, out.ctypes.data_as(C.POINTER(C.c_double)))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return out


def set_background(solver, background: Background | None) -> None:
    """The extended domain's background for the rays' outside time (RayKernels.cs:63-65); None clears it."""
    b = background.struct() if background is not None else None
    rc = L.load().ts_set_background(solver.handle, C.byref(b) if b is not None else None)
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
