"""Grid definitions of the forward path (Geo/SphericalGrid.cs) on the host side of the C ABI.

`GridDef` is the reference's GridDefinition (SphericalGrid.cs:13-75), with an optional depth array
for the variable-vertical-spacing extension. Node coordinates and trilinear resampling
(SphericalGrid.cs:96-116, 205-252) are vectorised with numpy for building forward models.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field, replace

import numpy as np

from ._lib import GridStruct

EARTH_RADIUS_KM = 6371.0  # Geo/GeoMath.cs:43
DEG2RAD = math.pi / 180.0


@dataclass(frozen=True)
class GridDef:
    """GridDefinition: nodes on the bounds, index x (lon) fastest, then y (lat), then z (depth)."""

    min_lon: float
    max_lon: float
    min_lat: float
    max_lat: float
    min_depth_km: float
    max_depth_km: float
    nx: int
    ny: int
    nz: int
    depth_km: np.ndarray | None = field(default=None, compare=False)

    @property
    def dlon(self) -> float:
        return (self.max_lon - self.min_lon) / max(1, self.nx - 1)

    @property
    def dlat(self) -> float:
        return (self.max_lat - self.min_lat) / max(1, self.ny - 1)

    @property
    def ddepth(self) -> float:
        return (self.max_depth_km - self.min_depth_km) / max(1, self.nz - 1)

    @property
    def count(self) -> int:
        return self.nx * self.ny * self.nz

    @property
    def shape(self) -> tuple[int, int, int]:
        """numpy shape of a field in grid order: (nz, ny, nx)."""
        return (self.nz, self.ny, self.nx)

    def refined(self, factor: int) -> "GridDef":
        """GridDefinition.Refined (SphericalGrid.cs:51-56)."""
        if factor <= 1:
            return self
        return replace(self, nx=(self.nx - 1) * factor + 1, ny=(self.ny - 1) * factor + 1,
                       nz=(self.nz - 1) * factor + 1, depth_km=None)

    def coarsened(self, factor: int) -> "GridDef":
        """The inversion grid a forward grid refines by `factor` (inverse of refined)."""
        return replace(self, nx=(self.nx - 1) // factor + 1, ny=(self.ny - 1) // factor + 1,
                       nz=(self.nz - 1) // factor + 1, depth_km=None)

    @staticmethod
    def from_spacing(min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km, horizontal_km, vertical_km):
        """GridDefinition.FromSpacing (SphericalGrid.cs:59-74)."""
        mid = 0.5 * (min_lat + max_lat) * DEG2RAD
        width = (max_lon - min_lon) * DEG2RAD * EARTH_RADIUS_KM * math.cos(mid)
        height = (max_lat - min_lat) * DEG2RAD * EARTH_RADIUS_KM
        rnd = lambda v: int(np.round(v))  # Math.Round: half to even
        return GridDef(min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km,
                       max(2, rnd(width / horizontal_km) + 1), max(2, rnd(height / horizontal_km) + 1),
                       max(2, rnd((max_depth_km - min_depth_km) / vertical_km) + 1))

    # ---- coordinates -----------------------------------------------------------------------
    def lon(self) -> np.ndarray:
        return self.min_lon + np.arange(self.nx) * self.dlon

    def lat(self) -> np.ndarray:
        return self.min_lat + np.arange(self.ny) * self.dlat

    def depth(self) -> np.ndarray:
        if self.depth_km is not None:
            return np.asarray(self.depth_km, np.float64)
        return self.min_depth_km + np.arange(self.nz) * self.ddepth

    def min_spacing_km(self) -> float:
        """SphericalGrid.MinSpacingKm (SphericalGrid.cs:159-164)."""
        dep = self.depth()
        r_min = EARTH_RADIUS_KM - dep[-1]
        cos_min = float(np.min(np.cos(self.lat() * DEG2RAD)))
        dz = self.ddepth if self.depth_km is None else float(np.min(np.diff(dep)))
        return min(dz, min(r_min * self.dlat * DEG2RAD, r_min * cos_min * self.dlon * DEG2RAD))

    def fractional(self, lon, lat, depth_km):
        """SphericalGrid.Fractional (SphericalGrid.cs:179-184), vectorised (no longitude unwrap)."""
        fx = (np.asarray(lon) - self.min_lon) / self.dlon
        fy = (np.asarray(lat) - self.min_lat) / self.dlat
        if self.depth_km is None:
            fz = (np.asarray(depth_km) - self.min_depth_km) / self.ddepth
        else:
            dep = self.depth()
            d = np.asarray(depth_km, np.float64)
            k = np.clip(np.searchsorted(dep, d, side="right") - 1, 0, self.nz - 2)
            fz = k + (d - dep[k]) / (dep[k + 1] - dep[k])
        return fx, fy, fz

    def interpolate(self, field: np.ndarray, lon, lat, depth_km) -> np.ndarray:
        """SphericalGrid.Interpolate at many points (trilinear, clamped; SphericalGrid.cs:205-235)."""
        f = np.asarray(field, np.float64).reshape(-1)
        fx, fy, fz = self.fractional(lon, lat, depth_km)
        fx = np.clip(fx, 0, self.nx - 1)
        fy = np.clip(fy, 0, self.ny - 1)
        fz = np.clip(fz, 0, self.nz - 1)
        i0 = np.minimum(fx.astype(np.int64), self.nx - 2)
        j0 = np.minimum(fy.astype(np.int64), self.ny - 2)
        k0 = np.minimum(fz.astype(np.int64), self.nz - 2)
        tx, ty, tz = fx - i0, fy - j0, fz - k0
        out = np.zeros(np.broadcast(fx, fy, fz).shape)
        for dk in (0, 1):
            for dj in (0, 1):
                for di in (0, 1):
                    w = (tx if di else 1 - tx) * (ty if dj else 1 - ty) * (tz if dk else 1 - tz)
                    out += f[((k0 + dk) * self.ny + (j0 + dj)) * self.nx + (i0 + di)] * w
        return out

    def resample_from(self, source: "GridDef", field: np.ndarray) -> np.ndarray:
        """SphericalGrid.ResampleFrom (SphericalGrid.cs:241-252): source-grid field onto this grid."""
        lon, lat, dep = np.meshgrid(self.lon(), self.lat(), self.depth(), indexing="ij")
        # grid order (z, y, x)
        lon, lat, dep = (a.transpose(2, 1, 0) for a in (lon, lat, dep))
        return source.interpolate(field, lon, lat, dep).reshape(-1)

    # ---- C ABI -----------------------------------------------------------------------------
    def struct(self) -> GridStruct:
        s = GridStruct(self.min_lon, self.max_lon, self.min_lat, self.max_lat, self.min_depth_km, self.max_depth_km,
                       self.nx, self.ny, self.nz, 0, None)
        if self.depth_km is not None:
            arr = np.ascontiguousarray(self.depth_km, np.float64)
            s._keep = arr  # keep the array alive with the struct
            s.depth_km = arr.ctypes.data_as(C.POINTER(C.c_double))
        return s
