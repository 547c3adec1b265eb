"""Event location on travel-time tables kept on the device, behind the reference's EventLocator
(Location/EventLocator.cs:59-342) as Relocation.Absolute uses it (Location/Relocation.cs:48-97).

`Tables` is a TravelTimeTableSet on the device (Forward/TravelTimeTable.cs:247-412): built by the
engine from a model and its stations, or uploaded from host float32 tables. `locate` runs
EventLocator.Locate for every event of a job in one call and returns the LocationResult fields of
each event and the residual of every pick.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .grid import GridDef

LocatorSettings = L.LocatorSettings
STATUS = {0: "ok", 1: "too few usable phases", 2: "search box outside the grid"}
LOCATION_DTYPE = np.dtype([(name, np.float64 if ctype is C.c_double else np.int32)
                           for name, ctype in L.Location._fields_])


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


class Tables:
    """Float32 tables of (station, phase) pairs on one uniform grid, resident on the device."""

    def __init__(self, solver, handle: C.c_void_p, grid: GridDef):
        self.solver, self.handle, self.grid = solver, handle, grid

    @classmethod
    def build(cls, solver, grid: GridDef, slowness: np.ndarray, sources: np.ndarray, phases: np.ndarray,
              precision: int = 64) -> "Tables":
        """TravelTimeTableSet.Build: table t is the field of sources[t] for the slowness of phases[t]."""
        sl = np.ascontiguousarray(slowness, np.float64).reshape(-1, grid.count)
        src = np.ascontiguousarray(sources, np.float64)
        ph = np.ascontiguousarray(phases, np.int32)
        h = C.c_void_p()
        stats = L.EikStats()
        gs = grid.struct()
        rc = L.load().ts_tables_build(solver.handle, C.byref(gs), _p(sl, C.c_double), len(sl), len(ph),
                                      _p(src, C.c_double), _p(ph, C.c_int32), precision, C.byref(h), C.byref(stats))
        if rc != L.TS_OK:
            raise L.TsError(rc, solver.last_error)
        t = cls(solver, h, grid)
        t.stats = stats
        return t

    @classmethod
    def upload(cls, solver, grid: GridDef, tables: np.ndarray) -> "Tables":
        tb = np.ascontiguousarray(tables, np.float32).reshape(-1, grid.count)
        h = C.c_void_p()
        gs = grid.struct()
        rc = L.load().ts_tables_upload(solver.handle, C.byref(gs), len(tb), _p(tb, C.c_float), C.byref(h))
        if rc != L.TS_OK:
            raise L.TsError(rc, solver.last_error)
        return cls(solver, h, grid)

    @property
    def count(self) -> int:
        n = C.c_int32()
        L.load().ts_tables_info(self.handle, C.byref(n), None)
        return n.value

    def copy(self, first: int = 0, count: int | None = None) -> np.ndarray:
        count = self.count - first if count is None else count
        out = np.empty((count, self.grid.count), np.float32)
        rc = L.load().ts_tables_copy(self.handle, first, count, _p(out, C.c_float))
        if rc != L.TS_OK:
            raise L.TsError(rc, "table copy failed")
        return out

    def close(self) -> None:
        if self.handle:
            L.load().ts_tables_free(self.handle)
            self.handle = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


@dataclass
class LocateResult:
    locations: np.ndarray    # LOCATION_DTYPE per event
    residuals: np.ndarray    # per pick (NaN for events not located)
    device_ms: float
    candidates: int
    rounds: int


def locate(solver, tables: Tables, start, offsets, table, seconds, weight, correction, table_station,
           settings: LocatorSettings | None = None) -> LocateResult:
    """EventLocator.Locate for every event: start (n_events, 3) lon, lat, depth; event e's picks are
    offsets[e] .. offsets[e+1]-1 (table index, seconds after the catalogue origin time, weight,
    station correction); table_station (n_tables, 2) lon, lat of each table's station."""
    st = np.ascontiguousarray(start, np.float64).reshape(-1, 3)
    off = np.ascontiguousarray(offsets, np.int32)
    tb = np.ascontiguousarray(table, np.int32)
    sec = np.ascontiguousarray(seconds, np.float64)
    w = np.ascontiguousarray(weight, np.float64)
    corr = np.ascontiguousarray(correction, np.float64)
    tsta = np.ascontiguousarray(np.asarray(table_station, np.float64)[:, :2])
    ne = len(off) - 1
    if len(st) != ne:
        raise ValueError("one start location per event")
    out = np.zeros(ne, LOCATION_DTYPE)
    res = np.empty(max(1, len(tb)))
    stats = L.LocateStats()
    s = settings if settings is not None else LocatorSettings()
    rc = L.load().ts_locate(solver.handle, tables.handle, C.byref(s), ne, _p(st, C.c_double), _p(off, C.c_int32),
                            _p(tb, C.c_int32), _p(sec, C.c_double), _p(w, C.c_double), _p(corr, C.c_double),
                            _p(tsta, C.c_double), out.ctypes.data_as(C.POINTER(L.Location)), _p(res, C.c_double),
                            C.byref(stats))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return LocateResult(out, res[: len(tb)], stats.device_ms, stats.candidates, stats.rounds)
