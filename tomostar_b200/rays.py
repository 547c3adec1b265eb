"""Rays and Jacobian rows on the GPU, behind the reference's RayKernels / RayRow surface.

`RayKernels(inversion_grid, forward_grid).compute(...)` mirrors Tomography/RayKernels.cs:30-115 for
curved rays: tables for the (station, phase) pairs in use are solved on the device, rounded to
float32 like the .qttb tables, and every arrival is back-traced (RayTracing.Backtrack) and
integrated on the inversion grid (RayTracing.Kernel). The result is a CSR Jacobian (int32 nodes,
float32 lengths — the RayRow contents, RayKernels.cs:15-19, 96-97) plus TCalc and the source
gradient per arrival; arrivals the reference drops have ok = False.

`trace_rows` traces on tables the caller already has (the per-arrival body alone).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .eikonal import EikonalCuda
from .grid import GridDef


@dataclass
class RayRow:
    """One traced arrival (RayKernels.cs:15): nodes ascending, float32 lengths (km)."""

    arrival: int
    nodes: np.ndarray
    length: np.ndarray
    tcalc: float
    ge: float
    gn: float
    gz: float


@dataclass
class Rows:
    """A CSR Jacobian: row r = arrival r; empty and ok=False where the reference drops the arrival."""

    row_ptr: np.ndarray      # int32 (n_rows + 1)
    col: np.ndarray          # int32 (nnz) inversion-grid node
    len: np.ndarray          # float32 (nnz) km
    tcalc_grad: np.ndarray   # float64 (n_rows, 4): TCalc, Ge, Gn, Gz
    ok: np.ndarray           # bool (n_rows)
    outside: np.ndarray | None = None  # float64 (n_rows): RayRow.OutsideTime (0 without a background)

    @property
    def n_rows(self) -> int:
        return len(self.ok)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1]) if len(self.row_ptr) else 0

    def row(self, r: int) -> RayRow | None:
        if not self.ok[r]:
            return None
        b, e = self.row_ptr[r], self.row_ptr[r + 1]
        t = self.tcalc_grad[r]
        return RayRow(r, self.col[b:e], self.len[b:e], float(t[0]), float(t[1]), float(t[2]), float(t[3]))

    def rows(self) -> list[RayRow]:
        """The reference's List<RayRow>, ordered by arrival, dropped arrivals left out."""
        return [r for r in (self.row(q) for q in range(self.n_rows)) if r is not None]

    def bytes(self) -> int:
        return self.row_ptr.nbytes + self.col.nbytes + self.len.nbytes + self.tcalc_grad.nbytes + self.ok.nbytes


def _fetch(handle) -> Rows:
    lib = L.load()
    n = C.c_int32()
    nnz = C.c_int64()
    lib.ts_rows_info(handle, C.byref(n), C.byref(nnz))
    rp = np.empty(n.value + 1, np.int32)
    col = np.empty(nnz.value, np.int32)
    ln = np.empty(nnz.value, np.float32)
    tg = np.empty((n.value, 4))
    ok = np.empty(n.value, np.uint8)
    P = C.POINTER
    rc = lib.ts_rows_copy(handle, rp.ctypes.data_as(P(C.c_int32)), col.ctypes.data_as(P(C.c_int32)),
                          ln.ctypes.data_as(P(C.c_float)), tg.ctypes.data_as(P(C.c_double)),
                          ok.ctypes.data_as(P(C.c_uint8)))
    out = np.empty(n.value)
    if rc == L.TS_OK:
        rc = lib.ts_rows_outside(handle, out.ctypes.data_as(P(C.c_double)))
    lib.ts_rows_free(handle)
    if rc != L.TS_OK:
        raise L.TsError(rc, "copying rows")
    return Rows(rp, col, ln, tg, ok.astype(bool), out)


def step_km(forward: GridDef, inversion: GridDef) -> float:
    """The back-tracing step of RayKernels.cs:62."""
    return 0.5 * min(forward.min_spacing_km(), inversion.min_spacing_km())


def trace_rows(solver: EikonalCuda, forward: GridDef, tables: np.ndarray, table_station: np.ndarray,
               inversion: GridDef, table_of: np.ndarray, events: np.ndarray, step: float | None = None) -> Rows:
    """Backtrack + Kernel of every ray on given float32 tables (n_tables, n)."""
    lib = L.load()
    tb = np.ascontiguousarray(tables, np.float32).reshape(-1, forward.count)
    ts_ = np.ascontiguousarray(table_station, np.float64).reshape(-1, 3)
    to = np.ascontiguousarray(table_of, np.int32)
    ev = np.ascontiguousarray(events, np.float64).reshape(-1, 3)
    if len(ev) != len(to):
        raise ValueError("one event per ray")
    fs, is_ = forward.struct(), inversion.struct()
    h = C.c_void_p()
    P = C.POINTER
    rc = lib.ts_rays_trace(solver.handle, C.byref(fs), len(tb), tb.ctypes.data_as(P(C.c_float)),
                           ts_.ctypes.data_as(P(C.c_double)), C.byref(is_), len(to), to.ctypes.data_as(P(C.c_int32)),
                           ev.ctypes.data_as(P(C.c_double)), step or step_km(forward, inversion), C.byref(h))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return _fetch(h)


class RayKernels:
    """RayKernels(grid, forwardGrid, RayMethod.FastMarching) with the tables on the GPU."""

    def __init__(self, inversion: GridDef, forward: GridDef, solver: EikonalCuda):
        self.grid = inversion
        self.forward = forward
        self.solver = solver
        self.last_stats = L.EikStats()

    def compute(self, slowness_fwd: np.ndarray, stations: np.ndarray, events: np.ndarray, arrivals: np.ndarray,
                precision: int | None = None, step: float | None = None, mode: int = L.MODE_FAST) -> Rows:
        """slowness_fwd: (n_phases, n) on the forward grid (ForwardModel); stations/events (k, 3)
        lon, lat, depth; arrivals (m, 3) int (event, station, phase). mode: L.MODE_FAST (tables within
        1e-10 relative of the reference's fields) or L.MODE_ENGINE (the reference's to the bit)."""
        lib = L.load()
        s = np.ascontiguousarray(slowness_fwd, np.float64).reshape(-1, self.forward.count)
        st = np.ascontiguousarray(stations, np.float64).reshape(-1, 3)
        ev = np.ascontiguousarray(events, np.float64).reshape(-1, 3)
        ar = np.ascontiguousarray(arrivals, np.int32).reshape(-1, 3)
        ae, ast, ap = (np.ascontiguousarray(ar[:, q]) for q in range(3))
        fs, is_ = self.forward.struct(), self.grid.struct()
        h = C.c_void_p()
        P = C.POINTER
        prec = self.solver.precision if precision is None else precision
        rc = lib.ts_forward(self.solver.handle, C.byref(fs), s.ctypes.data_as(P(C.c_double)), len(s), C.byref(is_),
                            len(st), st.ctypes.data_as(P(C.c_double)), len(ev), ev.ctypes.data_as(P(C.c_double)),
                            len(ar), ae.ctypes.data_as(P(C.c_int32)), ast.ctypes.data_as(P(C.c_int32)),
                            ap.ctypes.data_as(P(C.c_int32)), prec, mode, step or 0.0, C.byref(h),
                            C.byref(self.last_stats))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.solver.last_error)
        return _fetch(h)
