"""EikonalCuda — the CUDA counterpart of the reference's EikonalOpenCl (Forward/EikonalOpenCl.cs).

Same surface, same meaning: `try_create` builds a context and passes the self-test gate or returns
None (EikonalOpenCl.TryCreate, :88-118); `suggest_batch` (:121-132); `try_solve` returns
(ok, reason) and fills a caller-owned field-major output (:138-166); `self_test` (:346-374);
`device`, `last_stats`, `close` (Dispose). The solve runs on the GPU only: there is no CPU path.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Sequence

import numpy as np

from . import _lib as L
from .grid import GridDef

SELF_TEST_TOLERANCE = 1e-6      # EikonalOpenCl.SelfTestTolerance (:45)
SETTLE_TOLERANCE = 1e-7         # SphericalEikonal.SettleTolerance (SphericalEikonal.cs:332)


def _ptr(a: np.ndarray, ct):
    return a.ctypes.data_as(C.POINTER(ct))


def point_source(grid: GridDef, slowness: np.ndarray, lon: float, lat: float, depth_km: float,
                 origin_time: float = 0.0, radius_cells: float = 3.0):
    """SphericalEikonal.PointSource (SphericalEikonal.cs:68-100) via the library's host code."""
    lib = L.load()
    s = np.ascontiguousarray(slowness, np.float64).reshape(-1)
    gs = grid.struct()
    cap = 4096
    while True:
        idx = np.empty(cap, np.int32)
        t = np.empty(cap)
        n = lib.ts_point_source(C.byref(gs), _ptr(s, C.c_double), lon, lat, depth_km, origin_time, radius_cells,
                                _ptr(idx, C.c_int32), _ptr(t, C.c_double), cap)
        if n < 0:
            raise ValueError("invalid grid or slowness")
        if n <= cap:
            return idx[:n].copy(), t[:n].copy()
        cap = n


def pack_seeds(seed_sets: Sequence[tuple[np.ndarray, np.ndarray]]):
    """Seed sets as the C ABI takes them: offsets, node indices, times."""
    off = np.zeros(len(seed_sets) + 1, np.int32)
    for f, (si, _) in enumerate(seed_sets):
        off[f + 1] = off[f] + len(si)
    idx = np.ascontiguousarray(np.concatenate([np.asarray(si, np.int32) for si, _ in seed_sets]) if seed_sets
                               else np.zeros(0, np.int32))
    t = np.ascontiguousarray(np.concatenate([np.asarray(st, np.float64) for _, st in seed_sets]) if seed_sets
                             else np.zeros(0))
    return off, idx, t


class EikonalCuda:
    """A CUDA device that passed the self-test: batched eikonal solves on the B200."""

    def __init__(self, handle, device_index: int, precision: int):
        self._h = handle
        self.device_index = device_index
        self.precision = precision
        self.last_stats_struct = L.EikStats()

    # ---- creation / gate ------------------------------------------------------------------
    @classmethod
    def create(cls, device: int = 0, precision: int = 64) -> "EikonalCuda":
        """A context without the gate (raises when there is no device)."""
        lib = L.load()
        h = C.c_void_p()
        rc = lib.ts_cuda_create(device, C.byref(h))
        if rc != L.TS_OK:
            raise L.TsError(rc, "could not create a CUDA context")
        return cls(h, device, precision)

    @classmethod
    def try_create(cls, log: Callable[[str], None] | None = None, device: int = 0, precision: int = 64):
        """EikonalOpenCl.TryCreate: None when there is no device or the self-test fails."""
        try:
            solver = cls.create(device, precision)
        except (L.TsError, OSError, ImportError) as e:
            if log:
                log(f"CUDA eikonal unavailable ({e}); using CPU.")
            return None
        err, message = solver.self_test()
        if not (err <= SELF_TEST_TOLERANCE):
            if log:
                log(f"CUDA eikonal self-test failed ({message}); using CPU.")
            solver.close()
            return None
        if log:
            log(f"CUDA eikonal ready on {solver.device}: self-test {message}.")
        return solver

    def self_test(self) -> tuple[float, str]:
        """EikonalOpenCl.SelfTest: (max |dt| / field range, message)."""
        lib = L.load()
        rel = C.c_double()
        msg = C.create_string_buffer(256)
        lib.ts_cuda_selftest(self._h, self.precision, C.byref(rel), msg, 256)
        return rel.value, msg.value.decode()

    # ---- properties -----------------------------------------------------------------------
    @property
    def device(self) -> str:
        buf = C.create_string_buffer(256)
        L.load().ts_device_name(self._h, buf, 256)
        return buf.value.decode()

    @property
    def last_stats(self) -> str:
        return L.load().ts_last_stats(self._h).decode()

    @property
    def last_error(self) -> str:
        return L.load().ts_last_error(self._h).decode()

    @property
    def handle(self):
        return self._h

    def suggest_batch(self, nodes: int) -> int:
        """EikonalOpenCl.SuggestBatch."""
        return int(L.load().ts_eik_suggest_batch(self._h, nodes, self.precision))

    def cancel(self, flag: bool = True) -> None:
        L.load().ts_set_cancel(self._h, 1 if flag else 0)

    # ---- solving --------------------------------------------------------------------------
    def solve(self, grid: GridDef, slowness: np.ndarray, seed_sets, output: np.ndarray | None = None,
              mode: int = L.MODE_ENGINE, tol: float = SETTLE_TOLERANCE, max_rounds: int = 0,
              precision: int | None = None) -> np.ndarray:
        """Solves one field per seed set; raises TsError with the reason when the device declines."""
        lib = L.load()
        prec = self.precision if precision is None else precision
        s = np.ascontiguousarray(slowness, np.float64).reshape(-1)
        if s.size != grid.count:
            raise ValueError("Slowness and grid differ in size.")
        off, idx, t = pack_seeds(seed_sets)
        nf = len(seed_sets)
        if output is None:
            output = np.empty((nf, grid.count), np.float64)
        if output.dtype not in (np.float64, np.float32) or not output.flags.c_contiguous:
            raise ValueError("output must be a C-contiguous float64 or float32 array")
        if output.size < nf * grid.count:
            raise ValueError("output too small")
        out_type = L.OUT_F64 if output.dtype == np.float64 else L.OUT_F32
        gs = grid.struct()
        rc = lib.ts_eik_solve(self._h, C.byref(gs), _ptr(s, C.c_double), nf, _ptr(off, C.c_int32),
                              _ptr(idx, C.c_int32), _ptr(t, C.c_double), prec, mode, tol, max_rounds,
                              output.ctypes.data_as(C.c_void_p), out_type, C.byref(self.last_stats_struct))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.last_error)
        return output

    def solve_multi(self, grids: Sequence[GridDef], slownesses: Sequence[np.ndarray], field_grid: Sequence[int],
                    seed_sets, out_dtype=np.float64, mode: int = L.MODE_ENGINE, tol: float = SETTLE_TOLERANCE,
                    max_rounds: int = 0, precision: int | None = None):
        """Fields on grids of uneven size in one engine launch (ts_eik_solve_multi): field f lies on
        grids[field_grid[f]] with seeds seed_sets[f]. Returns one array per field (grid order), or
        None with out_dtype=None (the fields stay on the device; the timing is in last_stats_struct)."""
        lib = L.load()
        prec = self.precision if precision is None else precision
        ng, nf = len(grids), len(seed_sets)
        if len(slownesses) != ng or len(field_grid) != nf:
            raise ValueError("one slowness per grid and one grid index per field")
        keep = [g.struct() for g in grids]  # depth arrays stay alive through the structs' copies
        gs = (L.GridStruct * ng)(*keep)
        sl = [np.ascontiguousarray(s, np.float64).reshape(-1) for s in slownesses]
        for g, s in zip(grids, sl):
            if s.size != g.count:
                raise ValueError("Slowness and grid differ in size.")
        sp = (C.POINTER(C.c_double) * ng)(*[_ptr(s, C.c_double) for s in sl])
        fg = np.ascontiguousarray(field_grid, np.int32)
        off, idx, t = pack_seeds(seed_sets)
        if out_dtype is None:
            out, out_type, buf = None, L.OUT_NONE, None
        else:
            total = sum(grids[int(q)].count for q in fg)
            buf = np.empty(total, out_dtype)
            out_type = L.OUT_F64 if buf.dtype == np.float64 else L.OUT_F32
            out = buf.ctypes.data_as(C.c_void_p)
        rc = lib.ts_eik_solve_multi(self._h, ng, gs, sp, nf, _ptr(fg, C.c_int32), _ptr(off, C.c_int32),
                                    _ptr(idx, C.c_int32), _ptr(t, C.c_double), prec, mode, tol, max_rounds, out,
                                    out_type, C.byref(self.last_stats_struct))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.last_error)
        if buf is None:
            return None
        res, o = [], 0
        for q in fg:
            n = grids[int(q)].count
            res.append(buf[o:o + n])
            o += n
        return res

    def set_graph(self, enable: bool) -> None:
        """Capture one-shot engine solves as CUDA graphs and replay them for repeated jobs."""
        L.check(L.load().ts_engine_set_graph(self._h, 1 if enable else 0), self)

    @property
    def graph_replays(self) -> int:
        return int(L.load().ts_engine_graph_replays(self._h))

    def autotune(self, grids, slownesses, field_grid, seed_sets, mode: int = L.MODE_FAST, repeats: int = 1,
                 precision: int | None = None):
        """Times every compiled tile shape under both schedulers on the sample batch and keeps the
        fastest pair; returns (best shape id, best scheduler, {(shape id, scheduler): ms})."""
        lib = L.load()
        prec = self.precision if precision is None else precision
        ng = len(grids)
        keep = [g.struct() for g in grids]
        gs = (L.GridStruct * ng)(*keep)
        sl = [np.ascontiguousarray(s, np.float64).reshape(-1) for s in slownesses]
        sp = (C.POINTER(C.c_double) * ng)(*[_ptr(s, C.c_double) for s in sl])
        fg = np.ascontiguousarray(field_grid, np.int32)
        off, idx, t = pack_seeds(seed_sets)
        shapes = L.engine_shapes()
        ms = np.full(2 * len(shapes), np.inf)
        best, sched = C.c_int32(-1), C.c_int32(0)
        rc = lib.ts_engine_autotune(self._h, ng, gs, sp, len(seed_sets), _ptr(fg, C.c_int32), _ptr(off, C.c_int32),
                                    _ptr(idx, C.c_int32), _ptr(t, C.c_double), prec, mode, repeats, C.byref(best),
                                    C.byref(sched), _ptr(ms, C.c_double), len(ms))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.last_error)
        table = {(sid, sc): float(ms[2 * q + sc]) for q, (sid, *_) in enumerate(shapes) for sc in (0, 1)}
        return int(best.value), int(sched.value), table

    def try_solve(self, grid: GridDef, slowness: np.ndarray, seed_sets, output: np.ndarray, **kw) -> tuple[bool, str]:
        """EikonalOpenCl.TrySolve: (True, "") or (False, reason); output is field-major."""
        try:
            self.solve(grid, slowness, seed_sets, output, **kw)
            return True, ""
        except L.TsError as e:
            return False, e.reason

    def close(self) -> None:
        if self._h:
            L.load().ts_cuda_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
