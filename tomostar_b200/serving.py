"""The serving engine (ts_serve_*): a resident request loop with continuous batching.

Requests for travel-time fields — and rays on them — arrive from inversion iterations, L-curve
sweeps, resolution tests and relocation at their own pace and on grids of their own. `Server` keeps
the velocity models on the device; each `submit` queues a request (fields on one model and phase,
optionally rays), which is admitted when its device footprint fits in the HBM budget and then
solved by the engine together with every other field in flight, in epochs of a few sweep rounds.
`wait` returns the request's latency, rows (a CSR Jacobian, as RayKernels.Compute builds) and, if
asked for, its float32 tables. A field's result is the same whatever it was solved with.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib as L
from .eikonal import pack_seeds
from .grid import GridDef
from .rays import Rows, _fetch


@dataclass
class ServeResult:
    status: int
    error: str
    n_fields: int
    rounds: tuple[int, int]
    queue_ms: float
    latency_ms: float
    rows: Rows | None
    tables: np.ndarray | None


class Server:
    """One serving loop on one GPU (ts_serve_create)."""

    def __init__(self, device: int = 0, precision: int = 64, mode: int = L.MODE_FAST, tile: int = 2,
                 budget_bytes: float = 120e9, rounds_per_epoch: int = 1, scheduler: int = 0,
                 epoch_ms: float = 0.0):
        lib = L.load()
        h = C.c_void_p()
        rc = lib.ts_serve_create(device, precision, mode, tile, scheduler, float(budget_bytes), rounds_per_epoch,
                                 C.byref(h))
        if rc != L.TS_OK:
            raise L.TsError(rc, "ts_serve_create")
        self._h = h
        if epoch_ms > 0:
            L.check(lib.ts_serve_set_epoch_ms(h, float(epoch_ms)))
        self._models: dict[int, GridDef] = {}
        self._keep: dict[int, tuple] = {}

    @property
    def last_error(self) -> str:
        return L.load().ts_serve_last_error(self._h).decode()

    def model_put(self, grid: GridDef, slowness: np.ndarray) -> int:
        """A resident model: slowness of shape (n_phases, n) or (n,)."""
        s = np.ascontiguousarray(slowness, np.float64)
        phases = 1 if s.ndim == 1 else s.shape[0]
        if s.size != phases * grid.count:
            raise ValueError("Slowness and grid differ in size.")
        gs = grid.struct()
        mid = C.c_int32()
        rc = L.load().ts_serve_model_put(self._h, C.byref(gs), s.ctypes.data_as(C.POINTER(C.c_double)), phases,
                                         C.byref(mid))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.last_error)
        self._models[mid.value] = grid
        return mid.value

    def submit(self, model: int, phase: int, seed_sets, origins: np.ndarray | None = None,
               ray_field: Sequence[int] | None = None, ray_event: np.ndarray | None = None,
               inv: GridDef | None = None, step_km: float = 0.0, tables: bool = False) -> int:
        """Queues fields (one per seed set) on a model and phase, and rays traced on them from each
        ray's event to its field's origin. Returns the request id."""
        grid = self._models[model]
        off, idx, t = pack_seeds(seed_sets)
        nf = len(seed_sets)
        q = L.ServeRequest()
        q.model_id, q.phase, q.n_fields = model, phase, nf
        P = C.POINTER
        q.seed_offsets = off.ctypes.data_as(P(C.c_int32))
        q.seed_index = idx.ctypes.data_as(P(C.c_int32))
        q.seed_time = t.ctypes.data_as(P(C.c_double))
        keep = [off, idx, t]
        if origins is not None:
            o = np.ascontiguousarray(origins, np.float64).reshape(nf, 3)
            q.field_origin = o.ctypes.data_as(P(C.c_double))
            keep.append(o)
        if ray_field is not None and len(ray_field):
            rf = np.ascontiguousarray(ray_field, np.int32)
            ev = np.ascontiguousarray(ray_event, np.float64).reshape(len(rf), 3)
            q.n_rays = len(rf)
            q.ray_field = rf.ctypes.data_as(P(C.c_int32))
            q.ray_event = ev.ctypes.data_as(P(C.c_double))
            keep += [rf, ev]
        if inv is not None:
            ig = inv.struct()
            q.inv = C.pointer(ig)
            keep.append(ig)
        q.step_km = step_km
        out = None
        if tables:
            out = np.empty((nf, grid.count), np.float32)
            q.tables_out = out.ctypes.data_as(P(C.c_float))
        rid = C.c_int64()
        rc = L.load().ts_serve_submit(self._h, C.byref(q), C.byref(rid))
        if rc != L.TS_OK:
            raise L.TsError(rc, self.last_error)
        self._keep[rid.value] = (out,)  # the table buffer must outlive the request
        return rid.value

    def wait(self, rid: int, timeout: float | None = None) -> ServeResult | None:
        """The request's result, or None if it is not done within timeout seconds."""
        res = L.ServeResult()
        rc = L.load().ts_serve_wait(self._h, rid, -1.0 if timeout is None else float(timeout), C.byref(res))
        if rc == L.TS_E_TIMEOUT:
            return None
        if rc != L.TS_OK:
            raise L.TsError(rc, "unknown request")
        rows = _fetch(C.c_void_p(res.rows)) if res.rows else None
        out = self._keep.pop(rid, (None,))[0]
        return ServeResult(res.status, res.error.decode(), res.n_fields, (res.rounds[0], res.rounds[1]), res.queue_ms,
                           res.latency_ms, rows, out if res.status == L.TS_OK else None)

    def stats(self) -> dict:
        st = L.ServeStats()
        L.load().ts_serve_stats(self._h, C.byref(st))
        return {k: getattr(st, k) for k, _ in L.ServeStats._fields_}

    def close(self) -> None:
        if self._h:
            L.load().ts_serve_destroy(self._h)
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
