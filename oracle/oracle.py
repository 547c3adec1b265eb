"""ctypes front end of the C++ oracle (oracle.cpp) — TEST INFRASTRUCTURE ONLY.

The oracle restates the reference's CPU solvers (Forward/SphericalEikonal.cs, Forward/RayTracing.cs,
Forward/TravelTimeTable.cs, Tomography/RayKernels.cs) and the callers beside them (Numerics/Lsqr.cs,
Location/EventLocator.cs, Forward/ForwardDomain.cs). Parity status: the sweeping solver (or_relax,
or_relax_batch) and the LSQR products are pinned bit for bit to the reference's own device kernels
compiled for the CPU (oracle/ref.py, tests/test_ref_pin.py); fast marching, rays and location by the
reference's known-answer tests, LSQR also by SciPy's lsqr. The C# host code itself cannot run here
(no .NET).
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


class GridDef(C.Structure):
    """GridDefinition (Geo/SphericalGrid.cs:13-31) plus an optional depth array."""

    _fields_ = [
        ("min_lon", C.c_double), ("max_lon", C.c_double),
        ("min_lat", C.c_double), ("max_lat", C.c_double),
        ("min_depth_km", C.c_double), ("max_depth_km", C.c_double),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("_pad", C.c_int32),
        ("depth_km", C.POINTER(C.c_double)),
    ]


def build(force: bool = False) -> str:
    """Compile liboracle.so with the committed Makefile (g++ -O2 -ffp-contract=off)."""
    src = os.path.join(HERE, "oracle.cpp")
    if force or not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-C", HERE, "-B" if force else "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)
    return LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        d, i32, i64, dp, fp, ip = C.c_double, C.c_int32, C.c_int64, P(C.c_double), P(C.c_float), P(C.c_int32)
        g = P(GridDef)
        sig = {
            "or_metric": (None, [g, dp, dp, dp, dp]),
            "or_grid_coords": (None, [g, dp, dp, dp, dp]),
            "or_min_spacing_km": (d, [g]),
            "or_to_cartesian": (None, [d, d, d, dp]),
            "or_from_cartesian": (None, [dp, dp]),
            "or_trilinear": (None, [g, d, d, d, ip, dp]),
            "or_interpolate": (d, [g, dp, d, d, d]),
            "or_point_source": (i32, [g, dp, d, d, d, d, d, ip, dp, i32]),
            "or_relax": (i32, [g, dp, i32, ip, dp, i32, d, dp, ip]),
            "or_fmm": (i32, [g, dp, i32, ip, dp, dp]),
            "or_fmm_many": (None, [g, dp, ip, i32, ip, ip, dp, dp, i32]),
            "or_relax_many": (None, [g, dp, ip, i32, ip, ip, dp, d, dp, ip, ip, i32]),
            "or_to_table": (None, [dp, i64, fp]),
            "or_table_time": (d, [g, fp, d, d, d]),
            "or_table_gradient": (None, [g, fp, d, d, d, dp]),
            "or_backtrack": (i32, [g, fp, d, d, d, d, d, d, d, dp, i32]),
            "or_kernel": (i32, [g, dp, i32, ip, dp, i32]),
            "or_ray_row": (i32, [g, fp, d, d, d, g, d, d, d, d, ip, fp, i32, dp]),
            "or_ray_rows_many": (None, [g, fp, ip, dp, g, dp, i32, d, i32, ip, ip, fp, dp, i32]),
            "or_relax_wake": (i32, [g, dp, i32, ip, dp, d, d, i32, dp, ip, P(C.c_int64)]),
            "or_lsqr": (i32, [i32, i32, ip, ip, dp, dp, d, i32, d, d, d, dp, dp]),
            "or_csr_mul": (None, [i32, ip, ip, dp, dp, dp]),
            "or_relax_batch": (i32, [g, dp, i32, ip, ip, dp, i32, d, dp, ip]),
            "or_csr_transpose": (None, [i32, i32, ip, ip, dp, ip, ip, dp]),
            "or_locate_many": (None, [g, fp, i32, dp, C.c_void_p, i32, dp, ip, ip, dp, dp, dp, i32, C.c_void_p,
                                      dp]),
            "or_weighted_median": (d, [i32, dp, dp]),
            "or_median": (d, [i32, dp]),
            "or_gap": (d, [i32, dp]),
            "or_tick_seconds": (d, [d]),
            "or_resample": (None, [g, g, dp, i32, i32, dp, dp, dp, dp]),
            "or_covering": (i32, [g, i32, i32, dp, i64, g, ip, dp]),
            "or_background": (d, [dp, dp, i32, d]),
            "or_ray_rows_many_bg": (None, [g, fp, ip, ip, dp, g, dp, i32, d, i32, ip, ip, fp, dp, i32, dp, dp, dp, dp,
                                           i32]),
        }
        for name, (res, args) in sig.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class Grid:
    """A grid definition with the ctypes struct kept alive (and its depth array, if variable)."""

    def __init__(self, min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km, nx, ny, nz, depth_km=None):
        self.depth = None if depth_km is None else np.ascontiguousarray(depth_km, dtype=np.float64)
        self.struct = GridDef(min_lon, max_lon, min_lat, max_lat, min_depth_km, max_depth_km, nx, ny, nz, 0,
                              None if self.depth is None else _p(self.depth, C.c_double))
        self.nx, self.ny, self.nz = nx, ny, nz

    @classmethod
    def of(cls, g):
        """From any object with the GridDefinition fields (e.g. tomostar_b200.grid.GridDef)."""
        return cls(g.min_lon, g.max_lon, g.min_lat, g.max_lat, g.min_depth_km, g.max_depth_km, g.nx, g.ny, g.nz,
                   getattr(g, "depth_km", None))

    @property
    def count(self):
        return self.nx * self.ny * self.nz

    @property
    def ref(self):
        return C.byref(self.struct)


def metric(g: Grid):
    hlon = np.empty(g.ny * g.nz)
    hlat = np.empty(g.nz)
    hr = C.c_double()
    dz = np.empty(max(1, g.nz - 1))
    lib().or_metric(g.ref, _p(hlon, C.c_double), _p(hlat, C.c_double), C.byref(hr), _p(dz, C.c_double))
    return hlon, hlat, hr.value, (dz if g.depth is not None else None)


def coords(g: Grid):
    lon, lat, cl, dep = np.empty(g.nx), np.empty(g.ny), np.empty(g.ny), np.empty(g.nz)
    lib().or_grid_coords(g.ref, *(_p(a, C.c_double) for a in (lon, lat, cl, dep)))
    return lon, lat, cl, dep


def min_spacing_km(g: Grid) -> float:
    return lib().or_min_spacing_km(g.ref)


def to_cartesian(lon, lat, dep):
    out = np.empty(3)
    lib().or_to_cartesian(lon, lat, dep, _p(out, C.c_double))
    return out


def trilinear(g: Grid, lon, lat, dep):
    nodes = np.empty(8, np.int32)
    w = np.empty(8)
    lib().or_trilinear(g.ref, lon, lat, dep, _p(nodes, C.c_int32), _p(w, C.c_double))
    return nodes, w


def interpolate(g: Grid, field, lon, lat, dep):
    f = np.ascontiguousarray(field, np.float64)
    return lib().or_interpolate(g.ref, _p(f, C.c_double), lon, lat, dep)


def point_source(g: Grid, slowness, lon, lat, dep, origin_time=0.0, radius_cells=3.0):
    """SphericalEikonal.PointSource: (node indices int32, times float64)."""
    s = np.ascontiguousarray(slowness, np.float64)
    cap = 4096
    while True:
        idx = np.empty(cap, np.int32)
        t = np.empty(cap)
        n = lib().or_point_source(g.ref, _p(s, C.c_double), lon, lat, dep, origin_time, radius_cells,
                                  _p(idx, C.c_int32), _p(t, C.c_double), cap)
        if n <= cap:
            return idx[:n].copy(), t[:n].copy()
        cap = n


def relax(g: Grid, slowness, seed_idx, seed_t, tol=1e-7, max_rounds=0):
    """SphericalEikonal.Relax; returns (field, settled, rounds[2])."""
    s = np.ascontiguousarray(slowness, np.float64)
    si = np.ascontiguousarray(seed_idx, np.int32)
    st = np.ascontiguousarray(seed_t, np.float64)
    out = np.empty(g.count)
    rounds = np.zeros(2, np.int32)
    ok = lib().or_relax(g.ref, _p(s, C.c_double), len(si), _p(si, C.c_int32), _p(st, C.c_double), max_rounds, tol,
                        _p(out, C.c_double), _p(rounds, C.c_int32))
    return out, bool(ok), rounds


def relax_batch(g: Grid, slowness, seed_sets, tol=1e-7, max_rounds=0):
    """A batch on one slowness as EikonalOpenCl.Sweep solves it: one round flag for the whole batch.
    Returns (fields (batch, n), settled, rounds[2])."""
    s = np.ascontiguousarray(slowness, np.float64)
    off, idx, t = _seed_arrays(seed_sets)
    out = np.empty((len(seed_sets), g.count))
    rounds = np.zeros(2, np.int32)
    ok = lib().or_relax_batch(g.ref, _p(s, C.c_double), len(seed_sets), _p(off, C.c_int32), _p(idx, C.c_int32),
                              _p(t, C.c_double), max_rounds, tol, _p(out, C.c_double), _p(rounds, C.c_int32))
    return out, bool(ok), rounds


def relax_wake(g: Grid, slowness, seed_idx, seed_t, wake_rel, tol=1e-7, causal=False):
    """Relax with node-level due flags where a drop wakes the neighbours only above wake_rel of the
    new time (wake_rel = 0 is the reference's rule) and, with causal, only the neighbours holding
    more than the new time (the engine's fast mode uses both). Returns (field, settled, rounds[2],
    evaluations)."""
    s = np.ascontiguousarray(slowness, np.float64)
    si = np.ascontiguousarray(seed_idx, np.int32)
    st = np.ascontiguousarray(seed_t, np.float64)
    out = np.empty(g.count)
    rounds = np.zeros(2, np.int32)
    ev = C.c_int64()
    ok = lib().or_relax_wake(g.ref, _p(s, C.c_double), len(si), _p(si, C.c_int32), _p(st, C.c_double), tol, wake_rel,
                             1 if causal else 0, _p(out, C.c_double), _p(rounds, C.c_int32), C.byref(ev))
    return out, bool(ok), rounds, ev.value


def fmm(g: Grid, slowness, seed_idx, seed_t):
    """SphericalEikonal.Solve (fast marching)."""
    s = np.ascontiguousarray(slowness, np.float64)
    si = np.ascontiguousarray(seed_idx, np.int32)
    st = np.ascontiguousarray(seed_t, np.float64)
    out = np.empty(g.count)
    lib().or_fmm(g.ref, _p(s, C.c_double), len(si), _p(si, C.c_int32), _p(st, C.c_double), _p(out, C.c_double))
    return out


def _seed_arrays(seed_sets):
    off = np.zeros(len(seed_sets) + 1, np.int32)
    for f, (si, _) in enumerate(seed_sets):
        off[f + 1] = off[f] + len(si)
    idx = np.concatenate([np.asarray(si, np.int32) for si, _ in seed_sets]) if seed_sets else np.zeros(0, np.int32)
    t = np.concatenate([np.asarray(st, np.float64) for _, st in seed_sets]) if seed_sets else np.zeros(0)
    return off, np.ascontiguousarray(idx), np.ascontiguousarray(t)


def fmm_many(g: Grid, slownesses, sl_of, seed_sets, threads=None):
    """Fast marching of many fields on a thread pool; slownesses is (n_models, n)."""
    s = np.ascontiguousarray(slownesses, np.float64)
    so = np.ascontiguousarray(sl_of, np.int32)
    off, idx, t = _seed_arrays(seed_sets)
    out = np.empty((len(seed_sets), g.count))
    lib().or_fmm_many(g.ref, _p(s, C.c_double), _p(so, C.c_int32), len(seed_sets), _p(off, C.c_int32),
                      _p(idx, C.c_int32), _p(t, C.c_double), _p(out, C.c_double), threads or os.cpu_count())
    return out


def relax_many(g: Grid, slownesses, sl_of, seed_sets, tol=1e-7, threads=None):
    s = np.ascontiguousarray(slownesses, np.float64)
    so = np.ascontiguousarray(sl_of, np.int32)
    off, idx, t = _seed_arrays(seed_sets)
    nf = len(seed_sets)
    out = np.empty((nf, g.count))
    rounds = np.zeros((nf, 2), np.int32)
    settled = np.zeros(nf, np.int32)
    lib().or_relax_many(g.ref, _p(s, C.c_double), _p(so, C.c_int32), nf, _p(off, C.c_int32), _p(idx, C.c_int32),
                        _p(t, C.c_double), tol, _p(out, C.c_double), _p(rounds, C.c_int32),
                        _p(settled, C.c_int32), threads or os.cpu_count())
    return out, settled.astype(bool), rounds


def to_table(t):
    """TravelTimeTable.Write's float32 rounding (non-finite → +inf)."""
    t = np.ascontiguousarray(t, np.float64)
    out = np.empty(t.shape, np.float32)
    lib().or_to_table(_p(t, C.c_double), t.size, _p(out, C.c_float))
    return out


def table_time(g: Grid, table, lon, lat, dep):
    tb = np.ascontiguousarray(table, np.float32)
    return lib().or_table_time(g.ref, _p(tb, C.c_float), lon, lat, dep)


def table_gradient(g: Grid, table, lon, lat, dep):
    tb = np.ascontiguousarray(table, np.float32)
    out = np.empty(3)
    lib().or_table_gradient(g.ref, _p(tb, C.c_float), lon, lat, dep, _p(out, C.c_double))
    return out


def backtrack(g: Grid, table, station, lon, lat, dep, step_km):
    """RayTracing.Backtrack: (n, 3) array of (lon, lat, depth) points, or None."""
    tb = np.ascontiguousarray(table, np.float32)
    cap = 4096
    while True:
        pts = np.empty(3 * cap)
        n = lib().or_backtrack(g.ref, _p(tb, C.c_float), station[0], station[1], station[2], lon, lat, dep, step_km,
                               _p(pts, C.c_double), cap)
        if n == 0:
            return None
        if n > 0:
            return pts[: 3 * n].reshape(n, 3).copy()
        cap = -n


def kernel(inv: Grid, pts):
    """RayTracing.Kernel: (nodes in first-visit order, double lengths)."""
    p = np.ascontiguousarray(pts, np.float64).reshape(-1)
    cap = 8192
    while True:
        nodes = np.empty(cap, np.int32)
        lens = np.empty(cap)
        n = lib().or_kernel(inv.ref, _p(p, C.c_double), len(p) // 3, _p(nodes, C.c_int32), _p(lens, C.c_double), cap)
        if n >= 0:
            return nodes[:n].copy(), lens[:n].copy()
        cap = -n


def ray_row(fwd: Grid, table, station, inv: Grid, event, step_km):
    """One RayKernels arrival: (nodes asc int32, lengths float32, tcalc, (ge, gn, gz)) or None."""
    tb = np.ascontiguousarray(table, np.float32)
    cap = 8192
    while True:
        nodes = np.empty(cap, np.int32)
        lens = np.empty(cap, np.float32)
        tg = np.empty(4)
        n = lib().or_ray_row(fwd.ref, _p(tb, C.c_float), station[0], station[1], station[2], inv.ref, event[0],
                             event[1], event[2], step_km, _p(nodes, C.c_int32), _p(lens, C.c_float), cap,
                             _p(tg, C.c_double))
        if n == -1:
            return None
        if n >= 0:
            return nodes[:n].copy(), lens[:n].copy(), tg[0], tg[1:].copy()
        cap = -2 - n


def ray_rows_many(fwd: Grid, tables, tab_of, stations, inv: Grid, events, step_km, cap_per_row=4096, threads=None):
    """Many arrivals on a thread pool. tables (n_tables, n) float32; stations/events (n_rays, 3).
    nnz[a] >= 0 for a kept row (possibly empty), -1 for an arrival the reference drops."""
    tb = np.ascontiguousarray(tables, np.float32)
    to = np.ascontiguousarray(tab_of, np.int32)
    st = np.ascontiguousarray(stations, np.float64)
    ev = np.ascontiguousarray(events, np.float64)
    nr = len(to)
    nnz = np.zeros(nr, np.int32)
    nodes = np.empty(nr * cap_per_row, np.int32)
    lens = np.empty(nr * cap_per_row, np.float32)
    tg = np.empty((nr, 4))
    lib().or_ray_rows_many(fwd.ref, _p(tb, C.c_float), _p(to, C.c_int32), _p(st, C.c_double), inv.ref,
                           _p(ev, C.c_double), nr, step_km, cap_per_row, _p(nnz, C.c_int32), _p(nodes, C.c_int32),
                           _p(lens, C.c_float), _p(tg, C.c_double), threads or os.cpu_count())
    return nnz, nodes.reshape(nr, cap_per_row), lens.reshape(nr, cap_per_row), tg


LSQR_STOPS = ["empty system", "zero right-hand side", "A^T b = 0", "iteration budget exhausted",
              "residual reduced to tolerance (btol)", "normal equations satisfied (atol)",
              "condition-number limit reached (conlim)", "residual at machine precision",
              "normal equations at machine precision", "condition number at machine precision",
              "bidiagonalisation terminated"]


def lsqr(m, n, row_ptr, col, val, b, damp=0.0, max_iterations=500, atol=1e-8, btol=1e-8, conlim=1e8):
    """Lsqr.Solve (Numerics/Lsqr.cs:33-152) on a CSR matrix; returns (x, stop code, info dict)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col, np.int32)
    va = np.ascontiguousarray(val, np.float64)
    bb = np.ascontiguousarray(b, np.float64)
    x = np.empty(n)
    info = np.empty(4)
    code = lib().or_lsqr(m, n, _p(rp, C.c_int32), _p(ci, C.c_int32), _p(va, C.c_double), _p(bb, C.c_double), damp,
                         max_iterations, atol, btol, conlim, _p(x, C.c_double), _p(info, C.c_double))
    return x, int(code), {"iterations": int(info[0]), "bnorm": info[1], "rnorm": info[2], "acond": info[3]}


def csr_mul(row_ptr, col, val, x):
    """The product or_lsqr forms (CsrMatrix.MultiplyInto: one sequential sum per row)."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col, np.int32)
    va = np.ascontiguousarray(val, np.float64)
    xv = np.ascontiguousarray(x, np.float64)
    y = np.empty(len(rp) - 1)
    lib().or_csr_mul(len(rp) - 1, _p(rp, C.c_int32), _p(ci, C.c_int32), _p(va, C.c_double), _p(xv, C.c_double),
                     _p(y, C.c_double))
    return y


def csr_transpose(m, n, row_ptr, col, val):
    """CsrMatrix.Transpose as or_lsqr builds it: (row_ptr, col, val) of Aᵀ."""
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col, np.int32)
    va = np.ascontiguousarray(val, np.float64)
    trs = np.empty(n + 1, np.int32)
    tci = np.empty(len(ci), np.int32)
    tva = np.empty(len(ci))
    lib().or_csr_transpose(m, n, _p(rp, C.c_int32), _p(ci, C.c_int32), _p(va, C.c_double), _p(trs, C.c_int32),
                           _p(tci, C.c_int32), _p(tva, C.c_double))
    return trs, tci, tva


class LocatorSettings(C.Structure):
    """LocatorSettings (Location/EventLocator.cs:10-36) with the reference's defaults."""

    _fields_ = [("global_search", C.c_int32), ("coarse_candidates", C.c_int32),
                ("max_geiger_iterations", C.c_int32), ("min_phases", C.c_int32), ("damping", C.c_double),
                ("outlier_mads", C.c_double), ("outlier_floor", C.c_double), ("fix_depth", C.c_int32),
                ("reserved", C.c_int32)]

    def __init__(self, **kw):
        base = dict(global_search=1, coarse_candidates=8000, max_geiger_iterations=20, min_phases=4, damping=0.01,
                    outlier_mads=4.0, outlier_floor=0.5, fix_depth=0)
        base.update(kw)
        super().__init__(**base)


LOCATION_FIELDS = ["t0", "lon", "lat", "depth_km", "rms", "err_h_km", "err_minor_km", "err_azimuth_deg",
                   "err_depth_km", "err_time_s", "gap_deg"]
LOCATION_DTYPE = np.dtype([(f, np.float64) for f in LOCATION_FIELDS] +
                          [(f, np.int32) for f in ("used", "rejected", "iterations", "status")])


def locate_many(g: Grid, tables, table_station, settings: LocatorSettings, start, obs_offsets, obs_table, obs_seconds,
                obs_weight, obs_corr, threads=None):
    """EventLocator.Locate for every event (Relocation.Absolute's loop, Location/Relocation.cs:76-91).

    tables: (n_tables, nodes) float32; table_station: (n_tables, 2) lon, lat; start: (n_events, 3)
    lon, lat, depth. Returns (a LOCATION_DTYPE record per event, the residual of every observation).
    """
    tb = np.ascontiguousarray(tables, np.float32)
    ts_ = np.ascontiguousarray(table_station, np.float64)
    st = np.ascontiguousarray(start, np.float64)
    off = np.ascontiguousarray(obs_offsets, np.int32)
    ot = np.ascontiguousarray(obs_table, np.int32)
    osec = np.ascontiguousarray(obs_seconds, np.float64)
    ow = np.ascontiguousarray(obs_weight, np.float64)
    oc = np.ascontiguousarray(obs_corr, np.float64)
    ne = len(off) - 1
    out = np.zeros(ne, LOCATION_DTYPE)
    res = np.empty(max(1, len(ot)))
    lib().or_locate_many(g.ref, _p(tb, C.c_float), len(tb), _p(ts_, C.c_double), C.byref(settings), ne,
                         _p(st, C.c_double), _p(off, C.c_int32), _p(ot, C.c_int32), _p(osec, C.c_double),
                         _p(ow, C.c_double), _p(oc, C.c_double), threads or os.cpu_count(),
                         out.ctypes.data_as(C.c_void_p), _p(res, C.c_double))
    return out, res[: len(ot)]


def weighted_median(v, w):
    v = np.ascontiguousarray(v, np.float64)
    w = np.ascontiguousarray(w, np.float64)
    return lib().or_weighted_median(len(v), _p(v, C.c_double), _p(w, C.c_double))


def median(v):
    v = np.ascontiguousarray(v, np.float64)
    return lib().or_median(len(v), _p(v, C.c_double))


def gap(az):
    a = np.ascontiguousarray(az, np.float64)
    return lib().or_gap(len(a), _p(a, C.c_double))


def tick_seconds(t0):
    return lib().or_tick_seconds(t0)


def resample(fwd: Grid, inv: Grid, inv_slowness, background=None):
    """ForwardModel.FromInversionGrid (Forward/TravelTimeTable.cs:217-241): (n_phases, fwd nodes) slowness.
    background: (depth, vp, vs) arrays of a VelocityModel1D, or None for the plain refined domain."""
    s = np.ascontiguousarray(inv_slowness, np.float64).reshape(-1, inv.count)
    npz = len(s)
    if background is None:
        bd = bp = bs = np.zeros(1)
        nbg = 0
    else:
        bd, bp, bs = (np.ascontiguousarray(a, np.float64) for a in background)
        nbg = len(bd)
    out = np.empty((npz, fwd.count))
    lib().or_resample(fwd.ref, inv.ref, _p(s, C.c_double), npz, nbg, _p(bd, C.c_double), _p(bp, C.c_double),
                      _p(bs, C.c_double), _p(out, C.c_double))
    return out


def covering(inv: Grid, refinement: int, points, max_nodes: int = 12_000_000):
    """ForwardDomain.Covering (Forward/ForwardDomain.cs:51-107): (GridDef fields, extended, coarsening)."""
    pts = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
    out = GridDef()
    ext = C.c_int32()
    fac = C.c_double()
    rc = lib().or_covering(inv.ref, refinement, len(pts), _p(pts, C.c_double), max_nodes, C.byref(out), C.byref(ext),
                           C.byref(fac))
    if rc:
        raise ValueError("Stations and events outside the area span the whole globe")
    fields = (out.min_lon, out.max_lon, out.min_lat, out.max_lat, out.min_depth_km, out.max_depth_km, out.nx, out.ny,
              out.nz)
    return fields, bool(ext.value), fac.value


def background(depth, v, d):
    dd = np.ascontiguousarray(depth, np.float64)
    vv = np.ascontiguousarray(v, np.float64)
    return lib().or_background(_p(dd, C.c_double), _p(vv, C.c_double), len(dd), d)


def ray_rows_many_bg(fwd: Grid, tables, tab_of, tab_phase, stations, inv: Grid, events, step_km, background,
                     cap_per_row=4096, threads=None):
    """ray_rows_many with the extended domain's background (depth, vp, vs): also each row's outside time."""
    tb = np.ascontiguousarray(tables, np.float32)
    to = np.ascontiguousarray(tab_of, np.int32)
    tp = np.ascontiguousarray(tab_phase, np.int32)
    st = np.ascontiguousarray(stations, np.float64)
    ev = np.ascontiguousarray(events, np.float64)
    bd, bp, bs = (np.ascontiguousarray(a, np.float64) for a in background)
    nr = len(to)
    nnz = np.zeros(nr, np.int32)
    nodes = np.empty(nr * cap_per_row, np.int32)
    lens = np.empty(nr * cap_per_row, np.float32)
    tg = np.empty((nr, 4))
    out = np.zeros(nr)
    lib().or_ray_rows_many_bg(fwd.ref, _p(tb, C.c_float), _p(to, C.c_int32), _p(tp, C.c_int32), _p(st, C.c_double),
                              inv.ref, _p(ev, C.c_double), nr, step_km, cap_per_row, _p(nnz, C.c_int32),
                              _p(nodes, C.c_int32), _p(lens, C.c_float), _p(tg, C.c_double), len(bd),
                              _p(bd, C.c_double), _p(bp, C.c_double), _p(bs, C.c_double), _p(out, C.c_double),
                              threads or os.cpu_count())
    return nnz, nodes.reshape(nr, cap_per_row), lens.reshape(nr, cap_per_row), tg, out
