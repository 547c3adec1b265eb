"""Loads libtomostar_cuda.so (built in-tree) and declares the C ABI of include/tomostar_cuda.h.

There is no fallback: if the library is missing the import of the solver fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtomostar_cuda.so")

TS_OK, TS_E_ARG, TS_E_CUDA, TS_E_NOMEM, TS_E_UNSETTLED, TS_E_CANCELLED = 0, 1, 2, 3, 4, 5
TS_E_TIMEOUT, TS_E_CAPACITY, TS_E_NOSEEDS, TS_E_SELFTEST, TS_E_NODEVICE = 6, 7, 8, 9, 10
F64, F32 = 64, 32
MODE_ENGINE, MODE_PLAIN, MODE_FAST = 0, 1, 2
WAKE_REL = 1e-13
OUT_F64, OUT_F32, OUT_NONE = 0, 1, 2

ERROR_NAMES = {
    TS_E_ARG: "invalid argument", TS_E_CUDA: "CUDA error", TS_E_NOMEM: "out of device memory",
    TS_E_UNSETTLED: "not settled", TS_E_CANCELLED: "cancelled", TS_E_TIMEOUT: "device wait timed out",
    TS_E_CAPACITY: "capacity", TS_E_NOSEEDS: "no seed nodes", TS_E_SELFTEST: "self-test failed",
    TS_E_NODEVICE: "no CUDA device",
}


class TsError(RuntimeError):
    def __init__(self, code: int, reason: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {reason}")
        self.code = code
        self.reason = reason


class GridStruct(C.Structure):
    """ts_grid = GridDefinition (Geo/SphericalGrid.cs:13-31) + optional depth array."""

    _fields_ = [
        ("min_lon", C.c_double), ("max_lon", C.c_double),
        ("min_lat", C.c_double), ("max_lat", C.c_double),
        ("min_depth_km", C.c_double), ("max_depth_km", C.c_double),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32), ("reserved", C.c_int32),
        ("depth_km", C.POINTER(C.c_double)),
    ]


class EikStats(C.Structure):
    _fields_ = [
        ("rounds", C.c_int32 * 2), ("launches", C.c_int32), ("reserved", C.c_int32),
        ("node_updates", C.c_int64), ("tile_visits", C.c_int64), ("device_ms", C.c_double),
        ("kernel_ms", C.c_double),
    ]


# Every symbol the header declares, with its ctypes signature.
_P = C.POINTER
_vp, _i32, _i64, _d = C.c_void_p, C.c_int32, C.c_int64, C.c_double
_ip, _dp, _fp, _u8p = _P(C.c_int32), _P(C.c_double), _P(C.c_float), _P(C.c_uint8)
class ServeRequest(C.Structure):
    """ts_serve_request."""

    _fields_ = [
        ("model_id", C.c_int32), ("phase", C.c_int32), ("n_fields", C.c_int32), ("n_rays", C.c_int32),
        ("seed_offsets", C.POINTER(C.c_int32)), ("seed_index", C.POINTER(C.c_int32)),
        ("seed_time", C.POINTER(C.c_double)), ("field_origin", C.POINTER(C.c_double)),
        ("ray_field", C.POINTER(C.c_int32)), ("ray_event", C.POINTER(C.c_double)),
        ("inv", C.POINTER(GridStruct)), ("step_km", C.c_double), ("tables_out", C.POINTER(C.c_float)),
    ]


class ServeResult(C.Structure):
    """ts_serve_result."""

    _fields_ = [
        ("status", C.c_int32), ("n_fields", C.c_int32), ("rounds", C.c_int32 * 2), ("queue_ms", C.c_double),
        ("latency_ms", C.c_double), ("rows", C.c_void_p), ("error", C.c_char * 160),
    ]


class ServeStats(C.Structure):
    """ts_serve_stats_t."""

    _fields_ = [
        ("epochs", C.c_int64), ("fields_done", C.c_int64), ("requests_done", C.c_int64),
        ("node_updates", C.c_int64), ("device_ms", C.c_double), ("epoch_ms", C.c_double),
        ("complete_ms", C.c_double), ("bytes_in_use", C.c_double),
        ("peak_bytes", C.c_double), ("queued", C.c_int32), ("in_flight", C.c_int32),
    ]


class LsqrInfo(C.Structure):
    """ts_lsqr_info."""

    _fields_ = [("iterations", C.c_int32), ("stop", C.c_int32), ("bnorm", C.c_double), ("rnorm", C.c_double),
                ("acond", C.c_double), ("device_ms", C.c_double)]


class LocatorSettings(C.Structure):
    """ts_locator_settings = LocatorSettings (Location/EventLocator.cs:10-36), the reference's defaults."""

    _fields_ = [("global_search", C.c_int32), ("coarse_candidates", C.c_int32),
                ("max_geiger_iterations", C.c_int32), ("min_phases", C.c_int32), ("damping", C.c_double),
                ("outlier_mads", C.c_double), ("outlier_floor", C.c_double), ("fix_depth", C.c_int32),
                ("reserved", C.c_int32)]

    def __init__(self, **kw):
        base = dict(global_search=1, coarse_candidates=8000, max_geiger_iterations=20, min_phases=4, damping=0.01,
                    outlier_mads=4.0, outlier_floor=0.5, fix_depth=0)
        base.update(kw)
        super().__init__(**base)


class Location(C.Structure):
    """ts_location = LocationResult + Hypocentre."""

    _fields_ = [(f, C.c_double) for f in ("t0", "lon", "lat", "depth_km", "rms", "err_h_km", "err_minor_km",
                                          "err_azimuth_deg", "err_depth_km", "err_time_s", "gap_deg")] + \
               [(f, C.c_int32) for f in ("used", "rejected", "iterations", "status")]


class LocateStats(C.Structure):
    """ts_locate_stats."""

    _fields_ = [("device_ms", C.c_double), ("candidates", C.c_int64), ("rounds", C.c_int32),
                ("reserved", C.c_int32)]


class Background(C.Structure):
    """ts_background: a VelocityModel1D's nodes."""

    _fields_ = [("n", C.c_int32), ("reserved", C.c_int32), ("depth_km", _P(C.c_double)), ("vp", _P(C.c_double)),
                ("vs", _P(C.c_double))]


_gp = _P(GridStruct)
SIGNATURES = {
    "ts_domain_covering": (C.c_int, [_gp, _i32, _i32, _P(C.c_double), _i64, _gp, _P(_i32), _P(C.c_double)]),
    "ts_model_put_resampled": (C.c_int, [_vp, _gp, _gp, _P(C.c_double), _i32, _P(Background), _i32, _P(_i32)]),
    "ts_model_copy_slowness": (C.c_int, [_vp, _i32, _i32, _P(C.c_double)]),
    "ts_set_background": (C.c_int, [_vp, _P(Background)]),
    "ts_rows_outside": (C.c_int, [_vp, _P(C.c_double)]),
    "ts_tables_build": (C.c_int, [_vp, _gp, _dp, _i32, _i32, _dp, _ip, _i32, _P(_vp), _P(EikStats)]),
    "ts_tables_upload": (C.c_int, [_vp, _gp, _i32, _fp, _P(_vp)]),
    "ts_tables_info": (C.c_int, [_vp, _P(_i32), _P(_i64)]),
    "ts_tables_copy": (C.c_int, [_vp, _i32, _i32, _fp]),
    "ts_tables_free": (None, [_vp]),
    "ts_tables_write_qttb": (C.c_int, [_vp, _i32, _i32, _P(C.c_char_p), _P(C.c_char_p), _P(_i32)]),
    "ts_tables_load_qttb": (C.c_int, [_vp, _gp, _i32, _P(C.c_char_p), _P(_vp)]),
    "ts_locate": (C.c_int, [_vp, _vp, _P(LocatorSettings), _i32, _dp, _ip, _ip, _dp, _dp, _dp, _dp, _P(Location),
                            _dp, _P(LocateStats)]),
    "ts_lsqr_solve": (C.c_int, [_vp, _i32, _i32, _ip, _ip, _dp, _dp, _d, _i32, _d, _d, _d, _dp, _P(LsqrInfo)]),
    "ts_lsqr_solve_rows": (C.c_int, [_vp, _vp, _i32, _dp, _d, _i32, _d, _d, _d, _dp, _P(LsqrInfo)]),
    "ts_lsqr_set_callback": (C.c_int, [_vp, C.c_void_p, _vp]),
    "ts_lsqr_selftest": (C.c_int, [_vp, _dp, C.c_char_p, _i32]),
    "ts_serve_create": (C.c_int, [_i32, _i32, _i32, _i32, _i32, _d, _i32, _P(_vp)]),
    "ts_serve_destroy": (None, [_vp]),
    "ts_serve_set_epoch_ms": (C.c_int, [_vp, _d]),
    "ts_serve_last_error": (C.c_char_p, [_vp]),
    "ts_serve_model_put": (C.c_int, [_vp, _gp, _dp, _i32, _ip]),
    "ts_serve_submit": (C.c_int, [_vp, _P(ServeRequest), _P(C.c_int64)]),
    "ts_serve_wait": (C.c_int, [_vp, C.c_int64, _d, _P(ServeResult)]),
    "ts_serve_stats": (C.c_int, [_vp, _P(ServeStats)]),
    "ts_cuda_create": (C.c_int, [_i32, _P(_vp)]),
    "ts_cuda_destroy": (None, [_vp]),
    "ts_last_error": (C.c_char_p, [_vp]),
    "ts_device_name": (C.c_int, [_vp, C.c_char_p, _i32]),
    "ts_last_stats": (C.c_char_p, [_vp]),
    "ts_set_cancel": (None, [_vp, _i32]),
    "ts_eik_suggest_batch": (_i32, [_vp, _i64, _i32]),
    "ts_engine_shapes": (_i32, [_ip, _i32]),
    "ts_engine_set_tile": (C.c_int, [_vp, _i32, _i32]),
    "ts_engine_set_scheduler": (C.c_int, [_vp, _i32]),
    "ts_eik_solve_multi": (C.c_int, [_vp, _i32, _gp, _P(_dp), _i32, _ip, _ip, _ip, _dp, _i32, _i32, _d, _i32, _vp, _i32,
                                     _P(EikStats)]),
    "ts_engine_set_graph": (C.c_int, [_vp, _i32]),
    "ts_engine_graph_replays": (_i32, [_vp]),
    "ts_engine_autotune": (C.c_int, [_vp, _i32, _gp, _P(_dp), _i32, _ip, _ip, _ip, _dp, _i32, _i32, _i32, _ip, _ip,
                                     _dp, _i32]),
    "ts_point_source": (_i32, [_gp, _dp, _d, _d, _d, _d, _d, _ip, _dp, _i32]),
    "ts_eik_solve": (C.c_int, [_vp, _gp, _dp, _i32, _ip, _ip, _dp, _i32, _i32, _d, _i32, _vp, _i32, _P(EikStats)]),
    "ts_model_put": (C.c_int, [_vp, _gp, _dp, _i32, _i32, _ip]),
    "ts_model_drop": (C.c_int, [_vp, _i32]),
    "ts_eik_solve_model": (C.c_int, [_vp, _i32, _i32, _i32, _ip, _ip, _dp, _i32, _d, _i32, _vp, _i32, _P(EikStats)]),
    "ts_eik_solve_noalloc": (C.c_int, [_gp, _vp, _i32, _ip, _dp, _vp, _d, _i32, _vp, _ip]),
    "ts_cuda_selftest": (C.c_int, [_vp, _i32, _dp, C.c_char_p, _i32]),
    "ts_rays_trace": (C.c_int, [_vp, _gp, _i32, _fp, _dp, _gp, _i32, _ip, _dp, _d, _P(_vp)]),
    "ts_rays_set_warp_max": (C.c_int, [_vp, _i32]),
    "ts_forward": (C.c_int, [_vp, _gp, _dp, _i32, _gp, _i32, _dp, _i32, _dp, _i32, _ip, _ip, _ip, _i32, _i32, _d,
                             _P(_vp), _P(EikStats)]),
    "ts_rows_info": (C.c_int, [_vp, _ip, _P(C.c_int64)]),
    "ts_rows_copy": (C.c_int, [_vp, _ip, _ip, _fp, _dp, _u8p]),
    "ts_rows_free": (None, [_vp]),
}

_lib = None


def load() -> C.CDLL:
    """The library with every entry point typed; raises if it was not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run tomostar_b200.build.build() (nvcc, sm_100a)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(rc: int, solver=None) -> None:
    """Raises TsError for a non-zero return code, with the context's last error when there is one."""
    if rc != TS_OK:
        raise TsError(rc, solver.last_error if solver is not None else "")


def engine_shapes() -> list[tuple[int, int, int, int]]:
    """The engine's compiled tile shapes: (id, bx, by, bz)."""
    buf = (C.c_int32 * 64)()
    n = load().ts_engine_shapes(buf, 16)
    return [tuple(buf[4 * q:4 * q + 4]) for q in range(min(n, 16))]
