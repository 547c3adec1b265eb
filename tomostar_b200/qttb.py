""".qttb travel-time table files (Forward/TravelTimeTable.cs:14-111) from and to tables on the device.

`write` lays out TravelTimeTable.Write's file around device tables; `load` reads files that
TravelTimeTable.Open accepts into a resident table set. The header bytes are the caller's: a C# host
passes `JsonSerializer.SerializeToUtf8Bytes(header, TomoJson.Options)`. For Python callers
`header_json` writes the same document by System.Text.Json's documented rules for these options
(two-space indentation, declaration order, enums as names, shortest round-trip numbers in .NET's
layout, the default encoder's escapes), and `model_key` is ForwardModel.Key (:176-183).
"""
from __future__ import annotations

import ctypes as C
import hashlib
import math
from decimal import Decimal

import numpy as np

from . import _lib as L
from .grid import GridDef
from .location import Tables

MAGIC = b"QTTB\x01\x00\x00\x00"


def data_offset(json_len: int) -> int:
    """Where the float32 data start (TravelTimeTable.cs:108)."""
    return 12 + json_len + (64 - (12 + json_len) % 64) % 64


def net_number(x: float) -> str:
    """A double as System.Text.Json writes it: shortest round-trip digits; fixed notation when the
    decimal exponent lies in (-5, 15), otherwise d.dddE+XX; named literals for NaN and infinities."""
    if isinstance(x, (int, np.integer)) and not isinstance(x, bool):
        return str(int(x))
    x = float(x)
    if math.isnan(x):
        return '"NaN"'
    if math.isinf(x):
        return '"Infinity"' if x > 0 else '"-Infinity"'
    if x == 0:
        return "-0" if math.copysign(1.0, x) < 0 else "0"
    # Shortest round-trip digits (repr) and the decimal exponent of the first digit.
    t = Decimal(repr(abs(x))).normalize().as_tuple()
    digits = "".join(map(str, t.digits))
    e10 = len(digits) + t.exponent - 1
    sign = "-" if x < 0 else ""
    if -5 < e10 < 15:
        if e10 >= 0:
            whole = digits[: e10 + 1].ljust(e10 + 1, "0")
            frac = digits[e10 + 1:]
            return sign + whole + ("." + frac if frac else "")
        return sign + "0." + "0" * (-e10 - 1) + digits
    m = digits[0] + ("." + digits[1:] if len(digits) > 1 else "")
    return f"{sign}{m}E{'+' if e10 >= 0 else '-'}{abs(e10):02d}"


def _net_string(s: str) -> str:
    out = []
    for ch in s:
        o = ord(ch)
        if ch == "\\":
            out.append("\\\\")
        elif ch in "\n\r\t\b\f":
            out.append({"\n": "\\n", "\r": "\\r", "\t": "\\t", "\b": "\\b", "\f": "\\f"}[ch])
        elif o < 0x20 or o > 0x7e or ch in "\"&'+<>`":
            out.append(f"\\u{o:04X}")
        else:
            out.append(ch)
    return '"' + "".join(out) + '"'


def _grid_fields(g: GridDef):
    return [("MinLon", g.min_lon), ("MaxLon", g.max_lon), ("MinLat", g.min_lat), ("MaxLat", g.max_lat),
            ("MinDepthKm", g.min_depth_km), ("MaxDepthKm", g.max_depth_km), ("Nx", int(g.nx)), ("Ny", int(g.ny)),
            ("Nz", int(g.nz))]


def _object(fields, indent: int) -> str:
    pad, inner = "  " * indent, "  " * (indent + 1)
    lines = [f'{inner}"{k}": {v}' for k, v in fields]
    return "{\n" + ",\n".join(lines) + "\n" + pad + "}"


def grid_json(g: GridDef) -> bytes:
    """GridDefinition serialised with TomoJson.Options (the bytes ForwardModel.Key hashes)."""
    return _object([(k, net_number(v)) for k, v in _grid_fields(g)], 0).encode()


def header_json(station_id: str, phase: str, lon: float, lat: float, depth_km: float, grid: GridDef,
                model_key: str = "", solver: str = "") -> bytes:
    """TravelTimeTableHeader (TravelTimeTable.cs:14-27) serialised with TomoJson.Options."""
    g = _object([(k, net_number(v)) for k, v in _grid_fields(grid)], 1)
    fields = [("StationId", _net_string(station_id)), ("Phase", _net_string(phase)), ("Lon", net_number(lon)),
              ("Lat", net_number(lat)), ("DepthKm", net_number(depth_km)), ("Grid", g),
              ("ModelKey", _net_string(model_key)), ("Solver", _net_string(solver))]
    return _object(fields, 0).encode()


def model_key(grid: GridDef, slowness: np.ndarray) -> str:
    """ForwardModel.Key: the first 32 hex digits (upper case) of SHA-256 over the slowness as
    little-endian doubles followed by the grid definition's JSON."""
    s = np.ascontiguousarray(slowness, "<f8")
    return hashlib.sha256(s.tobytes() + grid_json(grid)).hexdigest().upper()[:32]


def write(tables: Tables, paths, headers, first: int = 0) -> None:
    """TravelTimeTable.Write of tables first .. first+len(paths)-1 to paths, with their header bytes."""
    n = len(paths)
    if len(headers) != n:
        raise ValueError("one header per path")
    cp = (C.c_char_p * n)(*[str(p).encode() for p in paths])
    hs = [bytes(h) for h in headers]
    ch = (C.c_char_p * n)(*hs)
    hl = (C.c_int32 * n)(*[len(h) for h in hs])
    rc = L.load().ts_tables_write_qttb(tables.handle, first, n, cp, ch, hl)
    if rc != L.TS_OK:
        raise L.TsError(rc, tables.solver.last_error)


def load(solver, grid: GridDef, paths) -> Tables:
    """TravelTimeTable.Open of every path into one resident table set on grid."""
    n = len(paths)
    cp = (C.c_char_p * n)(*[str(p).encode() for p in paths])
    h = C.c_void_p()
    gs = grid.struct()
    rc = L.load().ts_tables_load_qttb(solver.handle, C.byref(gs), n, cp, C.byref(h))
    if rc != L.TS_OK:
        raise L.TsError(rc, solver.last_error)
    return Tables(solver, h, grid)
