"""TravelTimeTable.Write / Open (Forward/TravelTimeTable.cs:57-111) as bytes — TEST INFRASTRUCTURE ONLY.

The reference commits no .qttb file, so the layout is restated from the writer and reader themselves:
magic "QTTB" 01 00 00 00, the header length (little-endian int32), the header JSON, zero bytes to a
multiple of 64, then one little-endian float32 per node, non-finite values as +inf ("parity pinned to
the source's layout rules", tests/test_qttb.py).
"""
from __future__ import annotations

import struct

import numpy as np

MAGIC = b"QTTB\x01\x00\x00\x00"


def write_bytes(header: bytes, times) -> bytes:
    """TravelTimeTable.Write (:57-80): times are doubles; each becomes (float)t, or +inf when not finite."""
    t = np.asarray(times, np.float64)
    with np.errstate(over="ignore"):  # (float) of a double beyond float's range is +-inf
        f = np.where(np.isfinite(t), t, np.inf).astype("<f4")
    pad = (64 - (12 + len(header)) % 64) % 64
    return MAGIC + struct.pack("<i", len(header)) + header + b"\0" * pad + f.tobytes()


def open_bytes(data: bytes):
    """TravelTimeTable.Open (:99-111) and Node (:113): (header bytes, float32 nodes)."""
    if data[:8] != MAGIC:
        raise ValueError("Not a travel-time table.")
    n = struct.unpack("<i", data[8:12])[0]
    header = data[12:12 + n]
    offset = 12 + n + (64 - (12 + n) % 64) % 64
    return header, np.frombuffer(data[offset:], "<f4")
