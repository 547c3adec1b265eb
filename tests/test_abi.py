"""The C-ABI library: it loads, exports every entry point include/*.h declares, and its host-side
code (seeds, grid checks) matches the oracle. No GPU compute here."""
import ctypes as C
import glob
import os
import re

import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import pack_seeds, point_source
from tomostar_b200.grid import GridDef

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        names |= set(re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(ts_[a-z_0-9]+)\s*\(", text, re.M))
    return names


def test_header_declares_the_abi():
    names = declared_symbols()
    for required in ("ts_cuda_create", "ts_eik_solve", "ts_cuda_selftest", "ts_rays_trace", "ts_forward",
                     "ts_rows_copy", "ts_point_source", "ts_eik_suggest_batch"):
        assert required in names


def test_library_exports_every_declared_symbol():
    lib = C.CDLL(L.LIB_PATH)
    missing = [n for n in sorted(declared_symbols()) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(L.SIGNATURES) >= declared_symbols()
    L.load()  # every signature binds


def test_no_device_is_an_error_not_a_crash():
    lib = L.load()
    h = C.c_void_p()
    rc = lib.ts_cuda_create(0, C.byref(h))
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        pytest.skip("a GPU is present")
    assert rc == L.TS_E_NODEVICE and not h.value


def test_engine_shapes():
    lib = L.load()
    buf = (C.c_int32 * 64)()
    n = lib.ts_engine_shapes(buf, 16)
    assert n >= 1
    shapes = [tuple(buf[4 * q: 4 * q + 4]) for q in range(n)]
    for sid, bx, by, bz in shapes:
        assert bx * by * bz % 32 == 0 and max(by, bz) <= 32 and bx <= 64


@pytest.mark.parametrize("src", [(10.37, 42.61, 8.3), (10.0, 42.0, -5.0), (12.0, 44.0, 200.0), (11.13, 43.5, 0.0)])
def test_point_source_matches_oracle_bitwise(src):
    """ts_point_source (product host code) equals the oracle's PointSource to the bit."""
    g, s, _ = syn.selftest_case()
    a_idx, a_t = point_source(g, s, *src)
    b_idx, b_t = O.point_source(O.Grid.of(g), s, *src)
    assert np.array_equal(a_idx, b_idx) and np.array_equal(a_t, b_t)


def test_point_source_single_source_61_matches_oracle():
    p = syn.single_source_61()
    a = point_source(p.grid, p.slowness[0], *p.stations[0])
    b = O.point_source(O.Grid.of(p.grid), p.slowness[0], *p.stations[0])
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    assert len(a[0]) > 50


def test_point_source_rejects_bad_grid():
    lib = L.load()
    g = GridDef(10, 9, 42, 43, 0, 10, 5, 5, 5).struct()  # inverted longitudes
    s = np.ones(125)
    n = lib.ts_point_source(C.byref(g), s.ctypes.data_as(C.POINTER(C.c_double)), 10.5, 42.5, 1, 0, 3,
                            None, None, 0)
    assert n == -1


def test_pack_seeds():
    off, idx, t = pack_seeds([(np.array([1, 2]), np.array([0.1, 0.2])), (np.array([5]), np.array([0.5]))])
    assert off.tolist() == [0, 2, 3] and idx.tolist() == [1, 2, 5] and t.tolist() == [0.1, 0.2, 0.5]
