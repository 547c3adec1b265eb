"""ts_eik_solve_noalloc: the solve for callers that cannot allocate device memory.

Such a caller (its device memory held by another allocator or a fixed budget, or a path that cannot
take an allocation's synchronisation) hands in its own device buffers; the entry point works in a
static array the library holds. These tests give it device buffers made here, run it twice in a row
(the second call reuses the array the first one left behind) and check each field against the
regular entry point ts_eik_solve, which equals the reference to the bit, so the check is bitwise.
Collected last on purpose, so that a run stopping at the first failure has run everything else.
"""
import ctypes as C

import numpy as np
import pytest

from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source
from tomostar_b200.grid import GridDef

pytestmark = pytest.mark.gpu

P = C.POINTER


def no_alloc_solve(grid, slowness, seeds, stream=None):
    """The caller's buffers are made here (torch), as a caller would bring its own; `stream` is a torch
    stream the call runs on (its handle passed through the C ABI), None for the default stream."""
    import torch

    lib = L.load()
    s_dev = torch.from_numpy(np.ascontiguousarray(slowness, np.float64)).cuda()
    out = torch.empty(grid.count, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    si = np.ascontiguousarray(seeds[0], np.int32)
    st = np.ascontiguousarray(seeds[1], np.float64)
    gs = grid.struct()
    rounds = np.zeros(2, np.int32)
    handle = C.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = lib.ts_eik_solve_noalloc(C.byref(gs), C.c_void_p(s_dev.data_ptr()), len(si), si.ctypes.data_as(P(C.c_int32)),
                                  st.ctypes.data_as(P(C.c_double)), C.c_void_p(out.data_ptr()), 1e-7, 0, handle,
                                  rounds.ctypes.data_as(P(C.c_int32)))
    assert rc == L.TS_OK, lib.ts_last_error(None).decode()
    if stream is not None:
        stream.synchronize()
    return out.cpu().numpy(), rounds


def regular_solve(solver, grid, slowness, seeds):
    return solver.solve(grid, slowness, [seeds], precision=64, mode=L.MODE_PLAIN)[0]


def test_no_alloc_matches_regular_entry_point_twice(solver):
    """Two calls in a row on different inputs, each equal to ts_eik_solve's field."""
    p = syn.single_source_61()
    a_seeds = point_source(p.grid, p.slowness[0], *p.stations[0])
    a, ra = no_alloc_solve(p.grid, p.slowness[0], a_seeds)
    assert np.array_equal(a, regular_solve(solver, p.grid, p.slowness[0], a_seeds))
    assert ra[0] >= 1 and ra[1] >= 1

    g = GridDef(10.0, 10.25, 42.0, 42.2, -1.0, 14.0, 26, 23, 16)
    rng = np.random.default_rng(31)
    s = 1 / (5 + rng.uniform(-0.4, 0.4, g.count))
    b_seeds = point_source(g, s, 10.1, 42.12, 4.0)
    b, _ = no_alloc_solve(g, s, b_seeds)
    assert np.array_equal(b, regular_solve(solver, g, s, b_seeds))


def test_no_alloc_rejects_grids_beyond_its_limit():
    lib = L.load()
    g = GridDef(10.0, 11.0, 42.0, 43.0, 0.0, 30.0, 401, 401, 121)  # 19.5 M nodes > the limit
    gs = g.struct()
    si = np.zeros(1, np.int32)
    st = np.zeros(1)
    rc = lib.ts_eik_solve_noalloc(C.byref(gs), C.c_void_p(16), 1, si.ctypes.data_as(P(C.c_int32)),
                                  st.ctypes.data_as(P(C.c_double)), C.c_void_p(16), 1e-7, 0, None, None)
    assert rc == L.TS_E_CAPACITY
    assert "limits" in lib.ts_last_error(None).decode()


def test_no_alloc_merges_seeds_on_a_side_stream(solver):
    """Duplicate seeds (the smallest time kept) and seeds off the grid (dropped), as TrySolve merges
    them, on a caller's non-default stream: bitwise against ts_eik_solve on the same seed list."""
    import torch

    g = GridDef(10.0, 10.2, 42.0, 42.18, -1.0, 11.0, 21, 19, 13)
    rng = np.random.default_rng(44)
    s = 1 / (5.2 + rng.uniform(-0.3, 0.3, g.count))
    si, st = point_source(g, s, 10.07, 42.1, 3.0)
    si = np.concatenate([si, si[:3], [g.count, g.count + 7, -1]]).astype(np.int32)
    st = np.concatenate([st, st[:3] - 0.002, [0.0, 0.0, 0.0]])
    side = torch.cuda.Stream()
    got, _ = no_alloc_solve(g, s, (si, st), stream=side)
    want = solver.solve(g, s, [(si, st)], precision=64, mode=L.MODE_PLAIN)[0]
    assert np.array_equal(got, want)


def test_no_alloc_refuses_host_buffers():
    """Buffers that are not device memory of the current device are refused before any launch."""
    import torch

    torch.cuda.init()
    lib = L.load()
    g = GridDef(10.0, 10.1, 42.0, 42.1, 0.0, 5.0, 9, 9, 6)
    host_s = np.full(g.count, 0.2)
    host_out = np.empty(g.count)
    si = np.array([40], np.int32)
    st = np.zeros(1)
    gs = g.struct()
    rc = lib.ts_eik_solve_noalloc(C.byref(gs), host_s.ctypes.data_as(C.c_void_p), 1, si.ctypes.data_as(P(C.c_int32)),
                                  st.ctypes.data_as(P(C.c_double)), host_out.ctypes.data_as(C.c_void_p), 1e-7, 0,
                                  None, None)
    assert rc == L.TS_E_ARG
    assert "device memory" in lib.ts_last_error(None).decode()
