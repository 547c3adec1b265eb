"""Eikonal parity on the GPU: the engine and the plain path against the oracle (SphericalEikonal.Relax).

FP64 must equal the oracle to the bit (the engine's tile wavefront is a reordering the Gauss-Seidel
sweep is invariant to); FP32 must be within 2e-5 relative of the FP64 oracle."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import EikonalCuda, point_source
from tomostar_b200.grid import GridDef

pytestmark = pytest.mark.gpu
F32_REL_TOL = 2e-5


def rel_err(a, ref):
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(a)), "reached sets differ"
    return float(np.max(np.abs(a[fin] - ref[fin]) / np.maximum(ref[fin], 1e-9)))


def oracle_fields(g, s, seeds, tol=1e-7):
    og = O.Grid.of(g)
    return np.stack([O.relax(og, s, si, st, tol=tol)[0] for si, st in seeds])


def hetero_case(nx, ny, nz, seed, nsrc=3):
    g = GridDef(10.0, 10.0 + 0.011 * (nx - 1), 42.0, 42.0 + 0.009 * (ny - 1), -1.0, -1.0 + 0.9 * (nz - 1), nx, ny, nz)
    rng = np.random.default_rng(seed)
    dep = g.depth()
    v = (5 + 0.04 * dep)[:, None, None] * (1 + 0.08 * rng.standard_normal((nz, ny, nx)).clip(-2, 2))
    s = (1 / v).reshape(-1)
    lon, lat = g.lon(), g.lat()
    srcs = [(rng.uniform(lon[0], lon[-1]), rng.uniform(lat[0], lat[-1]), rng.uniform(dep[0], dep[-1]))
            for _ in range(nsrc)]
    return g, s, [point_source(g, s, *x) for x in srcs]


def test_selftest_gate(solver):
    """EikonalOpenCl.SelfTest: FP64 agrees exactly; FP32 within the gate (1e-6 of range)."""
    solver.precision = 64
    rel, msg = solver.self_test()
    assert rel == 0.0, msg
    solver.precision = 32
    rel32, msg32 = solver.self_test()
    solver.precision = 64
    assert rel32 <= 1e-6, msg32


def test_try_create_passes_gate():
    s = EikonalCuda.try_create(precision=64)
    assert s is not None and "B200" in s.device or s is not None
    s.close()


@pytest.mark.parametrize("mode", [L.MODE_ENGINE, L.MODE_PLAIN])
def test_f64_bitwise_single_source_61(solver, mode):
    p = syn.single_source_61()
    seeds = [point_source(p.grid, p.slowness[0], *p.stations[0])]
    ref = oracle_fields(p.grid, p.slowness[0], seeds)
    out = solver.solve(p.grid, p.slowness[0], seeds, mode=mode, precision=64)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("shape", [(23, 19, 13), (9, 40, 7), (33, 17, 21), (2, 2, 2), (64, 3, 9)])
def test_f64_engine_bitwise_ragged_grids(solver, shape):
    """Grids that are not multiples of the tile, thin grids and the smallest grid."""
    g, s, seeds = hetero_case(*shape, seed=sum(shape))
    ref = oracle_fields(g, s, seeds)
    out = solver.solve(g, s, seeds, precision=64)
    assert np.array_equal(out, ref)


def test_f64_engine_bitwise_all_tile_shapes(solver):
    g, s, seeds = hetero_case(37, 29, 19, seed=11, nsrc=4)
    ref = oracle_fields(g, s, seeds)
    lib = L.load()
    buf = (C.c_int32 * 64)()
    n = lib.ts_engine_shapes(buf, 16)
    try:
        for q in range(n):
            assert lib.ts_engine_set_tile(solver.handle, 64, buf[4 * q]) == 0
            out = solver.solve(g, s, seeds, precision=64)
            assert np.array_equal(out, ref), f"shape {buf[4*q+1]}x{buf[4*q+2]}x{buf[4*q+3]}"
    finally:
        lib.ts_engine_set_tile(solver.handle, 64, 0)


def test_f64_exact_fixed_point(solver):
    """tol = 0 (the exact fixed point) also matches bitwise."""
    g, s, seeds = hetero_case(25, 21, 15, seed=5, nsrc=2)
    ref = oracle_fields(g, s, seeds, tol=0.0)
    out = solver.solve(g, s, seeds, precision=64, tol=0.0)
    assert np.array_equal(out, ref)


def test_f64_batch_equals_solo(solver):
    """A field is the same alone and in a batch (determinism)."""
    g, s, seeds = hetero_case(30, 26, 14, seed=9, nsrc=6)
    batch = solver.solve(g, s, seeds, precision=64)
    for f in (0, 3, 5):
        solo = solver.solve(g, s, [seeds[f]], precision=64)
        assert np.array_equal(solo[0], batch[f])


def test_f32_engine_equals_plain_and_oracle(solver):
    p = syn.single_source_61()
    seeds = [point_source(p.grid, p.slowness[0], *p.stations[0])]
    ref = oracle_fields(p.grid, p.slowness[0], seeds)
    a = solver.solve(p.grid, p.slowness[0], seeds, precision=32)
    b = solver.solve(p.grid, p.slowness[0], seeds, precision=32, mode=L.MODE_PLAIN)
    assert np.array_equal(a, b)
    assert rel_err(a[0], ref[0]) <= F32_REL_TOL


def test_f32_engine_all_tile_shapes_equal_plain(solver):
    """FP32 arithmetic is the same in every kernel, so each tile shape equals the plain path bitwise."""
    g, s, seeds = hetero_case(37, 29, 19, seed=13, nsrc=3)
    plain = solver.solve(g, s, seeds, precision=32, mode=L.MODE_PLAIN)
    lib = L.load()
    try:
        for sid, bx, by, bz in L.engine_shapes():
            assert lib.ts_engine_set_tile(solver.handle, 32, sid) == 0
            out = solver.solve(g, s, seeds, precision=32)
            assert np.array_equal(out, plain), f"shape {bx}x{by}x{bz}"
    finally:
        lib.ts_engine_set_tile(solver.handle, 32, 0)


def test_f64_tables_inversion_step_121_subset(solver):
    """121×121×61 at 0.5 km: P and S tables of three stations from the FP64 engine, written as
    float32 (.qttb), equal the oracle's tables to the bit — the headline error is float rounding alone."""
    p = syn.inversion_step_121()
    for ph in (0, 1):
        seeds = [point_source(p.grid, p.slowness[ph], *p.stations[q]) for q in (0, 7, 19)]
        ref = oracle_fields(p.grid, p.slowness[ph], seeds)
        out = solver.solve(p.grid, p.slowness[ph], seeds, precision=64, output=np.empty((3, p.grid.count), np.float32))
        for f in range(3):
            assert np.array_equal(out[f], O.to_table(ref[f]))
            assert rel_err(out[f].astype(np.float64), ref[f]) <= 6e-8


def test_f32_compute_error_profile_inversion_step_121(solver):
    """FP32 arithmetic (the reference's paired-float scheme: times as hi + lo floats, the update in
    float offsets from the smallest upwind neighbour): within 2e-5 relative of the FP64 oracle at
    every node, p99 near the float32 table rounding."""
    p = syn.inversion_step_121()
    for ph in (0, 1):
        seeds = [point_source(p.grid, p.slowness[ph], *p.stations[q]) for q in (0, 7, 19)]
        ref = oracle_fields(p.grid, p.slowness[ph], seeds)
        out = solver.solve(p.grid, p.slowness[ph], seeds, precision=32)
        for f in range(3):
            fin = np.isfinite(ref[f])
            rel = np.abs(out[f][fin] - ref[f][fin]) / np.maximum(ref[f][fin], 1e-9)
            assert np.percentile(rel, 99) <= 2e-7, (ph, f)
            assert rel.max() <= F32_REL_TOL, (ph, f, rel.max())


def test_f32_output_float32(solver):
    g, s, seeds = hetero_case(20, 20, 10, seed=2, nsrc=2)
    o64 = solver.solve(g, s, seeds, precision=32)
    o32 = solver.solve(g, s, seeds, precision=32, output=np.empty((2, g.count), np.float32))
    assert np.array_equal(o64.astype(np.float32), o32)


def test_f64_to_float32_table_output(solver):
    """An FP64 solve written as float32 is the .qttb rounding of the FP64 field (TravelTimeTable.cs:73)."""
    g, s, seeds = hetero_case(20, 18, 10, seed=4, nsrc=1)
    o64 = solver.solve(g, s, seeds, precision=64)
    o32 = solver.solve(g, s, seeds, precision=64, output=np.empty((1, g.count), np.float32))
    assert np.array_equal(O.to_table(o64[0]), o32[0])


def test_unsettled_is_refused(solver):
    """EikonalOpenCl.cs:269: a batch not settled within the cap is refused, not returned."""
    g, s, seeds = hetero_case(30, 30, 15, seed=1, nsrc=1)
    for mode in (L.MODE_ENGINE, L.MODE_PLAIN):
        ok, reason = solver.try_solve(g, s, seeds, np.empty((1, g.count)), max_rounds=1, mode=mode)
        assert not ok and "not settled" in reason


def test_no_seeds_is_refused(solver):
    g, s, _ = hetero_case(10, 10, 10, seed=1, nsrc=1)
    ok, reason = solver.try_solve(g, s, [(np.array([-5, 10 ** 6], np.int32), np.array([0.0, 1.0]))],
                                  np.empty((1, g.count)))
    assert not ok and "no seed nodes" in reason


def test_out_of_range_and_duplicate_seeds(solver):
    """TrySolve drops out-of-range seeds and keeps the smallest time of duplicates (EikonalOpenCl.cs:150-157)."""
    g, s, seeds = hetero_case(16, 14, 10, seed=8, nsrc=1)
    si, st = seeds[0]
    noisy = (np.concatenate([si, [-1, g.count, si[0]]]).astype(np.int32), np.concatenate([st, [0.0, 0.0, st[0] + 5]]))
    a = solver.solve(g, s, [noisy], precision=64)
    b = solver.solve(g, s, seeds, precision=64)
    assert np.array_equal(a, b)


def test_invalid_grid_is_an_error(solver):
    g = GridDef(10, 9, 42, 43, 0, 10, 5, 5, 5)
    ok, reason = solver.try_solve(g, np.ones(125), [(np.array([0], np.int32), np.array([0.0]))], np.empty((1, 125)))
    assert not ok and "inverted" in reason


def test_cancel(solver):
    g, s, seeds = hetero_case(20, 20, 10, seed=3, nsrc=1)
    solver.cancel(True)
    try:
        ok, reason = solver.try_solve(g, s, seeds, np.empty((1, g.count)))
        assert not ok and "cancel" in reason
        ok2, _ = solver.try_solve(g, s, seeds, np.empty((1, g.count)), mode=L.MODE_PLAIN)
        assert not ok2
    finally:
        solver.cancel(False)
    ok, _ = solver.try_solve(g, s, seeds, np.empty((1, g.count)))
    assert ok


def test_variable_vertical_spacing_f64_bitwise(solver):
    """Extension: geometric vertical spacing, engine and plain path against the extended oracle."""
    nz = 17
    dep = np.cumsum(np.concatenate([[0.0], 0.4 * 1.04 ** np.arange(nz - 1)])) - 1.0
    g = GridDef(10, 10.3, 42, 42.25, float(dep[0]), float(dep[-1]), 27, 25, nz, depth_km=dep)
    rng = np.random.default_rng(21)
    s = (1 / ((5 + 0.05 * dep)[:, None, None] * (1 + 0.05 * rng.standard_normal((nz, 25, 27))))).reshape(-1)
    seeds = [point_source(g, s, 10.12, 42.1, 2.0), point_source(g, s, 10.25, 42.2, 0.0)]
    og = O.Grid.of(g)
    for a, b in zip(seeds, [O.point_source(og, s, 10.12, 42.1, 2.0), O.point_source(og, s, 10.25, 42.2, 0.0)]):
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    ref = oracle_fields(g, s, seeds)
    for mode in (L.MODE_ENGINE, L.MODE_PLAIN):
        out = solver.solve(g, s, seeds, precision=64, mode=mode)
        assert np.array_equal(out, ref), mode
    out32 = solver.solve(g, s, seeds, precision=32)
    for f in range(2):
        assert rel_err(out32[f], ref[f]) <= F32_REL_TOL


def test_suggest_batch(solver):
    n = 401 * 401 * 121
    b32 = solver.suggest_batch(n)
    assert 100 < b32 <= 1024


WAKE = 1e-13


@pytest.mark.parametrize("shape", [(23, 19, 13), (33, 17, 21), (40, 40, 20)])
def test_fast_mode_equals_wake_oracle(solver, shape):
    """TS_MODE_FAST is the reference scheme with the wake threshold and the causal wake rule: equal
    to the oracle's relax_wake to the bit, and within 1e-10 relative of the reference (Relax)."""
    g, s, seeds = hetero_case(*shape, seed=3 * sum(shape))
    og = O.Grid.of(g)
    out = solver.solve(g, s, seeds, precision=64, mode=L.MODE_FAST)
    for f, (si, st) in enumerate(seeds):
        w, ok, _, _ = O.relax_wake(og, s, si, st, WAKE, causal=True)
        ref = O.relax(og, s, si, st)[0]
        assert ok and np.array_equal(out[f], w)
        assert rel_err(out[f], ref) <= 1e-10


def test_fast_mode_inversion_step_121_within_1e10(solver):
    p = syn.inversion_step_121()
    for ph in (0, 1):
        seeds = [point_source(p.grid, p.slowness[ph], *p.stations[q]) for q in (2, 13)]
        ref = oracle_fields(p.grid, p.slowness[ph], seeds)
        out = solver.solve(p.grid, p.slowness[ph], seeds, precision=64, mode=L.MODE_FAST)
        for f in range(2):
            assert rel_err(out[f], ref[f]) <= 1e-10


def test_fast_mode_all_tile_shapes(solver):
    g, s, seeds = hetero_case(37, 29, 19, seed=12, nsrc=3)
    lib = L.load()
    buf = (C.c_int32 * 64)()
    n = lib.ts_engine_shapes(buf, 16)
    og = O.Grid.of(g)
    want = np.stack([O.relax_wake(og, s, si, st, WAKE, causal=True)[0] for si, st in seeds])
    try:
        for q in range(n):
            assert lib.ts_engine_set_tile(solver.handle, 64, buf[4 * q]) == 0
            out = solver.solve(g, s, seeds, precision=64, mode=L.MODE_FAST)
            assert np.array_equal(out, want)
    finally:
        lib.ts_engine_set_tile(solver.handle, 64, 0)


def test_fast_mode_full_size_field_within_1e10(solver):
    """One field of the 401×401×121 forward step: fast mode against the bitwise engine (which equals
    the reference's Relax to the bit) within 1e-10 relative; float32 tables within 2e-5 (their
    rounding)."""
    p = syn.regional_401(n_stations=2, n_events=10, n_rays=10)
    seeds = [point_source(p.grid, p.slowness[1], *p.stations[0])]
    exact = solver.solve(p.grid, p.slowness[1], seeds, precision=64, mode=L.MODE_ENGINE)
    fast = solver.solve(p.grid, p.slowness[1], seeds, precision=64, mode=L.MODE_FAST)
    assert rel_err(fast[0], exact[0]) <= 1e-10
    t32 = solver.solve(p.grid, p.slowness[1], seeds, mode=L.MODE_FAST,
                       output=np.empty((1, p.grid.count), np.float32), precision=64)
    assert rel_err(t32[0].astype(np.float64), exact[0]) <= 2e-5


@pytest.mark.parametrize("mode", [L.MODE_ENGINE, L.MODE_FAST])
def test_flow_scheduler_all_tile_shapes(solver, mode):
    """The flow scheduler (fields advance on their own through a shared tile queue, no grid-wide
    barrier) gives the same fields as the lockstep one: bitwise vs Relax (exact mode) or vs the
    oracle's fast-mode rule, for every tile shape, several fields of one grid at once."""
    g, s, seeds = hetero_case(37, 29, 19, seed=14, nsrc=4)
    og = O.Grid.of(g)
    if mode == L.MODE_ENGINE:
        want = np.stack([O.relax(og, s, si, st)[0] for si, st in seeds])
    else:
        want = np.stack([O.relax_wake(og, s, si, st, WAKE, causal=True)[0] for si, st in seeds])
    lib = L.load()
    try:
        assert lib.ts_engine_set_scheduler(solver.handle, 1) == 0
        for sid, bx, by, bz in L.engine_shapes():
            assert lib.ts_engine_set_tile(solver.handle, 64, sid) == 0
            out = solver.solve(g, s, seeds, precision=64, mode=mode)
            assert np.array_equal(out, want), f"shape {bx}x{by}x{bz}"
    finally:
        lib.ts_engine_set_scheduler(solver.handle, 0)
        lib.ts_engine_set_tile(solver.handle, 64, 0)


def test_flow_scheduler_inversion_step_121_batch(solver):
    """A batch of config-1 fields (P and S) under the flow scheduler equals the lockstep one."""
    p = syn.inversion_step_121()
    seeds = [point_source(p.grid, p.slowness[0], *p.stations[q]) for q in range(6)]
    lib = L.load()
    a = solver.solve(p.grid, p.slowness[0], seeds, precision=64, mode=L.MODE_FAST)
    try:
        assert lib.ts_engine_set_scheduler(solver.handle, 1) == 0
        b = solver.solve(p.grid, p.slowness[0], seeds, precision=64, mode=L.MODE_FAST)
    finally:
        lib.ts_engine_set_scheduler(solver.handle, 0)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("precision", [64, 32])
@pytest.mark.parametrize("dtype", [np.float64, np.float32])
def test_many_fields_to_page_locked_memory_equal_pageable(solver, precision, dtype):
    """With 64 fields or more and a page-locked output the solve copies the first half of the fields
    to the host while the second half is solved; the result is the same as through pageable memory."""
    import torch

    g, s, _ = hetero_case(21, 19, 11, seed=8, nsrc=1)
    rng = np.random.default_rng(8)
    lon, lat, dep = g.lon(), g.lat(), g.depth()
    seeds = [point_source(g, s, rng.uniform(lon[0], lon[-1]), rng.uniform(lat[0], lat[-1]),
                          rng.uniform(dep[0], dep[-1])) for _ in range(70)]
    pageable = solver.solve(g, s, seeds, precision=precision, mode=L.MODE_FAST,
                            output=np.empty((70, g.count), dtype))
    tdt = torch.float64 if dtype == np.float64 else torch.float32
    locked = torch.empty((70, g.count), dtype=tdt, pin_memory=True).numpy()
    solver.solve(g, s, seeds, precision=precision, mode=L.MODE_FAST, output=locked)
    assert np.array_equal(locked, pageable)
