"""Fields on grids of uneven size in one engine launch (ts_eik_solve_multi), its CUDA-graph replay
and the tile-shape autotuner, against the oracle.

The batch is the uneven-grid workload at reduced dimensions: each source on its own grid, half of
them with geometrically growing depth spacing. FP64 fields equal the oracle's Relax (and, in fast
mode, its wake-threshold variant) to the bit on every grid; FP32 fields stay within 2e-5 relative
of the FP64 oracle."""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source

pytestmark = pytest.mark.gpu
F32_REL_TOL = 2e-5


@pytest.fixture(scope="module")
def batch():
    b = syn.uneven_grids(n_sources=10, seed=3, dims_scale=0.22)
    seeds = [point_source(g, s, *src) for g, s, src in zip(b.grids, b.slowness, b.sources)]
    return b, seeds


def oracle_field(g, s, seed, wake_rel=None):
    og = O.Grid.of(g)
    if wake_rel is None:
        return O.relax(og, s, seed[0], seed[1])[0]
    return O.relax_wake(og, s, seed[0], seed[1], wake_rel, causal=True)[0]


def test_batch_has_variable_and_uneven_grids(batch):
    b, _ = batch
    assert any(g.depth_km is not None for g in b.grids) and any(g.depth_km is None for g in b.grids)
    assert len({(g.nx, g.ny, g.nz) for g in b.grids}) == len(b.grids)


@pytest.mark.parametrize("mode", [L.MODE_ENGINE, L.MODE_FAST])
def test_multi_grid_fp64_bitwise(solver, batch, mode):
    b, seeds = batch
    fields = solver.solve_multi(b.grids, b.slowness, list(range(len(b.grids))), seeds, mode=mode, precision=64)
    wake = None if mode == L.MODE_ENGINE else L.WAKE_REL
    for q, (g, s) in enumerate(zip(b.grids, b.slowness)):
        ref = oracle_field(g, s, seeds[q], wake)
        assert np.array_equal(fields[q], ref), f"grid {q} {g.nx}x{g.ny}x{g.nz} variable={g.depth_km is not None}"


def test_multi_grid_fp64_bitwise_all_tile_shapes(solver, batch):
    """Every compiled tile shape (cube tiles and pencils) on uneven and variable grids."""
    b, seeds = batch
    n = 6
    refs = [oracle_field(g, s, seeds[q]) for q, (g, s) in enumerate(zip(b.grids[:n], b.slowness[:n]))]
    lib = L.load()
    try:
        for sid, bx, by, bz in L.engine_shapes():
            L.check(lib.ts_engine_set_tile(solver.handle, 64, sid), solver)
            fields = solver.solve_multi(b.grids[:n], b.slowness[:n], list(range(n)), seeds[:n], precision=64)
            for q in range(n):
                assert np.array_equal(fields[q], refs[q]), f"tile {bx}x{by}x{bz}, grid {q}"
    finally:
        lib.ts_engine_set_tile(solver.handle, 64, 0)


@pytest.mark.parametrize("mode", [L.MODE_ENGINE, L.MODE_FAST])
def test_multi_grid_flow_scheduler(solver, batch, mode):
    """Uneven and variable grids under the flow scheduler: each field advances on its own."""
    b, seeds = batch
    lib = L.load()
    try:
        L.check(lib.ts_engine_set_scheduler(solver.handle, 1), solver)
        fields = solver.solve_multi(b.grids, b.slowness, list(range(len(b.grids))), seeds, mode=mode, precision=64)
    finally:
        lib.ts_engine_set_scheduler(solver.handle, 0)
    wake = None if mode == L.MODE_ENGINE else L.WAKE_REL
    for q, (g, s) in enumerate(zip(b.grids, b.slowness)):
        assert np.array_equal(fields[q], oracle_field(g, s, seeds[q], wake)), f"grid {q}"


def test_multi_grid_shared_grids_and_float32_tables(solver, batch):
    """Several fields per grid (field_grid repeats grids), in mixed order; float32 output is the
    float32 rounding of the FP64 field."""
    b, seeds = batch
    grids, slow = b.grids[:3], b.slowness[:3]
    fg = [2, 0, 1, 0, 2]
    rng = np.random.default_rng(7)
    sets = []
    for q in fg:
        g = grids[q]
        lon = g.min_lon + rng.uniform(0.2, 0.8) * (g.max_lon - g.min_lon)
        lat = g.min_lat + rng.uniform(0.2, 0.8) * (g.max_lat - g.min_lat)
        sets.append(point_source(g, slow[q], lon, lat, rng.uniform(0, 0.5) * g.max_depth_km))
    f64 = solver.solve_multi(grids, slow, fg, sets, precision=64)
    f32 = solver.solve_multi(grids, slow, fg, sets, out_dtype=np.float32, precision=64)
    for f, q in enumerate(fg):
        assert np.array_equal(f64[f], oracle_field(grids[q], slow[q], sets[f]))
        assert np.array_equal(f32[f], f64[f].astype(np.float32))


def test_multi_grid_fp32_within_tolerance(solver, batch):
    b, seeds = batch
    fields = solver.solve_multi(b.grids, b.slowness, list(range(len(b.grids))), seeds, precision=32)
    worst = 0.0
    for q, (g, s) in enumerate(zip(b.grids, b.slowness)):
        ref = oracle_field(g, s, seeds[q])
        fin = np.isfinite(ref)
        assert np.array_equal(fin, np.isfinite(fields[q]))
        worst = max(worst, float(np.max(np.abs(fields[q][fin] - ref[fin]) / np.maximum(ref[fin], 1e-9))))
    # FP32 arithmetic (paired floats): within 2e-5 at every node, variable depth spacing included.
    assert worst <= F32_REL_TOL, worst


def test_graph_replay_repeats_the_job(solver, batch):
    b, seeds = batch
    n = 4
    args = (b.grids[:n], b.slowness[:n], list(range(n)), seeds[:n])
    solver.set_graph(True)
    try:
        before = solver.graph_replays
        first = solver.solve_multi(*args, mode=L.MODE_FAST, precision=64)
        second = solver.solve_multi(*args, mode=L.MODE_FAST, precision=64)
        assert solver.graph_replays == before + 1
        for a, c in zip(first, second):
            assert np.array_equal(a, c)
        # A different job is captured anew (no replay) and is still exact.
        third = solver.solve_multi(b.grids[1:n + 1], b.slowness[1:n + 1], list(range(n)), seeds[1:n + 1],
                                   mode=L.MODE_FAST, precision=64)
        assert solver.graph_replays == before + 1
        for q in range(n):
            g, s = b.grids[q + 1], b.slowness[q + 1]
            assert np.array_equal(third[q], oracle_field(g, s, seeds[q + 1], L.WAKE_REL))
    finally:
        solver.set_graph(False)


def test_autotune_selects_a_compiled_shape(solver, batch):
    b, seeds = batch
    n = 3
    best, sched, ms = solver.autotune(b.grids[:n], b.slowness[:n], list(range(n)), seeds[:n], precision=64)
    assert (best, sched) in ms and all(np.isfinite(v) and v > 0 for v in ms.values())
    assert ms[(best, sched)] == min(ms.values())
    # The selection stays on the context and gives the same fields; restore the defaults afterwards.
    lib = L.load()
    try:
        fields = solver.solve_multi(b.grids[:n], b.slowness[:n], list(range(n)), seeds[:n], mode=L.MODE_FAST,
                                    precision=64)
        for q in range(n):
            assert np.array_equal(fields[q], oracle_field(b.grids[q], b.slowness[q], seeds[q], L.WAKE_REL))
    finally:
        L.check(lib.ts_engine_set_tile(solver.handle, 64, 0), solver)
        L.check(lib.ts_engine_set_scheduler(solver.handle, 0), solver)
