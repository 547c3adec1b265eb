"""Parity at the named workloads' full sizes (slow: the oracle runs on the host cores).

* The 401x401x121 regional model: one P field of the FP64 engine against the oracle's Relax
  (to the bit), and the fast mode within 1e-10 relative of it.
* Three of the 200 uneven grids at full size (the largest horizontal grid, the largest depth, one
  with geometric depth spacing) in one ts_eik_solve_multi launch against the oracle (to the bit).
* 2,000 rays of the regional forward step (arrivals drawn with seed 5 among the events of two
  stations, P and S) traced on device tables and by the oracle on the same tables, under the
  ray bar of tests/test_rays_gpu.py.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import location as loc
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source
from tomostar_b200.rays import step_km, trace_rows

from test_rays_gpu import compare_rows

pytestmark = pytest.mark.gpu


def test_regional_401_field_equals_oracle(solver):
    p = syn.regional_401(n_stations=3, n_events=10, n_rays=10)
    seeds = point_source(p.grid, p.slowness[0], *p.stations[2])
    want, ok, _ = O.relax(O.Grid.of(p.grid), p.slowness[0], *seeds)
    assert ok
    got = solver.solve(p.grid, p.slowness[0], [seeds], precision=64, mode=L.MODE_ENGINE)[0]
    assert np.array_equal(got, want)
    fast = solver.solve(p.grid, p.slowness[0], [seeds], precision=64, mode=L.MODE_FAST)[0]
    fin = np.isfinite(want) & (want > 0)
    assert np.max(np.abs(fast[fin] - want[fin]) / want[fin]) <= 1e-10


def test_uneven_grids_full_size_equal_oracle(solver):
    b = syn.uneven_grids(200)
    horiz = max(range(200), key=lambda q: b.grids[q].nx * b.grids[q].ny)
    deep = max(range(200), key=lambda q: b.grids[q].nz)
    var = next(q for q in range(200) if b.grids[q].depth_km is not None and q not in (horiz, deep))
    pick = [horiz, deep, var]
    grids = [b.grids[q] for q in pick]
    slow = [b.slowness[q] for q in pick]
    seeds = [point_source(g, s, *b.sources[q]) for g, s, q in zip(grids, slow, pick)]
    got = solver.solve_multi(grids, slow, [0, 1, 2], seeds, precision=64, mode=L.MODE_ENGINE)
    for f in range(3):
        want, ok, _ = O.relax(O.Grid.of(grids[f]), slow[f], *seeds[f])
        assert ok and np.array_equal(got[f], want), f"grid {pick[f]} ({grids[f].nx}x{grids[f].ny}x{grids[f].nz})"


def test_regional_401_rays_sample_equal_oracle(solver):
    p = syn.regional_401(n_stations=400, n_events=5000, n_rays=10)
    rng = np.random.default_rng(5)
    stations = [17, 311]
    table_src = np.stack([p.stations[s] for s in stations for _ in (0, 1)])
    table_ph = np.array([0, 1, 0, 1], np.int32)
    with loc.Tables.build(solver, p.grid, p.slowness, table_src, table_ph) as tables:
        tb = tables.copy()
    ev = rng.choice(len(p.events), size=2000, replace=True)
    tab_of = rng.integers(0, 4, size=2000).astype(np.int32)
    events = p.events[ev]
    step = step_km(p.grid, p.inv)
    gpu = trace_rows(solver, p.grid, tb, table_src, p.inv, tab_of, events, step)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(p.grid), tb, tab_of, table_src[tab_of], O.Grid.of(p.inv), events,
                                           step, cap_per_row=8192)
    assert np.count_nonzero(nnz >= 0) > 1900
    compare_rows(gpu, nnz, nodes, lens, tg)
