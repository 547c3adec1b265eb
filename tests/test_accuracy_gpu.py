"""Accuracy of every precision against the FP64 oracle on each named workload (reduced where the
oracle would take minutes), with the figures printed (`pytest -s`): relative error max and p99, and
the largest absolute error in seconds.

* FP64 engine (exact rule): equal to the oracle's Relax (0).
* FP64 fast mode, delivered as float32 tables (the headline): within 2e-5 relative (in fact the
  float32 rounding, ~6e-8).
* FP32 arithmetic (the reference's paired-float scheme, times as hi + lo floats): within 2e-5
  relative at every node (measured: a few 1e-6 at most).
"""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source

pytestmark = pytest.mark.gpu


def errors(a, ref):
    fin = np.isfinite(ref)
    assert np.array_equal(fin, np.isfinite(a)), "reached sets differ"
    d = np.abs(a[fin].astype(np.float64) - ref[fin])
    rel = d / np.maximum(ref[fin], 1e-9)
    return float(rel.max()), float(np.percentile(rel, 99)), float(d.max())


def report(name, rows):
    print(f"\n{name}")
    for label, (mx, p99, ab) in rows:
        print(f"  {label:34s} max rel {mx:.2e}  p99 rel {p99:.2e}  max abs {ab:.2e} s")


def check(solver, name, cases):
    """cases: list of (grid, slowness, seed set); all compared against the oracle's Relax."""
    acc = {"fp64 engine": [], "fp64 fast -> float32 tables": [], "fp32 arithmetic": []}
    for g, s, seeds in cases:
        ref = O.relax(O.Grid.of(g), s, *seeds)[0]
        exact = solver.solve(g, s, [seeds], precision=64, mode=L.MODE_ENGINE)[0]
        tables = solver.solve(g, s, [seeds], precision=64, mode=L.MODE_FAST,
                              output=np.empty((1, g.count), np.float32))[0]
        f32 = solver.solve(g, s, [seeds], precision=32, mode=L.MODE_ENGINE)[0]
        acc["fp64 engine"].append(errors(exact, ref))
        acc["fp64 fast -> float32 tables"].append(errors(tables, ref))
        acc["fp32 arithmetic"].append(errors(f32, ref))
    rows = [(k, tuple(max(e[i] for e in v) for i in range(3))) for k, v in acc.items()]
    report(name, rows)
    r = dict(rows)
    assert r["fp64 engine"][0] == 0.0
    assert r["fp64 fast -> float32 tables"][0] <= 2e-5
    assert r["fp32 arithmetic"][0] <= 2e-5


def test_accuracy_single_source_61(solver):
    p = syn.single_source_61()
    check(solver, "61x61x31 at 1 km (one source)",
          [(p.grid, p.slowness[0], point_source(p.grid, p.slowness[0], *p.stations[0]))])


def test_accuracy_inversion_step_121(solver):
    p = syn.inversion_step_121()
    cases = [(p.grid, p.slowness[ph], point_source(p.grid, p.slowness[ph], *p.stations[q]))
             for ph in (0, 1) for q in (0, 7)]
    check(solver, "121x121x61 at 0.5 km (P and S, 2 stations)", cases)


def test_accuracy_uneven_grids_reduced(solver):
    b = syn.uneven_grids(n_sources=6, seed=3, dims_scale=0.35)
    cases = [(g, s, point_source(g, s, *src)) for g, s, src in zip(b.grids, b.slowness, b.sources)]
    check(solver, "uneven grids, half with geometric depth spacing (6 grids at 35 % size)", cases)


def test_accuracy_regional_401_one_field(solver):
    """The 401x401x121 workload against the bitwise FP64 engine (equal to Relax to the bit by the
    tests above; the oracle itself would take minutes here)."""
    p = syn.regional_401(n_stations=2, n_events=10, n_rays=10)
    seeds = point_source(p.grid, p.slowness[0], *p.stations[1])
    ref = solver.solve(p.grid, p.slowness[0], [seeds], precision=64, mode=L.MODE_ENGINE)[0]
    tables = solver.solve(p.grid, p.slowness[0], [seeds], precision=64, mode=L.MODE_FAST,
                          output=np.empty((1, p.grid.count), np.float32))[0]
    f32 = solver.solve(p.grid, p.slowness[0], [seeds], precision=32, mode=L.MODE_ENGINE)[0]
    rows = [("fp64 fast -> float32 tables", errors(tables, ref)), ("fp32 arithmetic", errors(f32, ref))]
    report("401x401x121 at 0.25 km (one P field)", rows)
    assert rows[0][1][0] <= 2e-5
    assert rows[1][1][0] <= 2e-5
