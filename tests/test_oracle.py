"""The CPU oracle against the reference's known-answer tests (tests/golden/kat.json) and its own
invariants. No GPU."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import synthetic as syn

KAT = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "kat.json")))


def grid_of(d):
    return O.Grid(d["min_lon"], d["max_lon"], d["min_lat"], d["max_lat"], d["min_depth_km"], d["max_depth_km"],
                  d["nx"], d["ny"], d["nz"])


def test_fast_marching_homogeneous_corners():
    """NumericsTests.FastMarchingMatchesStraightRaysInAHomogeneousModel (NumericsTests.cs:88-104)."""
    k = KAT["homogeneous_corners"]
    g = grid_of(k["grid"])
    assert (g.nx, g.ny, g.nz) == (61, 61, 31)
    s = np.full(g.count, 1 / k["velocity"])
    si, st = O.point_source(g, s, *k["source"])
    t = O.fmm(g, s, si, st)
    worst = max(abs(t[(kk * g.ny + j) * g.nx + i] - ex) / ex for (i, j, kk), ex in zip(k["nodes"], k["exact"]))
    assert worst < k["tolerance"]


def test_relax_homogeneous_corners():
    """The sweeping solver (the device scheme's host reference) meets the same known answer."""
    k = KAT["homogeneous_corners"]
    g = grid_of(k["grid"])
    s = np.full(g.count, 1 / k["velocity"])
    si, st = O.point_source(g, s, *k["source"])
    t, ok, rounds = O.relax(g, s, si, st)
    assert ok and rounds[0] >= 1 and rounds[1] >= 1
    worst = max(abs(t[(kk * g.ny + j) * g.nx + i] - ex) / ex for (i, j, kk), ex in zip(k["nodes"], k["exact"]))
    assert worst < k["tolerance"]


def test_trilinear_weights_known_answer():
    """NumericsTests.TrilinearWeightsSumToOneAndInterpolateLinearFieldsExactly (:107-123)."""
    k = KAT["trilinear"]
    g = grid_of(k["grid"])
    nodes, w = O.trilinear(g, *k["point"])
    assert abs(w.sum() - 1) < 1e-12
    lon, lat, cl, dep = O.coords(g)
    L, A, D = np.meshgrid(lon, lat, dep, indexing="ij")
    field = (2 * L - A + 0.1 * D).transpose(2, 1, 0).reshape(-1)
    assert abs(O.interpolate(g, field, *k["point"]) - k["linear_value"]) < 1e-9


def test_fast_marching_gradient_model_analytic():
    """Validation case eikonal-gradient (Program.cs:107-132): v = 4 + 0.05 z against the closed form,
    within the validation threshold (common.py: 5 %)."""
    k = KAT["gradient_model"]
    g = grid_of(k["grid"])
    lon, lat, cl, dep = O.coords(g)
    v = k["v0"] + k["gradient"] * dep
    s = np.broadcast_to((1 / v)[:, None, None], (g.nz, g.ny, g.nx)).reshape(-1).copy()
    si, st = O.point_source(g, s, *k["source"])
    t = O.fmm(g, s, si, st)
    rows = np.array(k["rows"])
    idx = ((rows[:, 2] * g.ny + rows[:, 1]) * g.nx + rows[:, 0]).astype(int)
    rel = np.abs(t[idx] - rows[:, 4]) / rows[:, 4]
    assert rel.max() < k["tolerance"]
    assert rel.mean() < 0.01


def test_relax_tolerance_zero_is_a_fixed_point():
    """tol = 0 runs to the exact fixed point: one more round changes nothing."""
    g = O.Grid(10, 11, 42, 43, 0, 30, 17, 15, 11)
    rng = np.random.default_rng(7)
    s = 1 / (5 + rng.uniform(-0.5, 0.5, g.count))
    si, st = O.point_source(g, s, 10.4, 42.3, 7)
    t, ok, rounds = O.relax(g, s, si, st, tol=0.0)
    assert ok
    t2, ok2, _ = O.relax(g, s, si, st, tol=0.0)
    assert np.array_equal(t, t2)


def test_relax_close_to_fast_marching():
    """Sweeping and marching solve the same discrete equations: close, not equal."""
    g = O.Grid(10, 11, 42, 43, 0, 30, 25, 21, 13)
    lon, lat, cl, dep = O.coords(g)
    s = np.broadcast_to((1 / (5 + 0.04 * dep))[:, None, None], (g.nz, g.ny, g.nx)).reshape(-1).copy()
    si, st = O.point_source(g, s, 10.5, 42.5, 5)
    a = O.fmm(g, s, si, st)
    b, ok, _ = O.relax(g, s, si, st)
    assert ok
    assert np.max(np.abs(a - b) / np.maximum(a, 1e-9)) < 0.02


def test_relax_unsettled_reports():
    g = O.Grid(10, 11, 42, 43, 0, 30, 25, 21, 13)
    s = np.full(g.count, 0.2)
    si, st = O.point_source(g, s, 10.5, 42.5, 5)
    _, ok, rounds = O.relax(g, s, si, st, max_rounds=1)
    assert not ok and rounds[0] == 1


def test_table_rounding():
    """TravelTimeTable.Write (TravelTimeTable.cs:73): float32, non-finite → +inf."""
    t = np.array([1.0, 1 / 3, np.inf, np.nan, -np.inf, 1e40])
    f = O.to_table(t)
    assert f[0] == 1.0 and f[1] == np.float32(1 / 3)
    assert np.isinf(f[2]) and np.isinf(f[3]) and f[4] == np.inf and np.isinf(f[5])


def test_ray_row_consistent_with_field_time():
    """Validation 'rays' case (Program.cs:173-183): Σ length·slowness along a traced ray is close to
    the field time (reference max 2.13 %, threshold 5 %)."""
    g = O.Grid(13, 13.5, 43, 43.4, 0, 20, 41, 45, 21)
    lon, lat, cl, dep = O.coords(g)
    s = np.broadcast_to((1 / (5 + 0.05 * dep))[:, None, None], (g.nz, g.ny, g.nx)).reshape(-1).copy()
    src = (13.25, 43.2, 0.0)
    si, st = O.point_source(g, s, *src)
    t, ok, _ = O.relax(g, s, si, st)
    tb = O.to_table(t)
    step = 0.25 * O.min_spacing_km(g)
    worst = 0
    for ev in [(13.05, 43.05, 12.0), (13.45, 43.35, 8.0), (13.3, 43.1, 18.0)]:
        ray = O.backtrack(g, tb, src, *ev, step)
        assert ray is not None and len(ray) > 3
        nodes, lens = O.kernel(g, ray)
        kt = float(np.sum(lens * s[nodes]))
        ft = O.table_time(g, tb, *ev)
        worst = max(worst, abs(kt - ft) / ft)
    assert worst < 0.05


def test_variable_spacing_uniform_limit():
    """Extension: an explicit depth array equal to the uniform one reproduces the uniform result closely
    (the non-uniform stencil reduces to the uniform one up to rounding)."""
    d = dict(min_lon=10, max_lon=11, min_lat=42, max_lat=43, min_depth_km=0, max_depth_km=24, nx=17, ny=15, nz=13)
    g = grid_of(d)
    gv = O.Grid(10, 11, 42, 43, 0, 24, 17, 15, 13, depth_km=np.linspace(0, 24, 13))
    s = np.full(g.count, 0.18)
    si, st = O.point_source(g, s, 10.5, 42.5, 6)
    a, ok, _ = O.relax(g, s, si, st)
    si2, st2 = O.point_source(gv, s, 10.5, 42.5, 6)
    b, ok2, _ = O.relax(gv, s, si2, st2)
    assert ok and ok2
    fin = np.isfinite(a)
    assert np.max(np.abs(a[fin] - b[fin]) / np.maximum(a[fin], 1e-9)) < 1e-3


def test_relax_wake_zero_is_relax():
    """Node-level due flags with every drop waking (the reference's rule) reproduce Relax to the bit."""
    g = O.Grid(10, 11, 42, 43, 0, 30, 19, 17, 11)
    rng = np.random.default_rng(17)
    s = 1 / (5 + rng.uniform(-0.5, 0.5, g.count))
    si, st = O.point_source(g, s, 10.4, 42.3, 7)
    a, ok, r, _ = O.relax_wake(g, s, si, st, 0.0)
    b, ok2, r2 = O.relax(g, s, si, st)
    assert ok and ok2 and np.array_equal(a, b) and list(r) == list(r2)


def test_relax_wake_threshold_bound():
    """Not propagating drops below 1e-13 of the time keeps fields within 1e-10 relative of Relax."""
    g = O.Grid(10, 11, 42, 43, 0, 30, 31, 29, 17)
    rng = np.random.default_rng(19)
    s = (1 / (5 + 0.04 * np.repeat(np.linspace(0, 30, 17), 31 * 29))) * (1 + 0.05 * rng.standard_normal(g.count))
    si, st = O.point_source(g, s, 10.4, 42.3, 3)
    a, ok, _, ev_fast = O.relax_wake(g, s, si, st, 1e-13)
    b, ok2, _, ev_exact = O.relax_wake(g, s, si, st, 0.0)
    fin = np.isfinite(b)
    assert ok and ok2 and np.array_equal(fin, np.isfinite(a))
    assert np.max(np.abs(a[fin] - b[fin]) / np.maximum(b[fin], 1e-9)) < 1e-10


def test_relax_wake_causal_rule_bound():
    """Waking only the neighbours above the new time (the engine's fast mode) skips evaluations that
    cannot lower a node: the field stays within 1e-10 relative of Relax with fewer evaluations."""
    g = O.Grid(10, 11, 42, 43, 0, 30, 31, 29, 17)
    rng = np.random.default_rng(23)
    s = (1 / (5 + 0.04 * np.repeat(np.linspace(0, 30, 17), 31 * 29))) * (1 + 0.05 * rng.standard_normal(g.count))
    si, st = O.point_source(g, s, 10.6, 42.5, 9)
    b, ok, _ = O.relax(g, s, si, st)
    _, _, _, ev_ref = O.relax_wake(g, s, si, st, 0.0)
    for wake in (0.0, 1e-13):
        a, ok2, _, ev = O.relax_wake(g, s, si, st, wake, causal=True)
        fin = np.isfinite(b)
        assert ok and ok2 and np.array_equal(fin, np.isfinite(a))
        assert np.max(np.abs(a[fin] - b[fin]) / np.maximum(b[fin], 1e-9)) < 1e-10
        assert ev < ev_ref


def test_lsqr_oracle_pinned_to_scipy():
    """The LSQR restatement (Lsqr.cs) follows the SOL kernel SciPy's lsqr implements: the same first
    iterates to rounding, the same stopping rule and solution at convergence, and the damped normal
    equations' solution."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as sla

    rng = np.random.default_rng(3)
    A = sp.random(300, 120, density=0.05, random_state=4, format="csr")
    b = rng.standard_normal(300)
    for damp in (0.0, 0.3):
        x5, code5, _ = O.lsqr(300, 120, A.indptr, A.indices, A.data, b, damp=damp, max_iterations=5, atol=0, btol=0,
                              conlim=0)
        r5 = sla.lsqr(A, b, damp=damp, atol=0, btol=0, conlim=0, iter_lim=5)
        assert code5 == 3 and np.max(np.abs(x5 - r5[0])) <= 1e-12 * np.max(np.abs(r5[0]))
        x, code, info = O.lsqr(300, 120, A.indptr, A.indices, A.data, b, damp=damp)
        r = sla.lsqr(A, b, damp=damp, atol=1e-8, btol=1e-8, conlim=1e8, iter_lim=500)
        assert code == 5 and r[1] == 2  # normal equations satisfied (atol) in both
        assert np.max(np.abs(x - r[0])) <= 1e-6 * np.max(np.abs(r[0]))
        xs = np.linalg.solve((A.T @ A).toarray() + damp ** 2 * np.eye(120), A.T @ b)
        assert np.max(np.abs(x - xs)) <= 1e-6 * np.max(np.abs(xs))
    # Degenerate systems end as the reference says.
    _, code, _ = O.lsqr(300, 120, A.indptr, A.indices, A.data, np.zeros(300))
    assert O.LSQR_STOPS[code] == "zero right-hand side"


def _oracle_tables(job):
    """The job's P and S tables from the oracle's sweeping (SphericalEikonal.Relax), rounded to float32."""
    g = O.Grid.of(job.grid)
    tabs = []
    for phase, src in zip(job.table_phase, job.table_source):
        idx, t = O.point_source(g, job.slowness[phase], *src)
        f, ok, _ = O.relax(g, job.slowness[phase], idx, t)
        assert ok
        tabs.append(O.to_table(f))
    return g, np.stack(tabs)


def test_location_helpers_known_answers():
    """WeightedMedian, Median and Gap (Location/EventLocator.cs:297-327) on hand-worked cases, and the
    origin time as a DateTime holds it (100 ns ticks, truncated)."""
    # Sorted (value, weight): (1, 1) (2, 1) (3, 1); NaN dropped; half of 3 is 1.5 -> 2.
    assert O.weighted_median([3, 1, 2, np.nan], [1, 1, 1, 5]) == 2.0
    # A heavy value takes the median: (1, 0.5) (5, 3) (9, 0.5) -> half 2, reached at 5.
    assert O.weighted_median([9, 1, 5], [0.5, 0.5, 3]) == 5.0
    # Ties keep their input order (stable): the first 2 reaches half.
    assert O.weighted_median([2, 2, 7], [1, 1, 1]) == 2.0
    assert O.weighted_median([np.nan], [1]) == 0.0
    assert O.median([4, 1, 3, 2]) == 2.5 and O.median([5, 1, 3]) == 3.0 and O.median([]) == 0.0
    assert O.median([np.nan, 2.0]) == 2.0
    assert O.gap([10, 100, 100, 300]) == 200.0 and O.gap([45]) == 360.0
    assert O.gap([0, 90, 180, 270]) == 90.0
    assert O.tick_seconds(1.23456789012) == 1.2345678
    assert O.tick_seconds(-2.00000019) == -2.0000001
    assert O.tick_seconds(3.0) == 3.0


def test_location_oracle_moves_events_towards_the_truth():
    """PipelineTests.RelocationMovesEventsTowardsTheTruth (tests/TomoStar.Tests/PipelineTests.cs:95-107):
    12 stations, 30 events, picks with 30 ms noise; every event located, the median horizontal error
    at least halved. Also: gross errors rejected, and the residuals of the kept picks near the noise."""
    job = syn.relocation_small()
    g, tabs = _oracle_tables(job)
    picks = syn.relocation_picks(job, tabs)
    ts_ = np.ascontiguousarray(job.table_source[:, :2])
    out, res = O.locate_many(g, tabs, ts_, O.LocatorSettings(), job.start, picks.offsets, picks.table,
                             picks.seconds, picks.weight, picks.correction)
    assert (out["status"] == 0).all()
    before = syn.surface_distance_km(job.start[:, 0], job.start[:, 1], job.truth[:, 0], job.truth[:, 1])
    after = syn.surface_distance_km(out["lon"], out["lat"], job.truth[:, 0], job.truth[:, 1])
    assert np.median(after) < 0.5 * np.median(before), (np.median(before), np.median(after))
    assert np.median(np.abs(out["t0"] - job.truth[:, 3])) < 0.1
    assert out["rejected"].sum() > 0 and np.median(out["rms"]) < 0.05
    assert (out["used"] + out["rejected"] == np.diff(picks.offsets)).all()
    assert np.isfinite(res).all() and (out["gap_deg"] > 0).all() and (out["gap_deg"] <= 360).all()


def test_location_oracle_fixed_depth_and_local_search():
    """FixDepth keeps every event at its start depth (EventLocator.cs:140, 150-153, 184); a local
    search (GlobalSearch off) from starts a few km off still moves the events towards the truth."""
    job = syn.relocation_small()
    g, tabs = _oracle_tables(job)
    picks = syn.relocation_picks(job, tabs)
    ts_ = np.ascontiguousarray(job.table_source[:, :2])
    args = (job.start, picks.offsets, picks.table, picks.seconds, picks.weight, picks.correction)
    fixed, _ = O.locate_many(g, tabs, ts_, O.LocatorSettings(fix_depth=1), *args)
    assert (fixed["status"] == 0).all() and np.array_equal(fixed["depth_km"], job.start[:, 2])
    assert (fixed["err_depth_km"] == 0).all()
    local, _ = O.locate_many(g, tabs, ts_, O.LocatorSettings(global_search=0), *args)
    before = syn.surface_distance_km(job.start[:, 0], job.start[:, 1], job.truth[:, 0], job.truth[:, 1])
    after = syn.surface_distance_km(local["lon"], local["lat"], job.truth[:, 0], job.truth[:, 1])
    assert (local["status"] == 0).all() and np.median(after) < 0.5 * np.median(before)
