"""Event location on device-resident tables (EventLocator.Locate, Relocation.Absolute) against the
oracle's restatement on the same float32 tables.

The grid search, the outlier rule and the residuals use no transcendental function, so with Geiger's
iterations switched off every location, origin time, residual and count equals the oracle's to the
bit. Geiger's step uses sin/cos/asin/atan2, whose last bits differ between CUDA and glibc, so with
the iterations on the bar is a tolerance: 1e-7 degrees (1 cm), 1e-5 km, 1e-6 s."""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import location as loc
from tomostar_b200 import synthetic as syn

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(solver):
    job = syn.relocation_small()
    tables = loc.Tables.build(solver, job.grid, job.slowness, job.table_source, job.table_phase)
    tabs = tables.copy()
    picks = syn.relocation_picks(job, tabs)
    yield job, tables, tabs, picks
    tables.close()


def _both(solver, job, tables, tabs, picks, start=None, **kw):
    start = job.start if start is None else start
    tsta = job.table_source[:, :2]
    dev = loc.locate(solver, tables, start, picks.offsets, picks.table, picks.seconds, picks.weight,
                     picks.correction, tsta, loc.LocatorSettings(**kw))
    ora, res = O.locate_many(O.Grid.of(job.grid), tabs, tsta, O.LocatorSettings(**kw), start, picks.offsets,
                             picks.table, picks.seconds, picks.weight, picks.correction)
    return dev, ora, res


def test_tables_equal_the_oracle_sweeping(small):
    """TravelTimeTableSet.Build on the device: every table is SphericalEikonal.Relax's field rounded to
    float32, to the bit."""
    job, _, tabs, _ = small
    g = O.Grid.of(job.grid)
    for t in (0, 5, 12, 23):
        ph = job.table_phase[t]
        idx, tt = O.point_source(g, job.slowness[ph], *job.table_source[t])
        f, ok, _ = O.relax(g, job.slowness[ph], idx, tt)
        assert ok and np.array_equal(tabs[t], O.to_table(f))


def test_grid_search_and_outlier_rule_bitwise(solver, small):
    """Geiger off: the search's node and weighted-median origin time, the outlier rounds, residuals,
    counts and gap equal the oracle's exactly; with the quality-class weights (the warp search) and
    with weights whose sums round (0.3 times them: the thread search)."""
    job, tables, tabs, picks = small
    odd = syn.Picks(picks.offsets, picks.table, picks.seconds, picks.weight * 0.3, picks.correction)
    for pk, kw in ((picks, {}), (picks, {"fix_depth": 1}), (picks, {"global_search": 0}),
                   (picks, {"coarse_candidates": 300}), (odd, {}), (odd, {"fix_depth": 1})):
        dev, ora, res = _both(solver, job, tables, tabs, pk, max_geiger_iterations=0, **kw)
        d = dev.locations
        for f in ("t0", "lon", "lat", "depth_km", "rms", "gap_deg", "used", "rejected", "iterations", "status"):
            assert np.array_equal(d[f], ora[f]), (kw, f)
        assert np.array_equal(dev.residuals, res), kw
        fin = np.isfinite(ora["err_h_km"])
        assert np.array_equal(fin, np.isfinite(d["err_h_km"]))
        for f in ("err_h_km", "err_minor_km", "err_depth_km", "err_time_s"):
            assert np.allclose(d[f][fin], ora[f][fin], rtol=1e-9, atol=1e-12), (kw, f)


@pytest.mark.parametrize("kw", [{}, {"fix_depth": 1}, {"global_search": 0}, {"damping": 0.5}])
def test_locate_matches_oracle(solver, small, kw):
    job, tables, tabs, picks = small
    dev, ora, res = _both(solver, job, tables, tabs, picks, **kw)
    d = dev.locations
    assert np.array_equal(d["status"], ora["status"]) and (d["status"] == 0).all()
    for f in ("used", "rejected"):
        assert np.array_equal(d[f], ora[f]), f
    assert np.max(np.abs(d["iterations"] - ora["iterations"])) <= 1
    assert np.max(np.abs(d["lon"] - ora["lon"])) <= 1e-7
    assert np.max(np.abs(d["lat"] - ora["lat"])) <= 1e-7
    assert np.max(np.abs(d["depth_km"] - ora["depth_km"])) <= 1e-5
    assert np.max(np.abs(d["t0"] - ora["t0"])) <= 1e-6
    assert np.max(np.abs(d["rms"] - ora["rms"])) <= 1e-6
    assert np.max(np.abs(dev.residuals - res)) <= 2e-6
    assert np.max(np.abs(d["gap_deg"] - ora["gap_deg"])) <= 1e-5
    for f in ("err_h_km", "err_minor_km", "err_depth_km", "err_time_s"):
        assert np.allclose(d[f], ora[f], rtol=1e-4, atol=1e-7), f
    # The job's own bar (PipelineTests.cs:104-106): events moved towards the truth.
    before = syn.surface_distance_km(job.start[:, 0], job.start[:, 1], job.truth[:, 0], job.truth[:, 1])
    after = syn.surface_distance_km(d["lon"], d["lat"], job.truth[:, 0], job.truth[:, 1])
    assert np.median(after) < 0.5 * np.median(before)


def test_locate_edge_cases(solver, small):
    """Too few phases (the start returned, status 1), an event with no picks, a local search from a
    start far outside the grid (status 2, nothing used), events of over 32 and over 128 picks (the larger
    search classes: every pick repeated), and unreachable nodes (+inf in a table) counted as the
    reference counts them."""
    job, tables, tabs, picks = small
    n = len(job.start)
    counts = np.diff(picks.offsets)
    # Event 0 keeps 3 picks, event 1 none, events 2 and 3 every pick repeated 3 and 8 times.
    sel, offs = [], [0]
    for e in range(n):
        q = np.arange(picks.offsets[e], picks.offsets[e + 1])
        q = q[:3] if e == 0 else q[:0] if e == 1 else np.repeat(q, 3) if e == 2 else np.repeat(q, 8) if e == 3 else q
        sel.append(q)
        offs.append(offs[-1] + len(q))
    sel = np.concatenate(sel)
    p2 = syn.Picks(np.array(offs, np.int32), picks.table[sel], picks.seconds[sel], picks.weight[sel],
                   picks.correction[sel])
    assert offs[3] - offs[2] > 32 and offs[4] - offs[3] > 128 and counts.max() < 32
    start = job.start.copy()
    start[4] = [start[4, 0] + 30.0, start[4, 1], start[4, 2]]
    dev, ora, res = _both(solver, job, tables, tabs, p2, start=start, global_search=0, max_geiger_iterations=0)
    d = dev.locations
    assert list(d["status"][:5]) == [1, 1, 0, 0, 2] and np.array_equal(d["status"], ora["status"])
    assert d["used"][0] == 3 and d["used"][1] == 0 and d["used"][4] == 0
    assert np.array_equal(d["lon"], ora["lon"]) and np.array_equal(d["t0"], ora["t0"])
    assert np.array_equal(np.isnan(dev.residuals), np.isnan(res))
    assert np.array_equal(dev.residuals[~np.isnan(res)], res[~np.isnan(res)])
    # Unreachable nodes: a block of +inf in every P table (the search's NaN residuals, Time's +inf).
    bad = tabs.copy()
    nx, ny = job.grid.nx, job.grid.ny
    block = np.zeros((job.grid.nz, ny, nx), bool)
    block[10:, :8, :8] = True
    bad[:12, block.reshape(-1)] = np.inf
    with loc.Tables.upload(solver, job.grid, bad) as t2:
        dev, ora, res = _both(solver, job, t2, bad, picks, max_geiger_iterations=0)
        for f in ("t0", "lon", "lat", "depth_km", "used", "rejected", "status"):
            assert np.array_equal(dev.locations[f], ora[f]), f
        assert np.array_equal(np.isnan(dev.residuals), np.isnan(res))


def test_locate_refusals(solver, small):
    job, tables, tabs, picks = small
    tsta = job.table_source[:, :2]
    big = np.array([0, 1025], np.int32)
    with pytest.raises(L.TsError):  # more than 1024 picks in one event
        loc.locate(solver, tables, job.start[:1], big, np.zeros(1025, np.int32), np.zeros(1025), np.ones(1025),
                   np.zeros(1025), tsta)
    with pytest.raises(L.TsError):  # a table index beyond the tables
        loc.locate(solver, tables, job.start[:1], np.array([0, 4], np.int32), np.array([0, 1, 2, 99], np.int32),
                   np.zeros(4), np.ones(4), np.zeros(4), tsta)
    with pytest.raises(L.TsError):  # tables need a uniform grid
        g = syn.regular_grid(9, 9, 5, 1.0, depth_km=np.array([0.0, 1.0, 2.5, 4.5, 7.0]))
        loc.Tables.upload(solver, g, np.zeros((1, g.count), np.float32))
