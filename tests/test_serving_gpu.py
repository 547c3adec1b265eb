"""The serving engine on the GPU: continuous batching gives every request the result it gets alone
(to the bit), which is also the one-shot engine's result; admission keeps the device footprint
within the HBM budget; requests beyond the budget are refused with an error."""
import numpy as np
import pytest

from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source
from tomostar_b200.rays import trace_rows
from tomostar_b200.serving import Server

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def models():
    return syn.serving_models()


def submit_spec(server, ids, models, r, tables=True):
    m = models[r.model]
    seeds = [point_source(m.grid, m.slowness[r.phase], *st) for st in r.stations]
    return server.submit(ids[r.model], r.phase, seeds, origins=r.stations,
                         ray_field=r.ray_field if len(r.events) else None,
                         ray_event=r.events if len(r.events) else None, tables=tables)


def rows_equal(a, b):
    if a is None or b is None:
        return a is None and b is None
    return (np.array_equal(a.row_ptr, b.row_ptr) and np.array_equal(a.col, b.col) and np.array_equal(a.len, b.len)
            and np.array_equal(a.tcalc_grad, b.tcalc_grad) and np.array_equal(a.ok, b.ok))


def test_solo_equals_mix_equals_one_shot(models, solver):
    stream = syn.serving_stream(models, rate=200, duration=0.25, seed=4)
    kinds = {r.kind for r in stream}
    assert {"eikonal+rays", "resolution"} <= kinds
    with Server(tile=2, budget_bytes=16e9, rounds_per_epoch=1) as server:
        ids = {name: server.model_put(m.grid, m.slowness) for name, m in models.items()}
        targets = [next(r for r in stream if r.kind == k) for k in ("eikonal+rays", "resolution", "relocation")
                   if any(r.kind == k for r in stream)]
        solo = []
        for r in targets:
            res = server.wait(submit_spec(server, ids, models, r))
            assert res.status == L.TS_OK, res.error
            solo.append(res)
        # The same requests inside the mix: everything of the stream submitted at once, so the
        # targets share epochs with other requests of other grids and are admitted mid-way.
        rid = [submit_spec(server, ids, models, r) for r in stream]
        mixed = {id(r): server.wait(q) for r, q in zip(stream, rid)}
        for r, a in zip(targets, solo):
            b = mixed[id(r)]
            assert b.status == L.TS_OK, b.error
            assert np.array_equal(a.tables, b.tables)
            assert rows_equal(a.rows, b.rows)
        st = server.stats()
        assert st["requests_done"] == len(targets) + len(stream) and st["queued"] == 0 and st["in_flight"] == 0
        assert st["bytes_in_use"] == 0
    # One-shot engine solve (fast mode, float32 tables) and the ray tracer on those tables.
    for r, a in zip(targets, solo):
        m = models[r.model]
        seeds = [point_source(m.grid, m.slowness[r.phase], *st) for st in r.stations]
        one = solver.solve(m.grid, m.slowness[r.phase], seeds, mode=L.MODE_FAST, precision=64,
                           output=np.empty((len(seeds), m.grid.count), np.float32))
        assert np.array_equal(a.tables, one)
        if len(r.events):
            want = trace_rows(solver, m.grid, one, r.stations, m.grid.coarsened(2), r.ray_field, r.events)
            assert rows_equal(a.rows, want)


def test_admission_keeps_within_budget(models, solver):
    m = models["checker81"]
    stream = [r for r in syn.serving_stream(models, rate=200, duration=1.0, seed=4) if r.kind == "resolution"][:4]
    # Room for a little more than one resolution batch at a time: 25 fields of 81×81×41 hold 3.57 MB
    # each (8×8×4 tiles, FP64 field, due masks and its float32 table).
    budget = 1.3 * 25 * 3.57e6
    with Server(tile=2, budget_bytes=budget, rounds_per_epoch=2) as server:
        ids = {name: server.model_put(mm.grid, mm.slowness) for name, mm in models.items() if name in ("checker81", "spike81")}
        rid = [submit_spec(server, ids, models, r) for r in stream]
        results = [server.wait(q) for q in rid]
        for res in results:
            assert res.status == L.TS_OK, res.error
        st = server.stats()
        assert 0 < st["peak_bytes"] <= budget
        # Queued behind the budget: the last request waited for the first ones.
        assert results[-1].queue_ms > 0
        r = stream[0]
        seeds = [point_source(m.grid, models[r.model].slowness[0], *s) for s in r.stations]
        one = solver.solve(m.grid, models[r.model].slowness[0], seeds, mode=L.MODE_FAST, precision=64,
                           output=np.empty((25, m.grid.count), np.float32))
        assert np.array_equal(results[0].tables, one)


def test_request_beyond_budget_is_refused(models):
    with Server(tile=2, budget_bytes=1e6) as server:
        m = models["checker81"]
        mid = server.model_put(m.grid, m.slowness)
        seeds = [point_source(m.grid, m.slowness[0], m.grid.min_lon + 0.1, m.grid.min_lat + 0.1, 0.0)]
        res = server.wait(server.submit(mid, 0, seeds))
        assert res.status == L.TS_E_CAPACITY and "budget" in res.error


def test_flow_scheduler_time_budgeted_epochs(models, solver):
    """Flow scheduler with epochs that end on time (fields pausing at a round end after 5 ms): every
    request still gets the one-shot engine's bits."""
    stream = syn.serving_stream(models, rate=200, duration=0.1, seed=4)
    with Server(tile=4, budget_bytes=16e9, rounds_per_epoch=8, scheduler=1, epoch_ms=5.0) as server:
        ids = {name: server.model_put(m.grid, m.slowness) for name, m in models.items()}
        rid = [submit_spec(server, ids, models, r) for r in stream]
        results = [server.wait(q) for q in rid]
        assert server.stats()["epochs"] > 1
    for r, res in zip(stream, results):
        assert res.status == L.TS_OK, res.error
        m = models[r.model]
        seeds = [point_source(m.grid, m.slowness[r.phase], *st) for st in r.stations]
        one = solver.solve(m.grid, m.slowness[r.phase], seeds, mode=L.MODE_FAST, precision=64,
                           output=np.empty((len(seeds), m.grid.count), np.float32))
        assert np.array_equal(res.tables, one)
