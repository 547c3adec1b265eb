"""Rays and Jacobian rows on the GPU against the oracle's RayTracing.Backtrack/Kernel and RayKernels
finalisation, on the same float32 tables.

Bar: the same arrivals kept/dropped; TCalc and the source gradient to 1e-9 relative; per row, node
sets identical except nodes a ray only grazes (length below 1e-6 of the row's total, the trace of a
ray passing within ~1e-6 of a cell face); common nodes' lengths within 1e-5 relative."""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source
from tomostar_b200.rays import RayKernels, trace_rows

pytestmark = pytest.mark.gpu
LEN_REL_TOL = 1e-5
GRAZE_FRAC = 1e-6


def compare_rows(gpu, nnz, nodes, lens, tg):
    n = len(nnz)
    assert gpu.n_rows == n
    assert np.array_equal(gpu.ok, nnz >= 0), "kept/dropped arrivals differ"
    worst_len, worst_t = 0.0, 0.0
    for r in range(n):
        if nnz[r] < 0:
            continue
        a = gpu.row(r)
        ref_nodes, ref_len = nodes[r, : nnz[r]], lens[r, : nnz[r]]
        worst_t = max(worst_t, abs(a.tcalc - tg[r, 0]) / abs(tg[r, 0]))
        for q in range(3):
            worst_t = max(worst_t, abs([a.ge, a.gn, a.gz][q] - tg[r, 1 + q]) / (np.abs(tg[r, 1:]).max() + 1e-30))
        total = max(float(ref_len.sum()), 1e-30)
        common, ia, ib = np.intersect1d(a.nodes, ref_nodes, return_indices=True)
        only_gpu = np.setdiff1d(np.arange(len(a.nodes)), ia)
        only_ref = np.setdiff1d(np.arange(len(ref_nodes)), ib)
        assert np.all(a.length[only_gpu] <= GRAZE_FRAC * total), (r, "extra nodes on the GPU")
        assert np.all(ref_len[only_ref] <= GRAZE_FRAC * total), (r, "missing nodes on the GPU")
        d = np.abs(a.length[ia].astype(np.float64) - ref_len[ib]) / np.maximum(ref_len[ib], GRAZE_FRAC * total)
        worst_len = max(worst_len, float(d.max()) if len(d) else 0.0)
        assert np.all(np.diff(a.nodes) > 0)
        if nnz[r] == 0:
            assert len(a.nodes) == 0
            continue
    assert worst_t <= 1e-9, worst_t
    assert worst_len <= LEN_REL_TOL, worst_len
    return worst_len


def single_source_61_tables():
    p = syn.single_source_61()
    og = O.Grid.of(p.grid)
    si, st = point_source(p.grid, p.slowness[0], *p.stations[0])
    t, ok, _ = O.relax(og, p.slowness[0], si, st)
    return p, O.to_table(t)


def test_trace_rows_single_source_61_vs_oracle(solver):
    """61×61×31 at 1 km: 25 surface receivers traced back to the source at (30, 30, 10) km."""
    p, tb = single_source_61_tables()
    step = p.step_km
    gpu = trace_rows(solver, p.grid, tb[None, :], p.stations, p.inv, np.zeros(25, np.int32), p.events, step)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(p.grid), tb[None, :], np.zeros(25, np.int32),
                                           np.repeat(p.stations, 25, axis=0), O.Grid.of(p.inv), p.events, step)
    assert np.all(nnz >= 0)
    compare_rows(gpu, nnz, nodes, lens, tg)


def test_trace_rows_edge_cases(solver):
    """Events outside the grid (clamped), at the station, on the surface and at the bottom, and an
    event in an unreached region (dropped)."""
    p, tb = single_source_61_tables()
    g = p.grid
    st = p.stations[0]
    ev = np.array([
        [g.min_lon - 0.01, g.min_lat - 0.01, 0.0],
        st,
        [g.max_lon, g.max_lat, g.max_depth_km],
        [0.5 * (g.min_lon + g.max_lon), g.min_lat, 5.0],
        [g.min_lon + 0.1, g.min_lat + 0.2, 29.9],
    ])
    tb2 = tb.copy()
    tb2[: g.nx * g.ny] = np.inf  # the surface unreached: arrivals there drop
    tables = np.stack([tb, tb2])
    table_of = np.array([0, 0, 0, 0, 0, 1, 1], np.int32)
    evs = np.vstack([ev, [[g.min_lon + 0.2, g.min_lat + 0.2, 0.0], [g.min_lon + 0.2, g.min_lat + 0.2, 15.0]]])
    stations = np.vstack([st, st])
    gpu = trace_rows(solver, g, tables, stations, p.inv, table_of, evs, p.step_km)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(g), tables, table_of, stations[table_of], O.Grid.of(p.inv), evs,
                                           p.step_km)
    assert nnz[5] == -1  # dropped: the surface is unreached
    assert nnz[1] == 0  # the event at the station: a kept, empty row
    compare_rows(gpu, nnz, nodes, lens, tg)


def test_trace_rows_inversion_step_121_sample_vs_oracle(solver):
    """121×121×61 at 0.5 km: 600 P and S rays (a seeded sample of the 7,500) on oracle tables."""
    p = syn.inversion_step_121()
    og = O.Grid.of(p.grid)
    st_ids = [0, 4, 11]
    tabs, tstations = [], []
    for ph in (0, 1):
        for q in st_ids:
            si, stt = point_source(p.grid, p.slowness[ph], *p.stations[q])
            tabs.append(O.to_table(O.relax(og, p.slowness[ph], si, stt)[0]))
            tstations.append(p.stations[q])
    tabs = np.stack(tabs)
    tstations = np.array(tstations)
    rng = np.random.default_rng(12)
    table_of = rng.integers(0, len(tabs), 600).astype(np.int32)
    evs = p.events[rng.integers(0, len(p.events), 600)]
    gpu = trace_rows(solver, p.grid, tabs, tstations, p.inv, table_of, evs, p.step_km)
    nnz, nodes, lens, tg = O.ray_rows_many(og, tabs, table_of, tstations[table_of], O.Grid.of(p.inv), evs, p.step_km)
    compare_rows(gpu, nnz, nodes, lens, tg)
    assert gpu.nnz == int(nnz[nnz >= 0].sum())


def test_forward_step_single_source_61_f64(solver):
    """RayKernels.Compute on the device (tables + rays) against the oracle pipeline, FP64."""
    p, tb = single_source_61_tables()
    rk = RayKernels(p.inv, p.grid, solver)
    gpu = rk.compute(p.slowness, p.stations, p.events, p.arrivals, precision=64, mode=L.MODE_ENGINE)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(p.grid), tb[None, :], np.zeros(25, np.int32),
                                           np.repeat(p.stations, 25, axis=0), O.Grid.of(p.inv), p.events, p.step_km)
    compare_rows(gpu, nnz, nodes, lens, tg)
    rows = gpu.rows()
    assert [r.arrival for r in rows] == list(range(25))


def test_forward_step_f32_close(solver):
    """The FP32 forward step: rows close to the FP64 oracle's (tables differ by the FP32 error)."""
    p, tb = single_source_61_tables()
    rk = RayKernels(p.inv, p.grid, solver)
    gpu = rk.compute(p.slowness, p.stations, p.events, p.arrivals, precision=32, mode=L.MODE_ENGINE)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(p.grid), tb[None, :], np.zeros(25, np.int32),
                                           np.repeat(p.stations, 25, axis=0), O.Grid.of(p.inv), p.events, p.step_km)
    assert np.array_equal(gpu.ok, nnz >= 0)
    for r in range(25):
        a = gpu.row(r)
        assert abs(a.tcalc - tg[r, 0]) / tg[r, 0] < 2e-5
        assert abs(a.length.sum() - lens[r, : nnz[r]].sum()) / lens[r, : nnz[r]].sum() < 1e-3


def test_row_time_consistency(solver):
    """Σ length·slowness of each row is close to TCalc (the reference's 'rays' validation, <5 %)."""
    p, tb = single_source_61_tables()
    rk = RayKernels(p.inv, p.grid, solver)
    gpu = rk.compute(p.slowness, p.stations, p.events, p.arrivals, precision=64, mode=L.MODE_ENGINE)
    s_inv = p.slowness[0].reshape(p.grid.shape)[::2, ::2, ::2].reshape(-1)  # inversion nodes are every other
    for row in gpu.rows():
        kt = float(np.sum(row.length * s_inv[row.nodes]))
        assert abs(kt - row.tcalc) / row.tcalc < 0.05


def _same_rows(a, b):
    assert np.array_equal(a.row_ptr, b.row_ptr)
    assert np.array_equal(a.col, b.col)
    assert np.array_equal(a.len.view(np.uint32), b.len.view(np.uint32))
    assert np.array_equal(a.tcalc_grad.view(np.uint64), b.tcalc_grad.view(np.uint64))
    assert np.array_equal(a.ok, b.ok)
    assert np.array_equal(a.outside.view(np.uint64), b.outside.view(np.uint64))


def test_warp_per_ray_equals_thread_per_ray(solver):
    """ts_rays_set_warp_max picks the kernel: one warp per ray (small calls) and one thread per ray
    trace the same 600 P and S rays of the inversion_step_121 sample to the same rows, bit for bit,
    and both agree with the oracle."""
    lib = L.load()
    p = syn.inversion_step_121()
    og = O.Grid.of(p.grid)
    tabs, tstations = [], []
    for ph in (0, 1):
        for q in (0, 4, 11):
            si, stt = point_source(p.grid, p.slowness[ph], *p.stations[q])
            tabs.append(O.to_table(O.relax(og, p.slowness[ph], si, stt)[0]))
            tstations.append(p.stations[q])
    tabs, tstations = np.stack(tabs), np.array(tstations)
    rng = np.random.default_rng(21)
    table_of = rng.integers(0, len(tabs), 600).astype(np.int32)
    evs = p.events[rng.integers(0, len(p.events), 600)]
    try:
        assert lib.ts_rays_set_warp_max(solver.handle, 100000) == L.TS_OK
        warp = trace_rows(solver, p.grid, tabs, tstations, p.inv, table_of, evs, p.step_km)
        assert lib.ts_rays_set_warp_max(solver.handle, 0) == L.TS_OK
        thread = trace_rows(solver, p.grid, tabs, tstations, p.inv, table_of, evs, p.step_km)
    finally:
        lib.ts_rays_set_warp_max(solver.handle, 2048)
    _same_rows(warp, thread)
    nnz, nodes, lens, tg = O.ray_rows_many(og, tabs, table_of, tstations[table_of], O.Grid.of(p.inv), evs, p.step_km)
    compare_rows(warp, nnz, nodes, lens, tg)
    assert lib.ts_rays_set_warp_max(solver.handle, -1) == L.TS_E_ARG
