"""ForwardModel.FromInversionGrid on the device (ts_model_put_resampled) against the oracle, bit for bit,
on the refined domain and on a covering domain with a 1-D background; and solves on that model."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import domain
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source

pytestmark = pytest.mark.gpu


def _model():
    inv = syn.regular_grid(21, 17, 9, 2.5)
    rng = np.random.default_rng(2)
    vp = syn.vp_linear(inv, 5.0, 0.05) * (1 + 0.04 * rng.standard_normal(inv.count))
    return inv, np.stack([1 / vp, 1.73 / vp])


@pytest.mark.parametrize("extended", [False, True])
@pytest.mark.parametrize("precision", [64, 32])
def test_resampled_model_matches_oracle(solver, extended, precision):
    inv, s = _model()
    bg = None
    pts = [[inv.min_lon + 0.1, inv.min_lat + 0.1, 1.0]]
    if extended:
        pts.append([inv.max_lon + 0.5, inv.min_lat - 0.3, 30.0])
        bg = domain.Background(np.array([0.0, 15.0, 15.0, 40.0]), np.array([5.2, 6.1, 6.6, 7.9]),
                               np.array([3.0, 3.5, 3.8, 4.5]))
    fwd, ext, _ = domain.covering(inv, 2, pts)
    assert ext == extended
    mid = domain.put_resampled(solver, fwd, inv, s, bg, precision)
    want = O.resample(O.Grid.of(fwd), O.Grid.of(inv), s,
                      None if bg is None else (bg.depth_km, bg.vp, bg.vs))
    for p in range(2):
        got = domain.copy_slowness(solver, mid, p, fwd.count)
        exp = want[p] if precision == 64 else want[p].astype(np.float32).astype(np.float64)
        assert np.array_equal(got, exp), (p, np.max(np.abs(got - exp)))
    if extended:  # nodes outside the inversion grid carry the background
        assert not np.allclose(want[0], want[0][0])
    # The resident model solves: the same field as a solve on the oracle's slowness.
    if precision == 64:
        idx, t = point_source(fwd, want[0], inv.min_lon + 0.2, inv.min_lat + 0.15, 0.0)
        idx = np.ascontiguousarray(idx, np.int32)
        t = np.ascontiguousarray(t, np.float64)
        off = np.array([0, len(idx)], np.int32)
        a = np.empty(fwd.count)
        P = C.POINTER
        rc = L.load().ts_eik_solve_model(solver.handle, mid, 0, 1, off.ctypes.data_as(P(C.c_int32)),
                                         idx.ctypes.data_as(P(C.c_int32)), t.ctypes.data_as(P(C.c_double)),
                                         L.MODE_ENGINE, 1e-7, 0, a.ctypes.data_as(C.c_void_p), 0, None)
        assert rc == 0, solver.last_error
        b = solver.solve(fwd, want[0], [(idx, t)], precision=64)[0]
        assert np.array_equal(a, b)
    assert L.load().ts_model_drop(solver.handle, mid) == 0


def test_resample_refusals(solver):
    inv, s = _model()
    g = syn.regular_grid(9, 9, 5, 1.0, depth_km=np.array([0.0, 1.0, 2.5, 4.5, 7.0]))
    with pytest.raises(L.TsError):
        domain.put_resampled(solver, g, inv, s)
    with pytest.raises(L.TsError):
        domain.put_resampled(solver, inv.refined(2), inv, np.concatenate([s, s]))  # three or four phases


def test_forward_step_extended_domain_outside_time(solver):
    """RayKernels.Compute on a covering domain (RayKernels.cs:63-95): stations and events outside the
    inversion grid, the forward model resampled with a 1-D background outside it, rays whose pieces
    outside the inversion grid give time outside (RayRow.OutsideTime) instead of row entries; against
    the oracle's pipeline on the same tables."""
    from test_rays_gpu import compare_rows
    from tomostar_b200.rays import RayKernels, step_km

    inv, s = _model()
    rng = np.random.default_rng(7)
    lon = lambda f: inv.min_lon + f * (inv.max_lon - inv.min_lon)  # noqa: E731
    lat = lambda f: inv.min_lat + f * (inv.max_lat - inv.min_lat)  # noqa: E731
    stations = np.array([[lon(0.2), lat(0.3), 0.0], [lon(0.8), lat(0.6), 0.0], [lon(0.5), lat(0.9), 0.0],
                         [lon(1.35), lat(0.5), 0.0], [lon(0.4), lat(-0.3), 0.0]])
    events = np.array([[lon(f), lat(g), d] for f, g, d in rng.uniform([0.1, 0.1, 3], [0.9, 0.9, 16], (6, 3))] +
                      [[lon(1.25), lat(0.2), 8.0], [lon(-0.3), lat(1.2), 12.0], [lon(0.5), lat(0.5), 28.0]])
    fwd, ext, _ = domain.covering(inv, 2, np.concatenate([stations, events]))
    assert ext
    bg = domain.Background(np.array([0.0, 12.0, 12.0, 40.0]), np.array([5.3, 6.0, 6.4, 7.8]),
                           np.array([3.05, 3.45, 3.7, 4.5]))
    slow = O.resample(O.Grid.of(fwd), O.Grid.of(inv), s, (bg.depth_km, bg.vp, bg.vs))
    arrivals = np.array([[e, k, p] for e in range(len(events)) for k in range(len(stations)) for p in (0, 1)],
                        np.int32)
    domain.set_background(solver, bg)
    try:
        gpu = RayKernels(inv, fwd, solver).compute(slow, stations, events, arrivals, precision=64,
                                                   mode=L.MODE_ENGINE)
    finally:
        domain.set_background(solver, None)
    og = O.Grid.of(fwd)
    tables, index = [], {}
    for p in (0, 1):
        for k in range(len(stations)):
            idx, t = point_source(fwd, slow[p], *stations[k])
            f, ok, _ = O.relax(og, slow[p], idx, t)
            assert ok
            index[(p, k)] = len(tables)
            tables.append(O.to_table(f))
    tab_of = np.array([index[(p, k)] for _, k, p in arrivals], np.int32)
    tab_phase = np.array([p for (p, _k) in sorted(index, key=index.get)], np.int32)
    nnz, nodes, lens, tg, outside = O.ray_rows_many_bg(og, np.stack(tables), tab_of, tab_phase,
                                                       stations[arrivals[:, 1]], O.Grid.of(inv), events[arrivals[:, 0]],
                                                       step_km(fwd, inv), (bg.depth_km, bg.vp, bg.vs))
    compare_rows(gpu, nnz, nodes, lens, tg)
    ok = nnz >= 0
    assert (outside[ok] > 0).sum() >= 10 and (outside[ok] == 0).sum() >= 10
    assert np.max(np.abs(gpu.outside[ok] - outside[ok])) <= 1e-9 * max(1.0, float(outside.max()))
    # Without the background the same rays keep every piece (outside time 0).
    plain = RayKernels(inv, fwd, solver).compute(slow, stations, events, arrivals, precision=64,
                                                 mode=L.MODE_ENGINE)
    assert not plain.outside.any() and plain.nnz > gpu.nnz
