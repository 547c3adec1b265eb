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
