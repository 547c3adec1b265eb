"""The CUDA engine against the reference's own device kernel run on the CPU (oracle/_ref: the
EikonalOpenCl.cs:387-624 kernel text compiled as C++ and driven in Sweep's launch order).

* FP64 (the QV_FP64 kernel): every tile shape and the plain path equal it to the bit.
* FP32 (the paired-float kernel, times as hi + lo floats): the engine's FP32 precision is that
  scheme term for term, so it equals it to the bit too, and within 2e-5 relative of the FP64 field.

The reference's batch shares one round flag across its fields (a settled field keeps being swept
while others converge); the engine settles each field on its own. Both equal a batch of one, which
is what is compared here (one field per reference solve). Skipped where oracle/_ref was not built.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn
from tomostar_b200.eikonal import point_source

pytestmark = [pytest.mark.gpu, pytest.mark.skipif(not R.available(), reason="oracle/_ref not built")]
F32_REL_TOL = 2e-5


def _cases():
    p0 = syn.single_source_61()
    yield "single_source_61", p0.grid, p0.slowness[0], p0.stations[0]
    gd, s, src = syn.selftest_case()
    yield "selftest_22x20x16", gd, s, src
    p1 = syn.inversion_step_121()
    yield "inversion_step_121 S", p1.grid, p1.slowness[1], p1.stations[2]


CASES = list(_cases())


@pytest.mark.parametrize("case", CASES, ids=[c[0] for c in CASES])
@pytest.mark.parametrize("precision", [64, 32])
def test_engine_equals_reference_kernel(solver, case, precision):
    _, g, s, src = case
    seeds = point_source(g, s, *src)
    want, st, _ = R.eik_solve(O.Grid.of(g), s, [seeds], precision)
    assert st == 0
    got = solver.solve(g, s, [seeds], precision=precision, mode=L.MODE_ENGINE)
    assert np.array_equal(got[0], want[0])
    if precision == 32:
        ref64 = O.relax(O.Grid.of(g), s, *seeds)[0]
        fin = np.isfinite(ref64) & (ref64 > 0)
        rel = np.abs(got[0] - ref64)[fin] / ref64[fin]
        assert rel.max() <= F32_REL_TOL


@pytest.mark.parametrize("precision", [64, 32])
def test_plain_path_and_every_tile_shape_equal_reference_kernel(solver, precision):
    """A ragged heterogeneous grid: the plain per-plane path and each tile shape, both precisions."""
    gd = syn.regular_grid(37, 29, 19, 0.6)
    rng = np.random.default_rng(23)
    s = 1 / (5.0 + 0.04 * np.repeat(gd.depth(), gd.nx * gd.ny) + 0.25 * rng.standard_normal(gd.count))
    lon, lat, dep = gd.lon(), gd.lat(), gd.depth()
    seeds = point_source(gd, s, lon[7], lat[20], dep[11])
    want, st, _ = R.eik_solve(O.Grid.of(gd), s, [seeds], precision)
    assert st == 0
    plain = solver.solve(gd, s, [seeds], precision=precision, mode=L.MODE_PLAIN)
    assert np.array_equal(plain[0], want[0])
    lib = L.load()
    try:
        for sid, bx, by, bz in L.engine_shapes():
            assert lib.ts_engine_set_tile(solver.handle, precision, sid) == 0
            for sched in (0, 1):
                assert lib.ts_engine_set_scheduler(solver.handle, sched) == 0
                out = solver.solve(gd, s, [seeds], precision=precision)
                assert np.array_equal(out[0], want[0]), f"shape {bx}x{by}x{bz} scheduler {sched}"
    finally:
        lib.ts_engine_set_tile(solver.handle, precision, 0)
        lib.ts_engine_set_scheduler(solver.handle, 0)
