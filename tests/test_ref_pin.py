"""The oracle pinned to the reference's own device code (oracle/_ref: the OpenCL kernel text of
EikonalOpenCl.cs:387-624 and LsqrOpenCl.cs:41-176 compiled as C++ and driven in the host's launch
order). No GPU. Skipped only where neither the reference tree nor a prebuilt oracle/_ref/libref.so is
present.

* FP64: the reference kernel's fields equal the restated Relax (oracle.cpp or_relax), which the CUDA
  engine is tested against bit for bit, to the last bit.
* Paired float (the reference's answer for devices without FP64): its error against the FP64 field
  per workload, the bar the CUDA FP32 mode is held to (2e-5 relative).
* LSQR: the reference's spmv and vector kernels equal the restated products.
"""
import numpy as np
import pytest

from oracle import oracle as O
from oracle import ref as R
from tomostar_b200 import synthetic as syn

pytestmark = pytest.mark.skipif(not R.available(), reason="no reference tree and no prebuilt oracle/_ref")


def _rel(got, want):
    fin = np.isfinite(want) & (want > 0)
    assert np.array_equal(np.isfinite(got), np.isfinite(want))
    return np.abs(got - want)[fin] / want[fin], np.abs(got - want)[fin]


def test_ref_fp64_equals_relax_single_source_61():
    """61x61x31 at 1 km, the source at (30, 30, 10) km: the reference kernel equals Relax to the bit."""
    p = syn.single_source_61()
    g = O.Grid.of(p.grid)
    seeds = O.point_source(g, p.slowness[0], *p.stations[0])
    got, st, rounds = R.eik_solve(g, p.slowness[0], [seeds], 64)
    want, ok, wr = O.relax(g, p.slowness[0], *seeds)
    assert st == 0 and ok and list(rounds) == list(wr)
    assert np.array_equal(got[0], want)


def test_ref_fp64_equals_relax_selftest_case():
    """The device self-test case (EikonalOpenCl.cs:346-374: 22x20x16, heterogeneous slowness)."""
    gd, s, src = syn.selftest_case()
    g = O.Grid.of(gd)
    seeds = O.point_source(g, s, *src)
    got, st, _ = R.eik_solve(g, s, [seeds], 64)
    want, ok, _ = O.relax(g, s, *seeds)
    assert st == 0 and ok and np.array_equal(got[0], want)


def _ragged(dims):
    nx, ny, nz = dims
    gd = syn.regular_grid(nx, ny, nz, 0.7)
    g = O.Grid.of(gd)
    rng = np.random.default_rng(nx * 100 + nz)
    s = 1 / (5.0 + 0.05 * np.repeat(gd.depth(), nx * ny) + 0.3 * rng.standard_normal(g.count))
    lon, lat, _, dep = O.coords(g)
    a = O.point_source(g, s, lon[nx // 3], lat[ny // 2], dep[nz // 2] * 0.9)
    b = O.point_source(g, s, lon[-1], lat[0], dep[-1])
    # A duplicate seed (the smallest time is kept) and one off the grid (dropped), as TrySolve merges.
    b = (np.concatenate([b[0], b[0][:1], [g.count + 5]]).astype(np.int32),
         np.concatenate([b[1], b[1][:1] - 0.01, [0.0]]))
    return g, s, [a, b]


RAGGED = [(7, 13, 5), (40, 9, 17), (3, 3, 50)]


@pytest.mark.parametrize("dims", RAGGED)
def test_ref_fp64_equals_relax_ragged(dims):
    """Ragged grids, one field per solve: the reference kernel equals Relax to the bit."""
    g, s, sets = _ragged(dims)
    for e, (si, tt) in enumerate(sets):
        got, st, _ = R.eik_solve(g, s, [(si, tt)], 64)
        keep = si < g.count
        want, ok, _ = O.relax(g, s, si[keep], tt[keep])
        assert st == 0 and ok and np.array_equal(got[0], want), f"field {e}"


@pytest.mark.parametrize("dims", RAGGED)
def test_ref_fp64_batch_equals_restated_batch(dims):
    """Two fields in one batch (the node-major layout): the reference's batch shares one round flag,
    which the restated batch (or_relax_batch) reproduces to the bit. Against the per-field settling
    of Relax (and of the CUDA engine) a field can differ by a few ulps, never more than 1e-12."""
    g, s, sets = _ragged(dims)
    got, st, rounds = R.eik_solve(g, s, sets, 64)
    want, ok, wr = O.relax_batch(g, s, sets)
    assert st == 0 and ok and list(rounds) == list(wr)
    assert np.array_equal(got, want)
    for e, (si, tt) in enumerate(sets):
        keep = si < g.count
        solo, _, _ = O.relax(g, s, si[keep], tt[keep])
        rel, _ = _rel(got[e], solo)
        assert rel.max() <= 1e-12, f"field {e}"


def test_ref_fp64_equals_relax_inversion_step_121():
    """121x121x61 at 0.5 km: one P and one S station field in one batch each."""
    p = syn.inversion_step_121()
    g = O.Grid.of(p.grid)
    for ph in (0, 1):
        seeds = O.point_source(g, p.slowness[ph], *p.stations[ph])
        got, st, _ = R.eik_solve(g, p.slowness[ph], [seeds], 64)
        want, ok, _ = O.relax(g, p.slowness[ph], *seeds)
        assert st == 0 and ok and np.array_equal(got[0], want), f"phase {ph}"


def test_ref_refuses_unsettled_like_relax():
    """Sweep refuses a batch that has not settled within the cap (EikonalOpenCl.cs:269)."""
    p = syn.single_source_61()
    g = O.Grid.of(p.grid)
    seeds = O.point_source(g, p.slowness[0], *p.stations[0])
    _, st, rounds = R.eik_solve(g, p.slowness[0], [seeds], 64, cap=1)
    _, ok, _ = O.relax(g, p.slowness[0], *seeds, max_rounds=1)
    assert st == 1 and not ok and rounds[0] == 1


def test_ref_paired_float_error_per_workload():
    """The reference's paired-float kernel (times as hi + lo floats) against the FP64 field: the
    FP32 target, printed per workload (max relative, p99, median, max absolute in seconds)."""
    cases = []
    p0 = syn.single_source_61()
    cases.append(("single_source_61", p0.grid, p0.slowness[0], p0.stations[0]))
    gd, s, src = syn.selftest_case()
    cases.append(("selftest_22x20x16", gd, s, src))
    p1 = syn.inversion_step_121()
    cases.append(("inversion_step_121 S", p1.grid, p1.slowness[1], p1.stations[2]))
    worst = 0.0
    for name, gd, s, src in cases:
        g = O.Grid.of(gd)
        seeds = O.point_source(g, s, *src)
        got, st, _ = R.eik_solve(g, s, [seeds], 32)
        want, ok, _ = O.relax(g, s, *seeds)
        assert st == 0 and ok
        rel, ab = _rel(got[0], want)
        print(f"paired float {name}: max rel {rel.max():.3g}, p99 {np.quantile(rel, 0.99):.3g}, "
              f"median {np.median(rel):.3g}, max abs {ab.max():.3g} s")
        worst = max(worst, rel.max())
    assert worst <= 2e-5


def test_ref_lsqr_products_equal_restatement():
    """spmv (one item per row, sequential sum) on A and on the reference's transpose, and the vector
    update xmby, equal the restated products to the bit; the paired-float product is within 1e-12."""
    rng = np.random.default_rng(17)
    m, n = 700, 300
    counts = rng.integers(0, 40, size=m)
    rp = np.concatenate([[0], np.cumsum(counts)]).astype(np.int32)
    ci = np.concatenate([np.sort(rng.choice(n, size=c, replace=False)) for c in counts]).astype(np.int32)
    va = rng.standard_normal(rp[-1])
    x = rng.standard_normal(n)
    assert np.array_equal(R.spmv(rp, ci, va, x), O.csr_mul(rp, ci, va, x))
    trs, tci, tva = O.csr_transpose(m, n, rp, ci, va)
    u = rng.standard_normal(m)
    assert np.array_equal(R.spmv(trs, tci, tva, u), O.csr_mul(trs, tci, tva, u))
    y = rng.standard_normal(n)
    assert np.array_equal(R.xmby(x, 0.37, y), x - 0.37 * y)
    paired = R.spmv(rp, ci, va, x, precision=32)
    exact = O.csr_mul(rp, ci, va, x)
    scale = np.abs(va)[None, :].max() * np.abs(x).max() * max(1, counts.max())
    assert np.max(np.abs(paired - exact)) <= 1e-12 * scale
