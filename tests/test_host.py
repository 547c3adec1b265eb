"""Host-side mirror (grids, synthetic inputs) against the oracle. No GPU."""
import numpy as np

from oracle import oracle as O
from tomostar_b200 import synthetic as syn
from tomostar_b200.grid import GridDef


def test_grid_coordinates_match_oracle():
    g = GridDef.from_spacing(13, 13.74, 43, 43.54, 0, 30, 1, 1)
    assert (g.nx, g.ny, g.nz) == (61, 61, 31)
    lon, lat, cl, dep = O.coords(O.Grid.of(g))
    assert np.allclose(g.lon(), lon, rtol=0, atol=1e-12)
    assert np.allclose(g.lat(), lat, rtol=0, atol=1e-12)
    assert np.allclose(g.depth(), dep, rtol=0, atol=1e-12)
    assert abs(g.min_spacing_km() - O.min_spacing_km(O.Grid.of(g))) < 1e-12


def test_refine_coarsen():
    g = GridDef(10, 11, 42, 43, 0, 30, 16, 11, 7)
    assert g.refined(2).coarsened(2) == g
    f = g.refined(2)
    assert (f.nx, f.ny, f.nz) == (31, 21, 13)


def test_interpolate_and_resample_match_oracle():
    g = GridDef(10, 11, 42, 43, 0, 30, 9, 7, 6)
    rng = np.random.default_rng(3)
    field = rng.uniform(4, 6, g.count)
    og = O.Grid.of(g)
    for pt in [(10.33, 42.71, 11.0), (9.9, 41.5, -3), (11.2, 43.3, 40)]:
        assert abs(g.interpolate(field, *pt) - O.interpolate(og, field, *pt)) < 1e-12
    f = g.refined(2)
    res = f.resample_from(g, field)
    lon, lat, dep = f.lon(), f.lat(), f.depth()
    q = (3 * f.ny + 5) * f.nx + 7
    assert abs(res[q] - O.interpolate(og, field, lon[7], lat[5], dep[3])) < 1e-12


def test_single_source_61_inputs():
    p = syn.single_source_61()
    assert (p.grid.nx, p.grid.ny, p.grid.nz) == (61, 61, 31)
    assert (p.inv.nx, p.inv.ny, p.inv.nz) == (31, 31, 16)
    assert p.slowness.shape == (1, p.grid.count)
    v = 1 / p.slowness[0]
    assert v.min() > 5.0 * 0.94 and v.max() < (5 + 0.03 * 30) * 1.06
    assert p.events.shape == (25, 3) and np.all(p.events[:, 2] == 0)
    # spacing about 1 km
    assert abs(p.grid.min_spacing_km() - 1.0) < 0.01


def test_inversion_step_121_inputs():
    p = syn.inversion_step_121()
    assert (p.grid.nx, p.grid.ny, p.grid.nz) == (121, 121, 61)
    assert p.slowness.shape == (2, p.grid.count)
    assert len(p.stations) == 25 and len(p.events) == 150 and len(p.arrivals) == 7500
    assert np.all((p.events[:, 2] >= 2) & (p.events[:, 2] <= 20))
    assert np.all(p.slowness[1] > p.slowness[0])
