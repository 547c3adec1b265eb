"""ForwardDomain.Covering (host, in the library) against the oracle, and VelocityModel1D's evaluation."""
import numpy as np
import pytest

from oracle import oracle as O
from tomostar_b200 import _lib as L
from tomostar_b200 import domain
from tomostar_b200 import synthetic as syn


def _inv():
    return syn.regular_grid(21, 17, 9, 2.5)


@pytest.mark.parametrize("case", ["inside", "east_deep", "south_west", "coarsened"])
def test_covering_matches_oracle(case):
    inv = _inv()
    lon0, lat0 = inv.min_lon, inv.min_lat
    pts = {"inside": [[lon0 + 0.1, lat0 + 0.1, 3.0], [inv.max_lon, inv.max_lat, 0.0]],
           "east_deep": [[lon0 + 0.1, lat0 + 0.1, 3.0], [inv.max_lon + 0.7, lat0 + 0.2, 35.0]],
           "south_west": [[lon0 - 1.3, lat0 - 0.4, 10.0], [lon0 + 0.2, lat0 + 0.1, -1.0]],
           "coarsened": [[lon0 - 3.0, lat0 - 2.0, 60.0], [inv.max_lon + 3.0, inv.max_lat + 2.0, 5.0]]}[case]
    max_nodes = 200_000 if case == "coarsened" else 12_000_000
    fwd, ext, fac = domain.covering(inv, 2, pts, max_nodes)
    want, ext_o, fac_o = O.covering(O.Grid.of(inv), 2, pts, max_nodes)
    got = (fwd.min_lon, fwd.max_lon, fwd.min_lat, fwd.max_lat, fwd.min_depth_km, fwd.max_depth_km, fwd.nx, fwd.ny,
           fwd.nz)
    assert got == want and ext == ext_o and fac == fac_o
    assert ext == (case != "inside") and (fac > 1) == (case == "coarsened")
    if case == "inside":
        assert (fwd.nx, fwd.ny, fwd.nz) == ((inv.nx - 1) * 2 + 1, (inv.ny - 1) * 2 + 1, (inv.nz - 1) * 2 + 1)
    else:
        assert fwd.count <= max_nodes
        for lon, lat, dep in pts:  # every point inside the covering grid (depths above the top sit on it)
            assert fwd.min_lon <= lon <= fwd.max_lon and fwd.min_lat <= lat <= fwd.max_lat and dep <= fwd.max_depth_km


def test_covering_refuses_the_globe():
    inv = _inv()
    with pytest.raises(L.TsError):
        domain.covering(inv, 2, [[inv.min_lon - 179.6, 0.0, 0.0], [inv.max_lon + 179.6, 10.0, 0.0]])
    with pytest.raises(ValueError):
        O.covering(O.Grid.of(inv), 2, [[inv.min_lon - 179.6, 0.0, 0.0], [inv.max_lon + 179.6, 10.0, 0.0]])


def test_background_model_known_answers():
    """VelocityModel1D (Model/VelocityModel1D.cs:8-45): linear between nodes, the first node's value
    above, the upper value on an interface, the lower just below it, the last node's below the last."""
    d = np.array([0.0, 10.0, 10.0, 30.0])
    v = np.array([5.0, 6.0, 6.5, 8.0])
    assert O.background(d, v, -1.0) == 5.0 and O.background(d, v, 5.0) == 5.5
    assert O.background(d, v, 10.0) == 6.0 and O.background(d, v, 20.0) == 7.25
    assert O.background(d, v, 40.0) == 8.0
    g = _inv()
    vp = 5.0 + np.arange(g.count) % 7 * 0.01
    bg = domain.Background.layer_mean(g, vp, vp / 1.73)
    assert len(bg.depth_km) == g.nz + 1 and bg.depth_km[-1] == 6370.0 and bg.vp[-1] == bg.vp[-2]


def test_covering_across_the_antimeridian():
    """Points east of 180° are unwrapped to the grid's side (GeoMath.UnwrapLon) before the box grows."""
    from tomostar_b200.grid import GridDef

    inv = GridDef(178.5, 179.5, -17.0, -16.0, 0.0, 20.0, 11, 11, 9)
    pts = [[-179.6, -16.5, 5.0], [179.0, -16.2, 3.0]]
    fwd, ext, fac = domain.covering(inv, 2, pts)
    want, ext_o, fac_o = O.covering(O.Grid.of(inv), 2, pts)
    assert (fwd.min_lon, fwd.max_lon, fwd.min_lat, fwd.max_lat, fwd.nx, fwd.ny, fwd.nz) == \
        (want[0], want[1], want[2], want[3], want[6], want[7], want[8])
    assert ext and fwd.max_lon > 180.0 and fwd.min_lon < inv.min_lon  # the margin applies on every side
