"""Seeded synthetic forward problems of the named workloads (no network: no real data sets).

Every "regular grid at h km" is a spherical GridDefinition anchored at 13.0°E, 43.0°N, depth 0,
as in the reference's known-answer test (tests/TomoStar.Tests/NumericsTests.cs:91): ΔLat = h / (R·π/180),
ΔLon = ΔLat / cos(centre latitude), depth spacing h. Positions given in km from the south-west top
corner map to lon/lat through the grid's own spacing. Checkerboards are the reference's smooth
sine-product pattern (Tomography/ResolutionTests.cs:62-82). Random numbers come from
numpy.random.default_rng with the named seeds.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

from .grid import DEG2RAD, EARTH_RADIUS_KM, GridDef

ANCHOR_LON, ANCHOR_LAT = 13.0, 43.0


def regular_grid(nx: int, ny: int, nz: int, h_km: float, depth_km: np.ndarray | None = None) -> GridDef:
    """A grid of nx×ny×nz nodes at about h km spacing anchored at (13.0°E, 43.0°N, 0 km)."""
    dlat = h_km / (EARTH_RADIUS_KM * DEG2RAD)
    centre_lat = ANCHOR_LAT + 0.5 * (ny - 1) * dlat
    dlon = dlat / math.cos(centre_lat * DEG2RAD)
    max_depth = (nz - 1) * h_km if depth_km is None else float(depth_km[-1])
    min_depth = 0.0 if depth_km is None else float(depth_km[0])
    return GridDef(ANCHOR_LON, ANCHOR_LON + (nx - 1) * dlon, ANCHOR_LAT, ANCHOR_LAT + (ny - 1) * dlat,
                   min_depth, max_depth, nx, ny, nz, depth_km)


def km_to_geo(grid: GridDef, x_km, y_km, h_km: float):
    """(x, y) km from the grid's south-west corner → (lon, lat) through the node spacing."""
    return grid.min_lon + np.asarray(x_km) / h_km * grid.dlon, grid.min_lat + np.asarray(y_km) / h_km * grid.dlat


def surface_distance_km(lon1, lat1, lon2, lat2):
    """GeoMath.SurfaceDistanceKm (Geo/GeoMath.cs:83-95), haversine."""
    p1, p2 = np.asarray(lat1) * DEG2RAD, np.asarray(lat2) * DEG2RAD
    dp = p2 - p1
    dl = (np.asarray(lon2) - np.asarray(lon1)) * DEG2RAD
    a = np.sin(dp / 2) ** 2 + np.cos(p1) * np.cos(p2) * np.sin(dl / 2) ** 2
    return 2 * np.arcsin(np.minimum(1, np.sqrt(a))) * EARTH_RADIUS_KM


def checkerboard(grid: GridDef, cell_h_km: float, cell_v_km: float, amplitude_percent: float) -> np.ndarray:
    """ResolutionPattern.Evaluate, checkerboard branch (ResolutionTests.cs:62-75): fractional
    perturbation at every node, grid order."""
    lon, lat, dep = grid.lon(), grid.lat(), grid.depth()
    L, A = np.meshgrid(lon, lat, indexing="xy")  # (ny, nx)
    x = surface_distance_km(grid.min_lon, A, L, A)
    y = surface_distance_km(L, grid.min_lat, L, A)
    z = dep - grid.min_depth_km
    horiz = np.sin(np.pi * x / cell_h_km) * np.sin(np.pi * y / cell_h_km)
    vert = np.sin(np.pi * (z + 0.5 * cell_v_km) / cell_v_km)
    return (amplitude_percent / 100 * vert[:, None, None] * horiz[None, :, :]).reshape(-1)


@dataclass
class Problem:
    """A forward problem: grid, slowness per phase, stations (field origins) and events."""

    name: str
    grid: GridDef                      # forward grid
    inv: GridDef                       # inversion grid (forward coarsened ×2)
    slowness: np.ndarray               # (n_phases, n) s/km
    stations: np.ndarray               # (n_stations, 3) lon, lat, depth
    events: np.ndarray                 # (n_events, 3)
    arrivals: np.ndarray = field(default_factory=lambda: np.zeros((0, 3), np.int32))  # (event, station, phase)
    h_km: float = 1.0

    @property
    def step_km(self) -> float:
        """RayKernels step (Tomography/RayKernels.cs:62)."""
        return 0.5 * min(self.grid.min_spacing_km(), self.inv.min_spacing_km())


def vp_linear(grid: GridDef, v0: float = 5.0, grad: float = 0.03) -> np.ndarray:
    dep = grid.depth()
    return np.broadcast_to((v0 + grad * dep)[:, None, None], grid.shape).reshape(-1).copy()


def single_source_61() -> Problem:
    """61×61×31 at 1 km; Vp = (5 + 0.03 z)·(1 ± 5 % checkerboard of 10 km); source (30, 30, 10) km;
    25 receivers uniformly at random on the surface (seed 0). FP64, compared with the CPU solver."""
    h = 1.0
    g = regular_grid(61, 61, 31, h)
    vp = vp_linear(g) * (1 + checkerboard(g, 10, 10, 5))
    slon, slat = km_to_geo(g, 30.0, 30.0, h)
    rng = np.random.default_rng(0)
    xy = rng.uniform(0, 60, size=(25, 2))
    rlon, rlat = km_to_geo(g, xy[:, 0], xy[:, 1], h)
    events = np.stack([rlon, rlat, np.zeros(25)], axis=1)
    arrivals = np.stack([np.arange(25), np.zeros(25, int), np.zeros(25, int)], axis=1).astype(np.int32)
    return Problem("single_source_61", g, g.coarsened(2), (1 / vp)[None, :], np.array([[slon, slat, 10.0]]), events,
                   arrivals, h)


def inversion_step_121() -> Problem:
    """121×121×61 at 0.5 km; Vp as the 61×61×31 model; Vp/Vs = 1.73·(1 ± 3 % checkerboard of 10 km); 25 surface
    stations (seed 1), 150 events in the box at 2–20 km depth (seed 2); P and S: 50 fields, 7,500 rays."""
    h = 0.5
    g = regular_grid(121, 121, 61, h)
    vp = vp_linear(g) * (1 + checkerboard(g, 10, 10, 5))
    vs = vp / (1.73 * (1 + checkerboard(g, 10, 10, 3)))
    span = 120 * h
    r1 = np.random.default_rng(1)
    sxy = r1.uniform(0, span, size=(25, 2))
    slon, slat = km_to_geo(g, sxy[:, 0], sxy[:, 1], h)
    stations = np.stack([slon, slat, np.zeros(25)], axis=1)
    r2 = np.random.default_rng(2)
    exyz = np.column_stack([r2.uniform(0, span, 150), r2.uniform(0, span, 150), r2.uniform(2, 20, 150)])
    elon, elat = km_to_geo(g, exyz[:, 0], exyz[:, 1], h)
    events = np.stack([elon, elat, exyz[:, 2]], axis=1)
    ev, st, ph = np.meshgrid(np.arange(150), np.arange(25), np.arange(2), indexing="ij")
    arrivals = np.stack([ev.ravel(), st.ravel(), ph.ravel()], axis=1).astype(np.int32)
    return Problem("inversion_step_121", g, g.coarsened(2), np.stack([1 / vp, 1 / vs]), stations, events, arrivals, h)


def selftest_case():
    """The reference's device self-test case (Forward/EikonalOpenCl.cs:348-358)."""
    g = GridDef(10, 12, 42, 44, -2, 120, 22, 20, 16)
    dep = g.depth()
    i = np.arange(g.nx)[None, None, :]
    j = np.arange(g.ny)[None, :, None]
    s = 1 / (5.8 + 0.02 * dep[:, None, None] + 0.2 * np.sin(0.7 * i) + 0.15 * np.cos(0.5 * j))
    return g, s.reshape(-1), (10.37, 42.61, 8.3)


def ellipsoid_bodies(grid: GridDef, h_km: float, rng, n: int = 3, amplitude: float = 0.08) -> np.ndarray:
    """Fractional perturbation of n ellipsoidal bodies with smooth edges (the super-Gaussian edge of
    the reference's TabularBody, ResolutionTests.cs:39-40: 1 inside, 1/2 at the nominal surface).
    Amplitudes alternate +amplitude, −amplitude, …; centres and semi-axes are drawn from rng."""
    nx, ny, nz = grid.nx, grid.ny, grid.nz
    x = np.arange(nx) * h_km
    y = np.arange(ny) * h_km
    z = grid.depth()
    span_x, span_y, span_z = x[-1], y[-1], z[-1]
    out = np.zeros((nz, ny, nx))
    for b in range(n):
        cx, cy = rng.uniform(0.2, 0.8) * span_x, rng.uniform(0.2, 0.8) * span_y
        cz = rng.uniform(0.2, 0.8) * span_z
        ax, ay = rng.uniform(0.08, 0.2) * span_x, rng.uniform(0.08, 0.2) * span_y
        az = rng.uniform(0.1, 0.3) * span_z
        amp = amplitude if b % 2 == 0 else -amplitude
        r2 = (((z - cz) / az) ** 2)[:, None, None] + (((y - cy) / ay) ** 2)[None, :, None] + \
            (((x - cx) / ax) ** 2)[None, None, :]
        out += amp * np.exp(-np.log(2) * r2 ** 3)
    return out.reshape(-1)


def regional_401(n_stations: int = 400, n_events: int = 5000, n_rays: int = 1_500_000, seed: int = 5,
                 dims: tuple = (401, 401, 121)) -> Problem:
    """401×401×121 at 0.25 km (19.46 M nodes): Vp = 5 + 0.04 z km/s plus three ellipsoidal ±8 % bodies,
    Vs = Vp / 1.73; 400 surface stations and 5,000 events (2–25 km deep) → 800 P and S fields;
    1.5 M (event, station, phase) arrivals drawn uniformly without replacement. One generator,
    seed 5, in that order. `dims` other than 401×401×121 gives the same model law on a smaller
    grid (profiling captures that must stay a few GB on the device); events stay within its depth.
    The grid stays square in x and y (stations and events are drawn over one span)."""
    assert dims[0] == dims[1], "regional grids are square in x and y"
    h = 0.25
    g = regular_grid(*dims, h)
    rng = np.random.default_rng(seed)
    vp = vp_linear(g, 5.0, 0.04) * (1 + ellipsoid_bodies(g, h, rng))
    vs = vp / 1.73
    span = (dims[0] - 1) * h
    sxy = rng.uniform(0, span, size=(n_stations, 2))
    slon, slat = km_to_geo(g, sxy[:, 0], sxy[:, 1], h)
    stations = np.stack([slon, slat, np.zeros(n_stations)], axis=1)
    exyz = np.column_stack([rng.uniform(0, span, n_events), rng.uniform(0, span, n_events),
                            rng.uniform(2, min(25.0, (dims[2] - 1) * h), n_events)])
    elon, elat = km_to_geo(g, exyz[:, 0], exyz[:, 1], h)
    events = np.stack([elon, elat, exyz[:, 2]], axis=1)
    pick = rng.choice(n_events * n_stations * 2, size=min(n_rays, n_events * n_stations * 2), replace=False)
    ev, rest = np.divmod(pick, n_stations * 2)
    st, ph = np.divmod(rest, 2)
    arrivals = np.stack([ev, st, ph], axis=1).astype(np.int32)
    slow = np.empty((2, g.count))
    np.divide(1.0, vp, out=slow[0])
    np.divide(1.0, vs, out=slow[1])
    return Problem("regional_401", g, g.coarsened(2), slow, stations, events, arrivals, h)


@dataclass
class GridBatch:
    """Sources each on its own grid: grids[q] with slowness[q] (grid order) and source q."""

    name: str
    grids: list
    slowness: list
    sources: np.ndarray      # (n, 3) lon, lat, depth km
    h_km: np.ndarray         # horizontal spacing of each grid


def smooth3(a: np.ndarray) -> np.ndarray:
    """Mean over the 3 nearest cells along each axis in turn (edges repeat the end cell)."""
    for ax in range(a.ndim):
        p = np.pad(a, [(1, 1) if d == ax else (0, 0) for d in range(a.ndim)], mode="edge")
        sl = lambda lo, hi: tuple(slice(lo, hi) if d == ax else slice(None) for d in range(a.ndim))
        a = (p[sl(0, -2)] + p[sl(1, -1)] + p[sl(2, None)]) / 3.0
    return a


def uneven_grids(n_sources: int = 200, seed: int = 3, variable_share: float = 0.5,
            dims_scale: float = 1.0) -> GridBatch:
    """200 sources, each on its own grid: nx, ny uniform in 48–192, nz in 32–96, spacing h uniform in
    0.25–1 km. Half the grids (a coin per grid) have depth levels whose spacing grows geometrically
    by a ratio r uniform in 1.02–1.05 over the same depth extent (nz−1)·h. Vp = 5.0 + 0.03·depth km/s
    times a lognormal cell factor exp(N(0, 0.04)) smoothed over 3 cells on every axis. One source
    per grid, horizontally in the middle 80 % and at a depth in the upper half. One generator,
    seed 3, drawn in that order grid by grid. dims_scale < 1 shrinks every dimension (test sizes)."""
    rng = np.random.default_rng(seed)
    grids, slow, src, hs = [], [], [], []
    for _ in range(n_sources):
        nx = int(rng.integers(48, 193))
        ny = int(rng.integers(48, 193))
        nz = int(rng.integers(32, 97))
        h = float(rng.uniform(0.25, 1.0))
        variable = bool(rng.uniform() < variable_share)
        r = float(rng.uniform(1.02, 1.05))
        if dims_scale != 1.0:
            nx, ny, nz = (max(4, int(round(v * dims_scale))) for v in (nx, ny, nz))
        depth = None
        if variable:
            steps = r ** np.arange(nz - 1)
            depth = np.concatenate([[0.0], np.cumsum(steps)]) * ((nz - 1) * h / steps.sum())
            depth[-1] = (nz - 1) * h
        g = regular_grid(nx, ny, nz, h, depth)
        z = g.depth()
        pert = np.exp(rng.normal(0.0, 0.04, size=g.shape))
        vp = (5.0 + 0.03 * z)[:, None, None] * smooth3(pert)
        fx, fy, fz = rng.uniform(0.1, 0.9), rng.uniform(0.1, 0.9), rng.uniform(0.0, 0.5)
        lon = g.min_lon + fx * (g.max_lon - g.min_lon)
        lat = g.min_lat + fy * (g.max_lat - g.min_lat)
        grids.append(g)
        slow.append((1.0 / vp).reshape(-1))
        src.append((lon, lat, fz * g.max_depth_km))
        hs.append(h)
    return GridBatch("uneven_grids", grids, slow, np.asarray(src), np.asarray(hs))


@dataclass
class ServeModel:
    """A resident model of the serving load: grid, slowness (phases, n) and node spacing."""

    name: str
    grid: GridDef
    slowness: np.ndarray
    h_km: float


@dataclass
class ServeRequestSpec:
    """One request of the serving load: arrival time (s), kind, model, phase, the stations its
    fields are seeded at (n_fields, 3) and its rays: events (n_rays, 3) and the field of each."""

    t: float
    kind: str
    model: str
    phase: int
    stations: np.ndarray
    events: np.ndarray
    ray_field: np.ndarray


def _surface_points(g: GridDef, h: float, n: int, rng) -> np.ndarray:
    span_x, span_y = (g.nx - 1) * h, (g.ny - 1) * h
    xy = rng.uniform(0, 1, size=(n, 2)) * [span_x, span_y]
    lon, lat = km_to_geo(g, xy[:, 0], xy[:, 1], h)
    return np.stack([lon, lat, np.zeros(n)], axis=1)


def _volume_points(g: GridDef, h: float, n: int, zmin: float, zmax: float, rng) -> np.ndarray:
    span_x, span_y = (g.nx - 1) * h, (g.ny - 1) * h
    x, y, z = rng.uniform(0, span_x, n), rng.uniform(0, span_y, n), rng.uniform(zmin, zmax, n)
    lon, lat = km_to_geo(g, x, y, h)
    return np.stack([lon, lat, z], axis=1)


def spikes(grid: GridDef, h_km: float, cell_km: float, amplitude_percent: float, n: int, rng) -> np.ndarray:
    """Spike-test perturbation (ResolutionTests.cs:62-82 spike branch in spirit): n isolated cubes
    of cell_km at random cell positions, alternately +/− amplitude, fractional, grid order."""
    x = np.arange(grid.nx) * h_km
    y = np.arange(grid.ny) * h_km
    z = grid.depth() - grid.min_depth_km
    out = np.zeros(grid.shape)
    for q in range(n):
        cx, cy, cz = (rng.integers(0, max(1, int(v // cell_km))) * cell_km for v in (x[-1], y[-1], z[-1]))
        sign = 1 if q % 2 == 0 else -1
        mz = (z >= cz) & (z < cz + cell_km)
        my = (y >= cy) & (y < cy + cell_km)
        mx = (x >= cx) & (x < cx + cell_km)
        out[np.ix_(mz, my, mx)] = sign * amplitude_percent / 100
    return out.reshape(-1)


def serving_models() -> dict:
    """Resident models of the serving load: the 121×121×61 forward model of the inversion step
    (the 121×121×61 inversion-step model, P and S); two 81×81×41 resolution-test models at 1 km (Vp(z) times a ±5 %
    checkerboard and ±5 % spikes of 8 km cells); a 161×161×81 relocation model at 0.5 km (Vp(z),
    Vs = Vp/1.73)."""
    p1 = inversion_step_121()
    models = {"forward121": ServeModel("forward121", p1.grid, p1.slowness, 0.5)}
    g81 = regular_grid(81, 81, 41, 1.0)
    v81 = vp_linear(g81)
    models["checker81"] = ServeModel("checker81", g81, (1 / (v81 * (1 + checkerboard(g81, 8, 8, 5))))[None, :], 1.0)
    rng = np.random.default_rng(4)
    models["spike81"] = ServeModel("spike81", g81, (1 / (v81 * (1 + spikes(g81, 1.0, 8, 5, 12, rng))))[None, :], 1.0)
    g161 = regular_grid(161, 161, 81, 0.5)
    v161 = vp_linear(g161)
    models["reloc161"] = ServeModel("reloc161", g161, np.stack([1 / v161, 1.73 / v161]), 0.5)
    return models


def serving_stream(models: dict, rate: float = 200.0, duration: float = 60.0, seed: int = 4) -> list:
    """The serving load: Poisson arrivals at `rate` per second for `duration` seconds, mixed 60 %
    single-station eikonal-plus-rays requests on forward121 (P or S, 20–150 rays from events at
    2–20 km), 25 % resolution-test batches of 25 fields on checker81 or spike81 (no rays), 15 %
    relocation requests on reloc161 (one station field, 10–40 rays from events at 2–25 km). One
    generator, stream seed 4."""
    rng = np.random.default_rng(seed)
    out, t = [], 0.0
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= duration:
            break
        u = rng.uniform()
        if u < 0.60:
            m = models["forward121"]
            nr = int(rng.integers(20, 151))
            out.append(ServeRequestSpec(t, "eikonal+rays", m.name, int(rng.integers(0, 2)),
                                        _surface_points(m.grid, m.h_km, 1, rng),
                                        _volume_points(m.grid, m.h_km, nr, 2, 20, rng), np.zeros(nr, np.int32)))
        elif u < 0.85:
            m = models["checker81" if rng.uniform() < 0.5 else "spike81"]
            out.append(ServeRequestSpec(t, "resolution", m.name, 0, _surface_points(m.grid, m.h_km, 25, rng),
                                        np.zeros((0, 3)), np.zeros(0, np.int32)))
        else:
            m = models["reloc161"]
            nr = int(rng.integers(10, 41))
            out.append(ServeRequestSpec(t, "relocation", m.name, int(rng.integers(0, 2)),
                                        _surface_points(m.grid, m.h_km, 1, rng),
                                        _volume_points(m.grid, m.h_km, nr, 2, 25, rng), np.zeros(nr, np.int32)))
    return out


@dataclass
class RelocationJob:
    """Events to locate on the tables of their stations (Relocation.Absolute, Location/Relocation.cs:48-97).

    Table t is station t % n_stations for phase t // n_stations (0 P, 1 S). truth holds each event's
    lon, lat, depth and origin time in s after its catalogue origin time; start is the catalogue
    location the search starts from."""

    name: str
    grid: GridDef
    slowness: np.ndarray       # (2, n) s/km, P then S
    stations: np.ndarray       # (n_stations, 3) lon, lat, depth
    truth: np.ndarray          # (n_events, 4)
    start: np.ndarray          # (n_events, 3)
    h_km: float

    @property
    def table_source(self) -> np.ndarray:
        return np.concatenate([self.stations, self.stations])

    @property
    def table_phase(self) -> np.ndarray:
        return np.repeat(np.arange(2, dtype=np.int32), len(self.stations))


def _relocation_job(name: str, g: GridDef, h: float, n_stations: int, n_events: int, rng) -> RelocationJob:
    vp = vp_linear(g, 5.0, 0.04) * (1 + ellipsoid_bodies(g, h, rng, n=2, amplitude=0.05))
    slow = np.empty((2, g.count))
    np.divide(1.0, vp, out=slow[0])
    np.divide(1.73, vp, out=slow[1])
    span_x, span_y = (g.nx - 1) * h, (g.ny - 1) * h
    sx, sy = rng.uniform(0.05 * span_x, 0.95 * span_x, n_stations), rng.uniform(0.05 * span_y, 0.95 * span_y, n_stations)
    slon, slat = km_to_geo(g, sx, sy, h)
    stations = np.stack([slon, slat, np.zeros(n_stations)], axis=1)
    bottom = g.max_depth_km
    ex = rng.uniform(0.15 * span_x, 0.85 * span_x, n_events)
    ey = rng.uniform(0.15 * span_y, 0.85 * span_y, n_events)
    ez = rng.uniform(0.15 * bottom, 0.75 * bottom, n_events)
    elon, elat = km_to_geo(g, ex, ey, h)
    truth = np.stack([elon, elat, ez, rng.uniform(-1.0, 1.0, n_events)], axis=1)
    # The catalogue locations: a few km off horizontally, off in depth, inside the grid.
    qx = np.clip(ex + rng.normal(0, 3.0, n_events), 0, span_x)
    qy = np.clip(ey + rng.normal(0, 3.0, n_events), 0, span_y)
    qz = np.clip(ez + rng.normal(0, 2.0, n_events), 0, bottom)
    qlon, qlat = km_to_geo(g, qx, qy, h)
    start = np.stack([qlon, qlat, qz], axis=1)
    return RelocationJob(name, g, slow, stations, truth, start, h)


def relocation_small(seed: int = 99) -> RelocationJob:
    """The reference's pipeline test set-up (tests/TomoStar.Tests/PipelineTests.cs:23-30, 95-107): 12
    stations, 30 events, a 5 km inversion grid down to 20 km refined twice for the tables: 21×21×17
    nodes at 2.5 km horizontally and 1.25 km vertically."""
    g0 = regular_grid(21, 21, 17, 2.5)
    g = GridDef(g0.min_lon, g0.max_lon, g0.min_lat, g0.max_lat, 0.0, 20.0, 21, 21, 17)
    return _relocation_job("relocation_small", g, 2.5, 12, 30, np.random.default_rng(seed))


def relocation_regional(n_stations: int = 60, n_events: int = 4000, seed: int = 8) -> RelocationJob:
    """A regional relocation: the 161×161×81 model at 0.5 km (2.1 M nodes), 60 surface stations (120 P
    and S tables, 1.0 GB of float32), 4,000 events 6–30 km deep."""
    g = regular_grid(161, 161, 81, 0.5)
    return _relocation_job("relocation_regional", g, 0.5, n_stations, n_events, np.random.default_rng(seed))


def table_time(g: GridDef, table: np.ndarray, lon, lat, dep) -> np.ndarray:
    """TravelTimeTable.Time (Forward/TravelTimeTable.cs:116-136) on a uniform grid for arrays of points:
    trilinear on the float32 nodes, +inf when a weighted corner is not finite."""
    lon, lat, dep = (np.atleast_1d(np.asarray(a, np.float64)) for a in (lon, lat, dep))
    fx = np.clip((lon - g.min_lon) / g.dlon, 0, g.nx - 1)
    fy = np.clip((lat - g.min_lat) / g.dlat, 0, g.ny - 1)
    fz = np.clip((dep - g.min_depth_km) / g.ddepth, 0, g.nz - 1)
    i0 = np.minimum(fx.astype(np.int64), g.nx - 2)
    j0 = np.minimum(fy.astype(np.int64), g.ny - 2)
    k0 = np.minimum(fz.astype(np.int64), g.nz - 2)
    tx, ty, tz = fx - i0, fy - j0, fz - k0
    t = np.zeros(len(lon))
    bad = np.zeros(len(lon), bool)
    for dk in (0, 1):
        for dj in (0, 1):
            for di in (0, 1):
                w = (tx if di else 1 - tx) * (ty if dj else 1 - ty) * (tz if dk else 1 - tz)
                v = table[((k0 + dk) * g.ny + j0 + dj) * g.nx + i0 + di].astype(np.float64)
                use = w != 0
                bad |= use & ~np.isfinite(v)
                t += np.where(use & np.isfinite(v), v * w, 0.0)
    return np.where(bad, np.inf, t)


@dataclass
class Picks:
    """The observations of every event, event after event (obs_offsets[e] .. obs_offsets[e+1])."""

    offsets: np.ndarray      # (n_events + 1,) int32
    table: np.ndarray        # int32
    seconds: np.ndarray      # pick time, s after the catalogue origin time
    weight: np.ndarray
    correction: np.ndarray   # station correction, s


def relocation_picks(job: RelocationJob, tables: np.ndarray, pick_share: float = 0.8, noise_s: float = 0.03,
                     outlier_share: float = 0.03, seed: int = 12) -> Picks:
    """Picks of P and S at a share of the stations: the travel time at the true hypocentre from the
    tables, the station correction, 30 ms of noise, a few gross errors of 1–3 s, and the weights of
    four quality classes (1, 0.75, 0.5, 0.25)."""
    rng = np.random.default_rng(seed)
    n_ev, n_st = len(job.truth), len(job.stations)
    nt = 2 * n_st
    corr = rng.normal(0, 0.05, nt)
    tt = np.stack([table_time(job.grid, tables[t], job.truth[:, 0], job.truth[:, 1], job.truth[:, 2])
                   for t in range(nt)], axis=1)                    # (n_events, n_tables)
    take = (rng.random((n_ev, nt)) < pick_share) & np.isfinite(tt)
    noise = rng.normal(0, noise_s, (n_ev, nt))
    gross = np.where(rng.random((n_ev, nt)) < outlier_share, rng.uniform(1.0, 3.0, (n_ev, nt)), 0.0)
    quality = rng.choice(np.array([1.0, 0.75, 0.5, 0.25]), size=(n_ev, nt), p=[0.5, 0.25, 0.15, 0.1])
    obs = job.truth[:, 3:4] + tt + corr[None, :] + noise + gross
    counts = take.sum(axis=1)
    offsets = np.zeros(n_ev + 1, np.int32)
    offsets[1:] = np.cumsum(counts)
    ev, tb = np.nonzero(take)
    return Picks(offsets, tb.astype(np.int32), obs[ev, tb], quality[ev, tb], corr[tb])
