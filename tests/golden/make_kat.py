"""Writes the known-answer fixtures of the forward path (run: python tests/golden/make_kat.py).

The reference checks in no golden arrays for this path (validation/results hold summary metrics
only), so the fixtures are its known-answer tests restated with their closed-form answers,
computed here with numpy alone — independently of the oracle under test:

  homogeneous_corners  tests/TomoStar.Tests/NumericsTests.cs:88-104 — 6 km/s, FromSpacing grid,
                       source (13.37, 43.27, 10): exact time = distance / 6 at four corner nodes.
  gradient_model       validation/TomoStar.Validation/Program.cs:107-132 — v = 4 + 0.05 z,
                       T = arccosh(1 + b² r² / (2 v1 v2)) / b at nodes r >= 3 km on four levels.
  trilinear            NumericsTests.cs:107-123 — weights of (10.37, 40.61, 7.3) sum to 1 and
                       interpolate 2·lon − lat + 0.1·depth exactly.
"""
import json
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
R = 6371.0
D2R = math.pi / 180.0


def cart(lon, lat, dep):
    r = R - dep
    la, lo = lat * D2R, lon * D2R
    return np.array([r * math.cos(la) * math.cos(lo), r * math.cos(la) * math.sin(lo), r * math.sin(la)])


def from_spacing(min_lon, max_lon, min_lat, max_lat, min_d, max_d, hk, vk):
    mid = 0.5 * (min_lat + max_lat) * D2R
    w = (max_lon - min_lon) * D2R * R * math.cos(mid)
    h = (max_lat - min_lat) * D2R * R
    rnd = lambda v: int(np.round(v))
    return dict(min_lon=min_lon, max_lon=max_lon, min_lat=min_lat, max_lat=max_lat, min_depth_km=min_d,
                max_depth_km=max_d, nx=max(2, rnd(w / hk) + 1), ny=max(2, rnd(h / hk) + 1),
                nz=max(2, rnd((max_d - min_d) / vk) + 1))


def node(g, i, j, k):
    lon = g["min_lon"] + i * (g["max_lon"] - g["min_lon"]) / (g["nx"] - 1)
    lat = g["min_lat"] + j * (g["max_lat"] - g["min_lat"]) / (g["ny"] - 1)
    dep = g["min_depth_km"] + k * (g["max_depth_km"] - g["min_depth_km"]) / (g["nz"] - 1)
    return lon, lat, dep


def main():
    out = {}
    g = from_spacing(13, 13.74, 43, 43.54, 0, 30, 1, 1)
    src = cart(13.37, 43.27, 10)
    nx, ny, nz = g["nx"], g["ny"], g["nz"]
    corners = [(0, 0, 0), (nx - 1, ny - 1, 0), (nx - 1, 0, nz - 1), (nx // 2, ny - 1, nz // 2)]
    out["homogeneous_corners"] = dict(
        grid=g, velocity=6.0, source=[13.37, 43.27, 10.0], tolerance=0.01, source_ref="NumericsTests.cs:88-104",
        nodes=[list(c) for c in corners],
        exact=[float(np.linalg.norm(cart(*node(g, *c)) - src) / 6.0) for c in corners])

    g2 = dict(min_lon=13.0, max_lon=13.8, min_lat=42.5, max_lat=43.1, min_depth_km=0.0, max_depth_km=40.0,
              nx=161, ny=121, nz=81)
    lon0, lat0, z0 = 13.4, 42.8, 15.0
    src2 = cart(lon0, lat0, z0)
    b = 0.05
    rows = []
    for z in (0.0, 5.0, 20.0, 30.0):
        k = int(round((z - g2["min_depth_km"]) / 0.5))
        for j in range(0, g2["ny"], 8):
            for i in range(0, g2["nx"], 8):
                lon, lat, dep = node(g2, i, j, k)
                r = float(np.linalg.norm(cart(lon, lat, dep) - src2))
                if r < 3:
                    continue
                v1, v2 = 4 + 0.05 * z0, 4 + 0.05 * dep
                rows.append([i, j, k, r, math.acosh(1 + b * b * r * r / (2 * v1 * v2)) / b])
    out["gradient_model"] = dict(grid=g2, v0=4.0, gradient=0.05, source=[lon0, lat0, z0], tolerance=0.05,
                                 source_ref="validation/TomoStar.Validation/Program.cs:107-132; common.py threshold",
                                 columns=["i", "j", "k", "distance_km", "exact_s"], rows=rows)

    g3 = dict(min_lon=10, max_lon=11, min_lat=40, max_lat=41, min_depth_km=0, max_depth_km=20, nx=5, ny=6, nz=7)
    out["trilinear"] = dict(grid=g3, point=[10.37, 40.61, 7.3], weight_sum=1.0,
                            linear_value=2 * 10.37 - 40.61 + 0.73, source_ref="NumericsTests.cs:107-123")
    with open(os.path.join(HERE, "kat.json"), "w") as f:
        json.dump(out, f, indent=1)


if __name__ == "__main__":
    main()
