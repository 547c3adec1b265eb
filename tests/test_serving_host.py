"""Host side of the serving engine: the C structs match their ctypes mirrors (sizes and offsets, from
a C compile of the header), and the serving load generator has the named mix and rate."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from tomostar_b200 import _lib as L
from tomostar_b200 import synthetic as syn

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {
    "ts_grid": (L.GridStruct, ["nx", "depth_km"]),
    "ts_eik_stats": (L.EikStats, ["node_updates", "kernel_ms"]),
    "ts_serve_request": (L.ServeRequest, ["n_rays", "seed_offsets", "inv", "step_km", "tables_out"]),
    "ts_serve_result": (L.ServeResult, ["queue_ms", "rows", "error"]),
    "ts_serve_stats_t": (L.ServeStats, ["device_ms", "complete_ms", "queued", "in_flight"]),
    "ts_lsqr_info": (L.LsqrInfo, [f for f, _ in L.LsqrInfo._fields_]),
    "ts_locator_settings": (L.LocatorSettings, [f for f, _ in L.LocatorSettings._fields_]),
    "ts_location": (L.Location, [f for f, _ in L.Location._fields_]),
    "ts_locate_stats": (L.LocateStats, [f for f, _ in L.LocateStats._fields_]),
}


def test_struct_layouts_match_the_header(tmp_path):
    src = ['#include <stdio.h>', '#include <stddef.h>', '#include "tomostar_cuda.h"', "int main(void) {"]
    for cname, (_, fields) in STRUCTS.items():
        src.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f in fields:
            src.append(f'printf("{cname} {f} %zu\\n", offsetof({cname}, {f}));')
    src.append("return 0; }")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), str(c), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    got = {}
    for line in out:
        if line:
            name, key, val = line.split()
            got[(name, key)] = int(val)
    for cname, (cls, fields) in STRUCTS.items():
        assert got[(cname, "size")] == C.sizeof(cls), cname
        for f in fields:
            assert got[(cname, f)] == getattr(cls, f).offset, (cname, f)


def test_serving_load_mix_and_rate():
    models = syn.serving_models()
    stream = syn.serving_stream(models, rate=200, duration=60, seed=4)
    n = len(stream)
    assert abs(n - 12000) < 4 * np.sqrt(12000)
    kinds = np.array([r.kind for r in stream])
    for kind, share in (("eikonal+rays", 0.60), ("resolution", 0.25), ("relocation", 0.15)):
        assert abs(np.mean(kinds == kind) - share) < 0.02
    t = np.array([r.t for r in stream])
    assert np.all(np.diff(t) > 0) and t[-1] < 60
    res = [r for r in stream if r.kind == "resolution"]
    assert all(len(r.stations) == 25 and len(r.events) == 0 for r in res)
    rel = [r for r in stream if r.kind == "relocation"]
    assert all(10 <= len(r.events) <= 40 for r in rel)
    eik = [r for r in stream if r.kind == "eikonal+rays"]
    assert all(20 <= len(r.events) <= 150 and r.model == "forward121" for r in eik)
    # Deterministic from the stream seed.
    again = syn.serving_stream(models, rate=200, duration=60, seed=4)
    assert np.allclose([r.t for r in again[:50]], t[:50])
    assert models["forward121"].grid.shape == (61, 121, 121)
    assert models["reloc161"].grid.count == 161 * 161 * 81
