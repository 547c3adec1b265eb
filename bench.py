"""Benchmark of the forward engine: travel-time fields/s on the large regional forward step
(401×401×121 nodes at 0.25 km, 400 stations × P and S = 800 fields), FP64 sweeping, float32 tables.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = every field of the job solved once by the batched engine (two launches: the P and the
S fields). `value` is fields/s with the velocity model resident in HBM and the fields left on the
device; `e2e` is the same job through the C-ABI entry point a host calls (ts_eik_solve: slowness and
seeds from host memory, float32 tables read back into pinned host memory). Under torchrun the N
ranks split one job of 400·N stations by station (station i on rank i % N, as the reference's MPI
session does; 800 fields per rank: weak scaling, no collective on the data path); rank 0 prints one
JSON line with the max-over-ranks time. At N = 1 the line also carries the
serving load (`serving`: Poisson arrivals at 200 requests/s of mixed eikonal, ray and resolution
requests on three grid sizes, p50/p99 latency and fields/s). `--impl reference` times the
reference's CPU solver (fast marching, restated in oracle/) on the host cores on a bounded sample of
the job. Fields are computed in FP64 (fast mode: within 1e-10 relative of the reference's sweeping)
and delivered as float32 tables (the .qttb rounding, within 6e-8 relative).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "travel-time fields/s + p99 solve latency, batched vs plain GPU, err\u22642e-5 rel"
UNIT = "fields/s"
FALLBACK_HBM_GBS = 6650.0


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.out = os.path.join(tempfile.gettempdir(), f"tomostar_clocks_{os.getpid()}.csv")

    def start(self):
        try:
            os.makedirs(os.path.dirname(self.out), exist_ok=True)
            self.f = open(self.out, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.out):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def setup_dist(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist_mod

        torch.cuda.set_device(local)
        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                    device_id=torch.device("cuda", local))
        dist = dist_mod
    return world, rank, local, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(dist, local, x: float) -> float:
    """The largest x over the ranks (a device tensor over NCCL, a host one over gloo)."""
    if dist is None:
        return x
    import torch

    dev = f"cuda:{local}" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_problem(world: int, dims=(401, 401, 121)):
    """The regional job for `world` GPUs: 400 surface stations per GPU on one model (seed 5), so that
    each GPU's share is the size of the 1-GPU job (weak scaling). `dims` smaller than 401x401x121 is
    only for profiling captures that must stay small."""
    from tomostar_b200 import synthetic as syn

    return syn.regional_401(n_stations=400 * world, dims=dims)


def rank_stations(problem, rank: int, world: int):
    """The stations rank `rank` solves: station i goes to rank i % world (Compute/MpiSession.cs:97), so
    the ranks split one job by station with no collective on the data path."""
    from tomostar_b200 import shard

    return problem.stations[shard.station_share(len(problem.stations), rank, world)]


def job_throughput(dist, local, world: int, fields_per_rank_step: int, steps: int, dev_ms: float):
    """Whole-job fields/s: every rank's fields over the slowest rank's device time."""
    dev_max = max_over_ranks(dist, local, dev_ms)
    return fields_per_rank_step * world * steps / (dev_max / 1e3), dev_max


def cpu_fmm_sample(problem, n_fields: int, threads: int):
    """The reference's CPU path (SphericalEikonal.Solve, one field per thread as TravelTimeTableSet
    does) on n_fields fields of the job; returns (fields/s, seconds)."""
    from oracle import oracle as O

    og = O.Grid.of(problem.grid)
    seeds, sl_of = [], []
    for q in range(n_fields):
        st, ph = q // 2, q % 2
        seeds.append(O.point_source(og, problem.slowness[ph], *problem.stations[st]))
        sl_of.append(ph)
    t0 = time.perf_counter()
    O.fmm_many(og, problem.slowness, np.array(sl_of, np.int32), seeds, threads=threads)
    dt = time.perf_counter() - t0
    return n_fields / dt, dt


def location_job(device: int, n_events: int, cpu_events: int, threads: int) -> dict:
    """Relocation of a regional catalogue on resident tables (Relocation.Absolute): the 120 P and S
    tables of 60 stations on the 161x161x81 model built by the engine and kept on the device, then
    EventLocator.Locate for every event in one call; the oracle locates a bounded sample of the same
    events on the host cores (the CPU baseline), whose results are compared with the device's."""
    from oracle import oracle as O
    from tomostar_b200 import location as loc
    from tomostar_b200 import synthetic as syn
    from tomostar_b200.eikonal import EikonalCuda

    job = syn.relocation_regional(n_events=n_events)
    with EikonalCuda.create(device, 64) as s:
        t0 = time.perf_counter()
        tables = loc.Tables.build(s, job.grid, job.slowness, job.table_source, job.table_phase)
        build_s = time.perf_counter() - t0
        tabs = tables.copy()
        picks = syn.relocation_picks(job, tabs)
        tsta = job.table_source[:, :2]

        def sub(k):
            o = picks.offsets[: k + 1]
            e = o[-1]
            return (job.start[:k], o, picks.table[:e], picks.seconds[:e], picks.weight[:e], picks.correction[:e])

        loc.locate(s, tables, *sub(min(64, n_events)), tsta)  # warm-up
        t1 = time.perf_counter()
        r = loc.locate(s, tables, job.start, picks.offsets, picks.table, picks.seconds, picks.weight,
                       picks.correction, tsta)
        wall = time.perf_counter() - t1
        # The tables as .qttb files (TravelTimeTable.Write) and back (TravelTimeTable.Open).
        from oracle import qttb as OQ
        from tomostar_b200 import qttb

        with tempfile.TemporaryDirectory() as tmp:
            heads = [qttb.header_json(f"S{t % 60:02d}", "PS"[job.table_phase[t]], *job.table_source[t], job.grid)
                     for t in range(len(tabs))]
            paths = [os.path.join(tmp, f"S{t % 60:02d}.{'PS'[job.table_phase[t]]}.qttb") for t in range(len(tabs))]
            t3 = time.perf_counter()
            qttb.write(tables, paths, heads)
            write_s = time.perf_counter() - t3
            t4 = time.perf_counter()
            back = qttb.load(s, job.grid, paths)
            load_s = time.perf_counter() - t4
            same = bool(np.array_equal(back.copy(0, 3), tabs[:3]))
            back.close()
            same_bytes = open(paths[0], "rb").read() == OQ.write_bytes(heads[0], tabs[0].astype(np.float64))
            t5 = time.perf_counter()
            for t in range(8):
                with open(os.path.join(tmp, "cpu.qttb"), "wb") as f:
                    f.write(OQ.write_bytes(heads[t], tabs[t].astype(np.float64)))
            cpu_write_s = (time.perf_counter() - t5) / 8 * len(tabs)
        gb = tabs.nbytes / 1e9
        qttb_line = {"tables": len(tabs), "gb": gb, "write_s": write_s, "write_gbs": gb / write_s, "load_s": load_s,
                     "load_gbs": gb / load_s, "round_trip_equal": same, "bytes_equal_restatement": same_bytes,
                     "cpu_baseline": {"write_gbs": gb / cpu_write_s, "kind": "port", "cores": 1,
                                      "sample": "8 tables written by the byte restatement (numpy), scaled to 120"}}
        tables.close()
    k = min(cpu_events, n_events)
    st, o, tb, sec, w, corr = sub(k)
    t2 = time.perf_counter()
    ora, _ = O.locate_many(O.Grid.of(job.grid), tabs, tsta, O.LocatorSettings(), st, o, tb, sec, w, corr,
                           threads=threads)
    cpu_s = time.perf_counter() - t2
    d = r.locations[:k]
    ok = r.locations["status"] == 0
    err = syn.surface_distance_km(r.locations["lon"], r.locations["lat"], job.truth[:, 0], job.truth[:, 1])
    err0 = syn.surface_distance_km(job.start[:, 0], job.start[:, 1], job.truth[:, 0], job.truth[:, 1])
    picks_per_event = float(np.mean(np.diff(picks.offsets)))
    return {
        "workload": "relocation_regional: 161x161x81 at 0.5 km, 60 stations x P,S = 120 float32 tables "
                    f"(1.0 GB) resident, {n_events} events, {picks_per_event:.1f} picks per event (seed 8)",
        "events": n_events, "located": int(ok.sum()), "wall_s": wall, "events_per_s": n_events / wall,
        "device_ms": r.device_ms, "rounds": r.rounds, "candidates": r.candidates,
        "candidates_per_s": r.candidates / (r.device_ms / 1e3),
        "node_misfits_picks_per_s": r.candidates * picks_per_event / (r.device_ms / 1e3),
        "tables_build_s": build_s,
        "qttb": qttb_line,
        "median_error_km": {"start": float(np.median(err0)), "located": float(np.median(err[ok]))},
        "cpu_baseline": {"events_per_s": k / cpu_s, "cores": threads, "kind": "port",
                         "sample": f"the first {k} events, oracle EventLocator restated in C++, one event per thread"},
        "speedup_vs_cpu": (n_events / wall) / (k / cpu_s),
        "parity_sample": {"events": k, "status_equal": bool(np.array_equal(d["status"], ora["status"])),
                          "used_equal": bool(np.array_equal(d["used"], ora["used"])),
                          "max_dlon_deg": float(np.max(np.abs(d["lon"] - ora["lon"]))),
                          "max_ddepth_km": float(np.max(np.abs(d["depth_km"] - ora["depth_km"]))),
                          "max_dt0_s": float(np.max(np.abs(d["t0"] - ora["t0"])))},
    }


def resample_job(device: int) -> dict:
    """ForwardModel.FromInversionGrid on the device for the 401x401x121 model: P and S slowness of
    the 19.46 M forward nodes from the 201x201x61 inversion grid (ts_model_put_resampled, end to end:
    inversion slowness from the host, the model left resident), against the C++ restatement on one core."""
    from oracle import oracle as O
    from tomostar_b200 import _lib as L
    from tomostar_b200 import domain
    from tomostar_b200 import synthetic as syn
    from tomostar_b200.eikonal import EikonalCuda

    g = syn.regular_grid(401, 401, 121, 0.25)
    inv = g.coarsened(2)
    rng = np.random.default_rng(21)
    vp = 5.0 + 0.04 * np.repeat(inv.depth(), inv.nx * inv.ny) + 0.2 * rng.standard_normal(inv.count)
    s_inv = np.stack([1 / vp, 1.73 / vp])
    times = []
    with EikonalCuda.create(device, 64) as s:
        for rep in range(4):
            t0 = time.perf_counter()
            mid = domain.put_resampled(s, g, inv, s_inv)
            times.append(time.perf_counter() - t0)
            if rep == 0:
                got = domain.copy_slowness(s, mid, 0, g.count)
            L.load().ts_model_drop(s.handle, mid)
    t_dev = min(times[1:])
    t1 = time.perf_counter()
    want = O.resample(O.Grid.of(g), O.Grid.of(inv), s_inv)
    cpu_s = time.perf_counter() - t1
    out_gb = 2 * g.count * 8 / 1e9
    return {"workload": "401x401x121 forward nodes (19.46 M) x P,S from the 201x201x61 inversion grid, FP64",
            "wall_s": t_dev, "nodes_per_s": 2 * g.count / t_dev, "slowness_gbs_written": out_gb / t_dev,
            "bitwise_equal_restatement": bool(np.array_equal(got, want[0])),
            "cpu_baseline": {"wall_s": cpu_s, "cores": 1, "kind": "port",
                             "sample": "the whole grid, the C++ restatement"},
            "speedup_vs_cpu": cpu_s / t_dev,
            "note": "end to end per call: 39 MB of inversion slowness uploaded, 311 MB model allocated and written"}


def _fmm_sample_fields_per_s(grids, slownesses, seed_sets, threads: int):
    """The reference's CPU solver (SphericalEikonal.Solve, fast marching, restated in oracle/) on the
    given fields, one field per host thread; returns (fields/s, seconds)."""
    from concurrent.futures import ThreadPoolExecutor

    from oracle import oracle as O

    def one(q):
        return O.fmm(O.Grid.of(grids[q]), slownesses[q], *seed_sets[q])

    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(one, range(len(grids))))
    dt = time.perf_counter() - t0
    return len(grids) / dt, dt


def inversion_job(device: int, threads: int) -> dict:
    """The forward step of a synthetic inversion (121x121x61 at 0.5 km, 25 stations x P,S = 50 fields,
    7,500 rays) in FP64 and FP32 (the paired-float scheme): engine fields/s (the 50 fields in one
    launch, P and S as two slowness models of the grid, the tile shape and scheduler picked by the
    autotuner on the job), its roofline, the forward step through ts_forward (tables + Jacobian rows),
    the plain per-plane GPU path on one field and the CPU solver on a sample of fields."""
    from oracle import oracle as O
    from tomostar_b200 import _lib as L
    from tomostar_b200 import synthetic as syn
    from tomostar_b200.eikonal import EikonalCuda, pack_seeds, point_source
    from tomostar_b200.rays import RayKernels

    p = syn.inversion_step_121()
    g = p.grid
    lib = L.load()
    P = C.POINTER
    peak, _ = measured_hbm_peak()
    seeds = {ph: [point_source(g, p.slowness[ph], *p.stations[q]) for q in range(len(p.stations))] for ph in (0, 1)}
    out = {"workload": "inversion_step_121: 121x121x61 at 0.5 km (0.89 M nodes), 25 stations x P,S = 50 fields, "
                       "150 events, 7,500 P+S rays into a CSR Jacobian"}
    # The P and S fields in one launch: the grid twice, with the P and the S slowness.
    grids, slows = [g, g], [p.slowness[0], p.slowness[1]]
    fg = [0] * 25 + [1] * 25
    sets = seeds[0] + seeds[1]
    with EikonalCuda.create(device, 64) as s:
        for prec in (64, 32):
            best, sched, _ = s.autotune(grids, slows, fg, sets, mode=L.MODE_FAST, precision=prec)
            lib.ts_engine_set_tile(s.handle, prec, best)
            lib.ts_engine_set_scheduler(s.handle, sched)

            def step():
                s.solve_multi(grids, slows, fg, sets, out_dtype=None, mode=L.MODE_FAST, precision=prec)
                st = s.last_stats_struct
                return st.device_ms, st.kernel_ms, st.node_updates

            for _ in range(3):
                step()
            runs = [step() for _ in range(5)]
            dev = sum(r[0] for r in runs) / 5
            kern = sum(r[1] for r in runs) / 5
            upd = runs[-1][2]
            ach = upd * 24 / (kern / 1e3) / 1e9
            shape = {sid: f"{bx}x{by}x{bz}" for sid, bx, by, bz in L.engine_shapes()}[best]
            rk = RayKernels(p.inv, g, s)
            rk.compute(p.slowness, p.stations, p.events, p.arrivals, precision=prec)  # warm-up
            t0 = time.perf_counter()
            rows = rk.compute(p.slowness, p.stations, p.events, p.arrivals, precision=prec)
            fwd_s = time.perf_counter() - t0
            tables_s = rk.last_stats.device_ms / 1e3
            out[f"fp{prec}"] = {
                "fields_per_s": 50 / (dev / 1e3), "ms_per_50_fields": dev, "node_updates": upd,
                "autotuned": {"shape": shape, "scheduler": ["lockstep", "flow"][sched]},
                "updates_per_s": upd / (kern / 1e3),
                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
                             "bytes_per_update": 24},
                "forward_step": {"wall_s": fwd_s, "tables_s": tables_s, "rows": int(rows.n_rows),
                                 "kept_rows": int(rows.ok.sum()), "nnz": int(rows.nnz),
                                 "rows_per_s": rows.n_rows / fwd_s,
                                 "rays_rows_per_s": rows.n_rows / max(1e-9, fwd_s - tables_s)},
            }
        # FP32 against the FP64 fields on two of the fields (the bitwise engine is the FP64 oracle).
        sub_seeds = [seeds[0][0], seeds[1][7]]
        worst = 0.0
        for q, ph in enumerate((0, 1)):
            f64 = s.solve(g, p.slowness[ph], [sub_seeds[q]], precision=64, mode=L.MODE_ENGINE)[0]
            f32 = s.solve(g, p.slowness[ph], [sub_seeds[q]], precision=32, mode=L.MODE_ENGINE)[0]
            fin = np.isfinite(f64) & (f64 > 0)
            worst = max(worst, float(np.max(np.abs(f32[fin] - f64[fin]) / f64[fin])))
        out["fp32_max_rel_err_vs_fp64"] = worst
        # Plain per-plane GPU path, one field.
        t0 = time.perf_counter()
        s.solve(g, p.slowness[0], [seeds[0][0]], precision=64, mode=L.MODE_PLAIN)
        out["plain_gpu"] = {"fields_per_s": 1 / (time.perf_counter() - t0), "sample": "1 P field, one launch per plane"}
    n_cpu = min(threads, 50)
    gl = [g] * n_cpu
    sl = [p.slowness[q % 2] for q in range(n_cpu)]
    ss = [seeds[q % 2][q // 2 % 25] for q in range(n_cpu)]
    r, dt = _fmm_sample_fields_per_s(gl, sl, ss, threads)
    out["cpu_baseline"] = {"fields_per_s": r, "cores": threads, "kind": "port",
                           "sample": f"{n_cpu} of the 50 fields, fast marching one field per thread"}
    out["speedup_fp64_vs_cpu"] = out["fp64"]["fields_per_s"] / r
    out["speedup_fp64_vs_plain_gpu"] = out["fp64"]["fields_per_s"] / out["plain_gpu"]["fields_per_s"]
    return out


def uneven_job(device: int, threads: int) -> dict:
    """200 sources each on its own grid (48-192 x 48-192 x 32-96 nodes, half with geometric depth
    spacing) solved in one persistent engine launch, the tile shape and scheduler picked by the
    autotuner on a 40-grid sample, the job captured as a CUDA graph and replayed; FP32 (the named
    precision: paired floats) and FP64. Baselines: the plain per-plane GPU path and the CPU solver on
    samples of the grids."""
    from tomostar_b200 import _lib as L
    from tomostar_b200 import synthetic as syn
    from tomostar_b200.eikonal import EikonalCuda, point_source

    b = syn.uneven_grids(200)
    seeds = [point_source(g, s, *src) for g, s, src in zip(b.grids, b.slowness, b.sources)]
    fg = list(range(len(b.grids)))
    nodes = sum(g.count for g in b.grids)
    peak, _ = measured_hbm_peak()
    out = {"workload": f"uneven_grids: 200 grids ({nodes / 1e6:.1f} M nodes in all, {sum(g.depth_km is not None for g in b.grids)} "
                       "with geometric depth spacing), one source each, seed 3"}
    with EikonalCuda.create(device, 64) as s:
        lib = L.load()
        for prec in (32, 64):
            sample = list(range(0, 200, 5))
            best, sched, table = s.autotune([b.grids[q] for q in sample], [b.slowness[q] for q in sample],
                                            list(range(len(sample))), [seeds[q] for q in sample], mode=L.MODE_FAST,
                                            precision=prec)
            lib.ts_engine_set_tile(s.handle, prec, best)
            lib.ts_engine_set_scheduler(s.handle, sched)
            s.set_graph(True)
            times, kern, upd = [], [], 0
            for rep in range(4):
                s.solve_multi(b.grids, b.slowness, fg, seeds, out_dtype=None, mode=L.MODE_FAST, precision=prec)
                st = s.last_stats_struct
                if rep >= 1:  # the first call captures the graph
                    times.append(st.device_ms)
                    kern.append(st.kernel_ms)
                    upd = st.node_updates
            replays = s.graph_replays
            s.set_graph(False)
            ms = float(np.median(times))
            shape = {sid: f"{bx}x{by}x{bz}" for sid, bx, by, bz in L.engine_shapes()}[best]
            k_ms = float(np.median(kern)) if any(k > 0 for k in kern) else ms
            ach = upd * 24 / (k_ms / 1e3) / 1e9
            out[f"fp{prec}"] = {"fields_per_s": 200 / (ms / 1e3), "ms_per_job": ms, "node_updates": int(upd),
                                "updates_per_s": upd / (ms / 1e3), "graph_replays": int(replays),
                                "autotuned": {"shape": shape, "scheduler": ["lockstep", "flow"][sched]},
                                "roofline": {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s",
                                             "frac": ach / peak, "bytes_per_update": 24}}
        lib.ts_engine_set_tile(s.handle, 64, 0)
        lib.ts_engine_set_tile(s.handle, 32, 0)
        lib.ts_engine_set_scheduler(s.handle, 0)
        # Plain per-plane GPU path on four of the grids (one field each).
        t0 = time.perf_counter()
        for q in (0, 50, 100, 150):
            s.solve(b.grids[q], b.slowness[q], [seeds[q]], precision=64, mode=L.MODE_PLAIN)
        plain = 4 / (time.perf_counter() - t0)
    out["plain_gpu"] = {"fields_per_s": plain, "sample": "grids 0, 50, 100, 150 one at a time, one launch per plane"}
    n_cpu = min(threads, 32)
    q = list(range(0, 200, 200 // n_cpu))[:n_cpu]
    r, dt = _fmm_sample_fields_per_s([b.grids[i] for i in q], [b.slowness[i] for i in q], [seeds[i] for i in q],
                                     threads)
    out["cpu_baseline"] = {"fields_per_s": r, "cores": threads, "kind": "port",
                           "sample": f"{n_cpu} of the 200 grids, fast marching one grid per thread"}
    out["speedup_vs_plain_gpu"] = out["fp32"]["fields_per_s"] / plain
    out["speedup_vs_cpu"] = out["fp32"]["fields_per_s"] / r
    return out


def run_reference(args, problem_fn):
    # The CPU arm needs no process group: rank 0 alone runs it and prints the line.
    if int(os.environ.get("RANK", "0")) != 0:
        return 0
    threads = os.cpu_count() or 1
    p = problem_fn(1)
    n = threads  # one field per host thread: ~one fast-marching solve of time per step
    rates = []
    for step in range(args.warmup + args.steps):
        r, dt = cpu_fmm_sample(p, n, threads)
        if step >= args.warmup:
            rates.append(r)
    v = float(np.mean(rates))
    line = {
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * n / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "regional forward step: 401x401x121 at 0.25 km, 800 P+S fields (400 stations)",
                   "sample": f"{n} fields per step"},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                         "sample": f"{n} of 800 fields per step, fast marching (oracle/oracle.cpp or_fmm_many)"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args, problem_fn):
    world, rank, local, dist = setup_dist(args)
    from tomostar_b200 import _lib as L
    from tomostar_b200.eikonal import EikonalCuda, pack_seeds, point_source

    lib = L.load()
    p = problem_fn(world)
    g = p.grid
    n = g.count
    my_st = rank_stations(p, rank, world)
    n_st = min(len(my_st), args.fields) if args.fields > 0 else len(my_st)
    solver = EikonalCuda.create(local, 64)
    rel, msg = solver.self_test()
    if not (rel <= 1e-6):
        raise SystemExit(f"self-test failed: {msg}")
    lib.ts_engine_set_tile(solver.handle, 64, args.tile)
    lib.ts_engine_set_scheduler(solver.handle, args.scheduler)
    # Seeds of every (station, phase) field, on the host before timing (PointSource, C ABI).
    seeds = {ph: [point_source(g, p.slowness[ph], *my_st[q]) for q in range(n_st)] for ph in (0, 1)}
    packed = {ph: pack_seeds(seeds[ph]) for ph in (0, 1)}
    gs = g.struct()
    mid = C.c_int32()
    s_all = np.ascontiguousarray(p.slowness)
    rc = lib.ts_model_put(solver.handle, C.byref(gs), s_all.ctypes.data_as(C.POINTER(C.c_double)), 2, 64,
                          C.byref(mid))
    if rc:
        raise SystemExit(f"model upload failed: {solver.last_error}")
    P = C.POINTER
    stats = L.EikStats()

    def step_resident():
        dev_ms = kern_ms = 0.0
        upd = 0
        for ph in (0, 1):
            off, idx, t = packed[ph]
            rc = lib.ts_eik_solve_model(solver.handle, mid.value, ph, n_st, off.ctypes.data_as(P(C.c_int32)),
                                        idx.ctypes.data_as(P(C.c_int32)), t.ctypes.data_as(P(C.c_double)),
                                        args.mode, 1e-7, 0, None, L.OUT_NONE, C.byref(stats))
            if rc:
                raise SystemExit(f"solve failed: {solver.last_error}")
            dev_ms += stats.device_ms
            kern_ms += stats.kernel_ms
            upd += stats.node_updates
            if args.verbose:
                print(f"phase {ph}: {n_st} fields device {stats.device_ms:.1f} ms kernel {stats.kernel_ms:.1f} ms "
                      f"node updates {stats.node_updates} tile visits {stats.tile_visits} "
                      f"rounds {stats.rounds[0]}+{stats.rounds[1]}", file=sys.stderr, flush=True)
        return dev_ms, kern_ms, upd, (stats.rounds[0], stats.rounds[1])

    for _ in range(args.warmup):
        step_resident()
    barrier(dist)
    clocks = ClockSampler(local)
    clocks.start()
    dev = kern = 0.0
    updates = 0
    t_wall = time.perf_counter()
    for _ in range(args.steps):
        d, k, u, rounds = step_resident()
        dev += d
        kern += k
        updates += u
    t_wall = time.perf_counter() - t_wall
    clk = clocks.stop()
    barrier(dist)
    value, dev_max = job_throughput(dist, local, world, 2 * n_st, args.steps, dev)

    # Roofline of the sweeping kernel: algorithmic bytes per node update (FP64: the node's time read
    # and written, its slowness read = 24 B) over the kernel's event time.
    peak, peak_kind = measured_hbm_peak()
    launches = 2 * args.steps
    achieved = updates * 24 / (kern / 1e3) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "engine_traffic.json")
    if os.path.exists(prof):
        try:
            bpu = json.load(open(prof))["dram_bytes_per_node_update_f64"]
            traffic = bpu * updates / launches
        except Exception:
            traffic = None

    # End to end through ts_eik_solve: host slowness and seeds in, float32 tables out to pinned memory.
    e2e = None
    if not args.no_e2e:
        import torch

        out = torch.empty((n_st, n), dtype=torch.float32, pin_memory=True)
        out_np = out.numpy()
        s_pin = [torch.from_numpy(np.ascontiguousarray(p.slowness[ph])).pin_memory() for ph in (0, 1)]
        h2d = d2h = 0

        def step_e2e():
            nonlocal h2d, d2h
            for ph in (0, 1):
                off, idx, t = packed[ph]
                rc = lib.ts_eik_solve(solver.handle, C.byref(gs), C.cast(s_pin[ph].data_ptr(), P(C.c_double)), n_st,
                                      off.ctypes.data_as(P(C.c_int32)), idx.ctypes.data_as(P(C.c_int32)),
                                      t.ctypes.data_as(P(C.c_double)), 64, args.mode, 1e-7, 0,
                                      out_np.ctypes.data_as(C.c_void_p), L.OUT_F32, C.byref(stats))
                if rc:
                    raise SystemExit(f"e2e solve failed: {solver.last_error}")
                h2d += n * 8 + off.nbytes + idx.nbytes + t.nbytes
                d2h += n_st * n * 4

        step_e2e()  # warm-up (allocations)
        h2d = d2h = 0
        barrier(dist)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            step_e2e()
        e2e_s = max_over_ranks(dist, local, time.perf_counter() - t0)
        e2e = {"value": 2 * n_st * world * args.e2e_steps / e2e_s, "unit": UNIT,
               "h2d_bytes_per_step": h2d // args.e2e_steps, "d2h_bytes_per_step": d2h // args.e2e_steps,
               "steps": args.e2e_steps}

    # Baselines on rank 0: the plain per-plane GPU path on one field, the CPU solver on a sample.
    plain = cpu = None
    if rank == 0 and not args.no_baselines:
        off, idx, t = pack_seeds(seeds[0][:1])
        rc = lib.ts_eik_solve_model(solver.handle, mid.value, 0, 1, off.ctypes.data_as(P(C.c_int32)),
                                    idx.ctypes.data_as(P(C.c_int32)), t.ctypes.data_as(P(C.c_double)), L.MODE_PLAIN,
                                    1e-7, 0, None, L.OUT_NONE, C.byref(stats))
        if rc == 0:
            plain = {"value": 1e3 / stats.device_ms, "unit": UNIT, "sample": "1 P field, one launch per plane",
                     "launches": int(stats.launches)}
        threads = os.cpu_count() or 1
        r, dt = cpu_fmm_sample(p, threads, threads)
        cpu = {"value": r, "unit": UNIT, "cores": threads, "kind": "port",
               "sample": f"{threads} of 800 fields, fast marching one field per thread (oracle/oracle.cpp)"}

    solver.close()
    # The whole forward step through RayKernels.Compute's drop-in (ts_forward): the 800 tables, then
    # every arrival back-traced into its Jacobian row, rows copied to the host.
    forward = None
    if world == 1 and not args.no_forward:
        from tomostar_b200 import lsqr

        fsolver = EikonalCuda.create(local, 64)
        lib.ts_engine_set_tile(fsolver.handle, 64, args.tile)
        fs, is_ = g.struct(), p.inv.struct()
        s_all = np.ascontiguousarray(p.slowness)
        st = np.ascontiguousarray(p.stations)
        ev = np.ascontiguousarray(p.events)
        ar = np.ascontiguousarray(p.arrivals, np.int32)
        ae, ast, aph = (np.ascontiguousarray(ar[:, q]) for q in range(3))
        fstats = L.EikStats()

        def forward_call(mode):
            hh = C.c_void_p()
            t = time.perf_counter()
            rc = lib.ts_forward(fsolver.handle, C.byref(fs), s_all.ctypes.data_as(P(C.c_double)), len(s_all),
                                C.byref(is_), len(st), st.ctypes.data_as(P(C.c_double)), len(ev),
                                ev.ctypes.data_as(P(C.c_double)), len(ar), ae.ctypes.data_as(P(C.c_int32)),
                                ast.ctypes.data_as(P(C.c_int32)), aph.ctypes.data_as(P(C.c_int32)), 64, mode, 0.0,
                                C.byref(hh), C.byref(fstats))
            if rc:
                raise SystemExit(f"forward step failed: {fsolver.last_error}")
            return hh, time.perf_counter() - t

        # The bitwise mode first (its tables only are reported), then the default fast mode.
        exact = None
        if not args.no_forward_exact:
            hx, fwd_x = forward_call(L.MODE_ENGINE)
            exact = {"mode": "engine (the reference's fields to the bit)", "wall_s": fwd_x,
                     "tables_s": fstats.device_ms / 1e3, "node_updates": int(fstats.node_updates)}
            lib.ts_rows_free(hx)
        h, fwd_s = forward_call(args.mode)
        fields_s = fstats.device_ms / 1e3
        fwd_stats = fsolver.last_stats  # the step's timing: tables, then the rays' host and device parts
        # LSQR (Lsqr.Solve) on the rows where they lie: 100 iterations, no early stop (fixed work).
        b = np.random.default_rng(11).standard_normal(len(ar)) * 0.05
        t1 = time.perf_counter()
        lres = lsqr.solve_rows(fsolver, h, p.inv.count, b, damp=0.1, max_iterations=100, atol=0, btol=0, conlim=0)
        lsqr_wall = time.perf_counter() - t1
        # Rows to pinned host buffers (the host side of RayKernels.Compute's result), then freed.
        import torch

        n_rows_c, nnz_c = C.c_int32(), C.c_int64()
        lib.ts_rows_info(h, C.byref(n_rows_c), C.byref(nnz_c))
        n_rows, nnz = int(n_rows_c.value), int(nnz_c.value)
        pin = {k: torch.empty(sz, dtype=dt, pin_memory=True)
               for k, sz, dt in (("rp", n_rows + 1, torch.int32), ("col", max(1, nnz), torch.int32),
                                 ("len", max(1, nnz), torch.float32), ("tg", 4 * n_rows, torch.float64),
                                 ("ok", n_rows, torch.uint8))}
        t2 = time.perf_counter()
        rc = lib.ts_rows_copy(h, C.cast(pin["rp"].data_ptr(), P(C.c_int32)), C.cast(pin["col"].data_ptr(), P(C.c_int32)),
                              C.cast(pin["len"].data_ptr(), P(C.c_float)), C.cast(pin["tg"].data_ptr(), P(C.c_double)),
                              C.cast(pin["ok"].data_ptr(), P(C.c_uint8)))
        copy_s = time.perf_counter() - t2
        lib.ts_rows_free(h)
        if rc:
            raise SystemExit("row copy failed")
        kept = int(pin["ok"].numpy().astype(bool).sum())
        # Algorithmic bytes of one LSQR iteration: A·v and Aᵀ·u each read every non-zero's column
        # index and float32 length (4 + 4 B, the rows as the rays leave them) and read and write their
        # output vector.
        it_bytes = 2 * nnz * 8 + 16 * (n_rows + p.inv.count)
        it_ms = lres.device_ms / max(1, lres.iterations)
        lsqr_gbs = it_bytes / (it_ms / 1e3) / 1e9
        peak, _ = measured_hbm_peak()
        # Roofline of the ray kernels: per row, one 8-corner float32 gather (32 B) per back-tracing step,
        # the row's non-zeros (int32 node + float32 length) and 32 B of row scalars, over the ray
        # pipeline's device time (both from the call's own counters).
        import re

        m_dev = re.search(r"on the device ([0-9.]+) ms", fwd_stats)
        m_steps = re.search(r"([0-9]+) steps\)", fwd_stats)
        ray_roof = None
        if m_dev and m_steps:
            ray_dev_s = float(m_dev.group(1)) / 1e3
            steps = int(m_steps.group(1))
            ray_bytes = steps * 32 + nnz * 8 + n_rows * 32
            ach_r = ray_bytes / ray_dev_s / 1e9
            ray_roof = {"bound": "hbm", "achieved": ach_r, "peak": peak, "unit": "GB/s", "frac": ach_r / peak,
                        "bytes_per_row": ray_bytes / max(1, n_rows), "steps_per_row": steps / max(1, n_rows),
                        "device_s": ray_dev_s, "device_rows_per_s": n_rows / ray_dev_s}
        forward = {"arrivals": n_rows, "tables": 2 * len(p.stations), "wall_s": fwd_s + copy_s,
                   "rows_per_s": n_rows / (fwd_s + copy_s), "tables_s": fields_s,
                   "rays_and_copy_s": fwd_s - fields_s + copy_s,
                   "rays_rows_per_s": n_rows / max(1e-9, fwd_s - fields_s + copy_s), "nnz": nnz,
                   "nnz_per_row": nnz / max(1, kept), "kept_rows": kept,
                   "copy_s": copy_s, "copy_gbs": (nnz * 8 + n_rows * 45) / copy_s / 1e9,
                   "timing": fwd_stats,
                   "rays_roofline": ray_roof,
                   "mode": ("fast" if args.mode == L.MODE_FAST else "engine (bitwise)") +
                           " tables (FP64 fields as float32), rays FP64",
                   "exact_mode": exact,
                   "lsqr": {"iterations": lres.iterations, "columns": p.inv.count, "damp": 0.1,
                            "wall_s": lsqr_wall, "device_ms": lres.device_ms, "ms_per_iteration": it_ms,
                            "achieved_gbs": lsqr_gbs, "hbm_frac": lsqr_gbs / peak,
                            "setup_s": lsqr_wall - lres.device_ms / 1e3,
                            "note": "setup = transpose built on the device from the resident rows, column order as the host transpose"}}
        del pin
        fsolver.close()
    location = resample = None
    if world == 1 and not args.no_location:
        # Sections beside the headline: a failure is reported in the line, not fatal to it.
        try:
            location = location_job(local, args.location_events, args.location_cpu_events, os.cpu_count() or 1)
        except Exception as exc:  # noqa: BLE001
            location = {"error": repr(exc)[:300]}
        try:
            resample = resample_job(local)
        except Exception as exc:  # noqa: BLE001
            resample = {"error": repr(exc)[:300]}
    inversion = uneven = None
    if world == 1 and not args.no_configs:
        try:
            inversion = inversion_job(local, os.cpu_count() or 1)
        except Exception as exc:  # noqa: BLE001
            inversion = {"error": repr(exc)[:300]}
        try:
            uneven = uneven_job(local, os.cpu_count() or 1)
        except Exception as exc:  # noqa: BLE001
            uneven = {"error": repr(exc)[:300]}
    # The serving load (Poisson stream of mixed requests) on one GPU, after the batch job's buffers
    # are released; at N = 1 only (the scaling runs measure the batch job).
    serving = None
    if world == 1 and not args.no_serving:
        from tomostar_b200.serve_load import run as serve_run

        serving = serve_run(seconds=args.serve_seconds, rate=200.0, tile=args.serve_tile,
                            rounds_per_epoch=args.serve_rounds, budget_bytes=120e9, device=local,
                            scheduler=args.serve_scheduler, epoch_ms=args.serve_epoch_ms)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": dev_max / args.steps, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"regional forward step: 401x401x121 nodes at 0.25 km (19.46 M), {n_st} surface stations x P,S "
                                   f"= {2 * n_st} fields per GPU, Vp 1-D gradient + 3 ellipsoids +-8 % (seed 5)",
                       "global_fields": 2 * n_st * world, "tile": args.tile,
                       "scheduler": {0: "lockstep diagonals", 1: "flow (per-field diagonals, tile queue)"}[args.scheduler],
                       "mode": {0: "engine (bitwise with the reference)",
                                2: "fast (a drop wakes only neighbours above the new time, and only when above "
                                   "1e-13 of it; within 1e-10 rel of bitwise)"}[args.mode],
                       "l2": "inputs larger than L2 (fields 2 x 65 GB per step)",
                       "rounds_last": list(rounds)},
            # Per solve call: the init, seed, engine and state-gather kernels.
            "gpu_launches": 4 * launches,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": "engine_kernel (FP64), 24 B per node update"},
            "clocks": clk,
            "e2e": e2e,
            "cpu_baseline": cpu,
            "plain_gpu": plain,
            "forward_step": forward,
            "location": location,
            "resample": resample,
            "inversion_step_121": inversion,
            "uneven_grids": uneven,
            "serving": serving,
            "node_updates_per_step": updates // args.steps,
            "wall_s_timed": t_wall,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--tile", type=int, default=6)
    ap.add_argument("--mode", type=int, default=2, help="0 engine (bitwise), 2 fast (wake threshold 1e-13)")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-baselines", action="store_true")
    ap.add_argument("--fields", type=int, default=0, help="stations per step (default all 400; fewer = a small case)")
    ap.add_argument("--verbose", action="store_true", help="per-launch statistics on stderr")
    ap.add_argument("--scheduler", type=int, default=0, help="0 lockstep diagonals, 1 flow (per field)")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving-load measurement")
    ap.add_argument("--no-forward", action="store_true", help="skip the forward step (tables + rays)")
    ap.add_argument("--no-forward-exact", action="store_true", help="skip the bitwise-mode forward step")
    ap.add_argument("--no-location", action="store_true", help="skip the relocation measurement")
    ap.add_argument("--no-configs", action="store_true",
                    help="skip the 121x121x61 inversion step and the 200 uneven grids sections")
    ap.add_argument("--location-events", type=int, default=4000)
    ap.add_argument("--location-cpu-events", type=int, default=256, help="events the CPU baseline locates")
    ap.add_argument("--serve-scheduler", type=int, default=1)
    ap.add_argument("--serve-seconds", type=float, default=60.0)
    ap.add_argument("--serve-tile", type=int, default=6)
    ap.add_argument("--serve-rounds", type=int, default=2, help="sweep rounds per serving epoch")
    ap.add_argument("--serve-epoch-ms", type=float, default=0.0,
                    help="flow scheduler: fields pause at their next round end after this long (0: off)")
    ap.add_argument("--dims", default="401,401,121",
                    help="grid of the regional job (smaller only for profiling captures; the bench line is 401,401,121)")
    args = ap.parse_args()
    dims = tuple(int(v) for v in args.dims.split(","))
    problem_fn = lambda world: job_problem(world, dims)  # noqa: E731

    if args.impl == "reference":
        return run_reference(args, problem_fn)
    return run_ours(args, problem_fn)


if __name__ == "__main__":
    sys.exit(main())
