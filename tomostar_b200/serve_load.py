"""Drives the serving engine with the serving load (Poisson arrivals of mixed requests) and reports
latency percentiles and throughput. Used by bench.py; `python -m tomostar_b200.serve_load` runs it
alone."""
from __future__ import annotations

import argparse
import json
import threading
import time

import numpy as np

from . import _lib as L
from . import synthetic as syn
from .eikonal import point_source
from .serving import Server


def run(seconds: float = 60.0, rate: float = 200.0, tile: int = 6, rounds_per_epoch: int = 2,
        budget_bytes: float = 120e9, device: int = 0, seed: int = 4, scheduler: int = 1,
        epoch_ms: float = 0.0) -> dict:
    models = syn.serving_models()
    stream = syn.serving_stream(models, rate=rate, duration=seconds, seed=seed)
    # Seeds of every field on the host before the clock starts (PointSource, ts_point_source).
    prepared = []
    for r in stream:
        m = models[r.model]
        prepared.append([point_source(m.grid, m.slowness[r.phase], *st) for st in r.stations])
    server = Server(device=device, tile=tile, budget_bytes=budget_bytes, rounds_per_epoch=rounds_per_epoch,
                    scheduler=scheduler, epoch_ms=epoch_ms)
    try:
        ids = {name: server.model_put(m.grid, m.slowness) for name, m in models.items()}

        def submit(r, seeds):
            return server.submit(ids[r.model], r.phase, seeds, origins=r.stations,
                                 ray_field=r.ray_field if len(r.events) else None,
                                 ray_event=r.events if len(r.events) else None)

        # Warm-up outside the clock: one request of each kind (pool allocations, first launches).
        seen = {}
        for r, sd in zip(stream, prepared):
            seen.setdefault(r.kind, (r, sd))
        for r, sd in seen.values():
            server.wait(submit(r, sd))
        base = server.stats()

        results = [None] * len(stream)
        rids = [None] * len(stream)
        ready = threading.Semaphore(0)

        def waiter():
            for q in range(len(stream)):
                ready.acquire()
                results[q] = server.wait(rids[q])

        th = threading.Thread(target=waiter)
        th.start()
        t0 = time.perf_counter()
        for q, (r, sd) in enumerate(zip(stream, prepared)):
            delay = t0 + r.t - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
            rids[q] = submit(r, sd)
            ready.release()
        th.join()
        wall = time.perf_counter() - t0
        st = server.stats()
    finally:
        server.close()
    ok = [res for res in results if res.status == L.TS_OK]
    lat = np.array([res.latency_ms for res in ok])
    queue = np.array([res.queue_ms for res in ok])
    fields = sum(res.n_fields for res in ok)
    rays = sum(res.rows.n_rows for res in ok if res.rows is not None)
    by_kind = {}
    for r, res in zip(stream, results):
        if res.status == L.TS_OK:
            by_kind.setdefault(r.kind, []).append(res.latency_ms)
    return {
        "requests": len(stream), "failed": len(stream) - len(ok), "seconds": seconds, "rate_per_s": rate,
        "wall_s": wall, "fields": fields, "fields_per_s": fields / wall, "rays": rays, "rays_per_s": rays / wall,
        "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
        "max_ms": float(lat.max()), "queue_p99_ms": float(np.percentile(queue, 99)),
        "p99_ms_by_kind": {k: float(np.percentile(v, 99)) for k, v in by_kind.items()},
        "p50_ms_by_kind": {k: float(np.percentile(v, 50)) for k, v in by_kind.items()},
        "epochs": st["epochs"] - base["epochs"], "engine_busy_s": (st["device_ms"] - base["device_ms"]) / 1e3,
        "epoch_wall_s": (st["epoch_ms"] - base["epoch_ms"]) / 1e3,
        "complete_wall_s": (st["complete_ms"] - base["complete_ms"]) / 1e3,
        "node_updates": st["node_updates"] - base["node_updates"], "peak_hbm_gb": st["peak_bytes"] / 1e9,
        "budget_gb": budget_bytes / 1e9, "tile": tile, "rounds_per_epoch": rounds_per_epoch,
        "scheduler": {0: "lockstep", 1: "flow"}[scheduler], "epoch_ms": epoch_ms,
        "errors": sorted({res.error for res in results if res.status != L.TS_OK})[:3],
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--seconds", type=float, default=60.0)
    ap.add_argument("--rate", type=float, default=200.0)
    ap.add_argument("--tile", type=int, default=6)
    ap.add_argument("--rounds-per-epoch", type=int, default=2)
    ap.add_argument("--budget-gb", type=float, default=120.0)
    ap.add_argument("--scheduler", type=int, default=1)
    ap.add_argument("--epoch-ms", type=float, default=0.0)
    a = ap.parse_args()
    print(json.dumps(run(a.seconds, a.rate, a.tile, a.rounds_per_epoch, a.budget_gb * 1e9, scheduler=a.scheduler,
                         epoch_ms=a.epoch_ms)))


if __name__ == "__main__":
    main()
