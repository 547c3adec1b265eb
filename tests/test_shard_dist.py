"""Station sharding of the forward step (MpiSession.cs:76-133) on two CPU ranks (gloo): the
partition rule, and the gather of the ranks' row blocks to rank 0 in arrival order, against the
rows of the same arrivals traced in one process. The rows are the oracle's (RayTracing.Backtrack +
Kernel on the same float32 tables), so the test needs no GPU; on GPUs each rank's block comes from
ts_forward on its own device and the gather is the same code over NCCL."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

from tomostar_b200 import shard

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_covers_every_arrival_once():
    rng = np.random.default_rng(3)
    arrivals = np.stack([rng.integers(0, 50, 400), rng.integers(0, 13, 400), rng.integers(0, 2, 400)], axis=1)
    for world in (1, 2, 3, 8):
        parts = [shard.local_arrivals(arrivals, r, world) for r in range(world)]
        allidx = np.sort(np.concatenate(parts))
        assert np.array_equal(allidx, np.arange(400))
        for r, p in enumerate(parts):
            assert np.all(arrivals[p, 1] % world == r)
        st = np.sort(np.concatenate([shard.station_share(13, r, world) for r in range(world)]))
        assert np.array_equal(st, np.arange(13))


def _problem():
    """A small forward step: 41x41x21 at 0.5 km, 5 surface stations x P and S, 7 events."""
    from oracle import oracle as O
    from tomostar_b200 import synthetic as syn

    g = syn.regular_grid(41, 41, 21, 0.5)
    inv = g.coarsened(2)
    vp = syn.vp_linear(g, 5.0, 0.03)
    slow = np.stack([1 / vp, 1.73 / vp])
    rng = np.random.default_rng(11)
    slon, slat = syn.km_to_geo(g, rng.uniform(2, 18, 5), rng.uniform(2, 18, 5), 0.5)
    stations = np.stack([slon, slat, np.zeros(5)], axis=1)
    elon, elat = syn.km_to_geo(g, rng.uniform(3, 17, 7), rng.uniform(3, 17, 7), 0.5)
    events = np.stack([elon, elat, rng.uniform(2, 8, 7)], axis=1)
    arrivals = np.array([(e, s, p) for e in range(7) for s in range(5) for p in range(2)], np.int32)
    og = O.Grid.of(g)
    tables = {}
    for s in range(5):
        for p in range(2):
            seeds = O.point_source(og, slow[p], *stations[s])
            tables[(s, p)] = O.to_table(O.relax(og, slow[p], *seeds)[0])
    return g, inv, slow, stations, events, arrivals, tables


def _oracle_block(prob, idx):
    """The oracle's rows of the arrivals idx, as a RowBlock."""
    from oracle import oracle as O
    from tomostar_b200.rays import step_km

    g, inv, _, stations, events, arrivals, tables = prob
    keys = sorted(tables)
    tab = np.stack([tables[k] for k in keys])
    ar = arrivals[idx]
    tab_of = np.array([keys.index((int(s), int(p))) for _, s, p in ar], np.int32)
    nnz, nodes, lens, tg = O.ray_rows_many(O.Grid.of(g), tab, tab_of, stations[ar[:, 1]], O.Grid.of(inv),
                                           events[ar[:, 0]], step_km(g, inv), threads=1)
    counts = np.maximum(nnz, 0).astype(np.int64)
    row_ptr = np.concatenate([[0], np.cumsum(counts)])
    col = np.concatenate([nodes[r, : counts[r]] for r in range(len(idx))]) if len(idx) else np.zeros(0, np.int32)
    ln = np.concatenate([lens[r, : counts[r]] for r in range(len(idx))]) if len(idx) else np.zeros(0, np.float32)
    return shard.RowBlock(np.asarray(idx, np.int64), row_ptr, col.astype(np.int32), ln.astype(np.float32), tg,
                          (nnz >= 0).astype(np.uint8), np.zeros(len(idx)))


def _rank(rank, world, port, out, fail_rank):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        prob = _problem()
        arrivals = prob[5]
        block, err = None, None
        if rank == fail_rank:
            err = "no device memory for the tables"  # this rank's share failed on its device
        else:
            block = _oracle_block(prob, shard.local_arrivals(arrivals, rank, world))
        try:
            merged = shard.gather_rows(block, len(arrivals), dist, error=err)
            if rank == 0:
                whole = _oracle_block(prob, np.arange(len(arrivals)))
                out["same"] = all(np.array_equal(getattr(merged, f), getattr(whole, f))
                                  for f in ("arrival", "row_ptr", "col", "length", "tcg", "ok", "outside"))
                out["rows"] = merged.n_rows
                out["nnz"] = merged.nnz
            else:
                out[f"none{rank}"] = merged is None
        except RuntimeError as exc:
            out[f"error{rank}"] = str(exc)
    finally:
        dist.destroy_process_group()


def _run(world, fail_rank=-1):
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out, fail_rank)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(300)
            assert p.exitcode == 0
        return dict(out)


def test_gather_two_ranks_equals_one_process():
    res = _run(2)
    assert res["same"], res
    assert res["rows"] == 70 and res["nnz"] > 0
    assert res["none1"]


def test_gather_reports_the_failing_rank():
    """A rank whose share failed still takes every collective step; rank 0 raises naming it
    (MpiSession.Dispatch, MpiSession.cs:84-85)."""
    res = _run(2, fail_rank=1)
    assert "rank 1: no device memory" in res["error0"]
    assert res["none1"]
