"""The multi-GPU path of bench.py on CPU ranks (gloo, world size 2): the ranks split one job by
station (station i on rank i % N; no collective on the data path) and the whole-job throughput
divides every rank's fields by the slowest rank's time, reduced with one all-reduce."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        dev_ms = [1000.0, 1250.0][rank]  # the second rank is slower
        value, dev_max = bench.job_throughput(dist, 0, world, 800, 3, dev_ms)
        p = bench.job_problem(world, dims=(41, 41, 21))
        out[rank] = (value, dev_max, bench.rank_stations(p, rank, world).tolist(), p.stations.tolist())
    finally:
        dist.destroy_process_group()


def test_weak_scaling_throughput_two_ranks():
    world = 2
    port = _free_port()
    with mp.Manager() as mgr:
        out = mgr.dict()
        ctx = mp.get_context("spawn")
        procs = [ctx.Process(target=_rank, args=(r, world, port, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(180)
            assert p.exitcode == 0
        res = dict(out)
    for r in range(world):
        value, dev_max, _, _ = res[r]
        assert dev_max == 1250.0
        assert value == pytest.approx(800 * 2 * 3 / 1.25)
    # One job (the same stations on both ranks), split by station: 400 per rank, disjoint, complete.
    allst = res[0][3]
    assert res[1][3] == allst and len(allst) == 800
    assert len(res[0][2]) == len(res[1][2]) == 400
    assert sorted(map(tuple, res[0][2] + res[1][2])) == sorted(map(tuple, allst))
