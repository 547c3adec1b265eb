"""The forward step split by station across GPUs, one process per GPU (Compute/MpiSession.cs:76-122).

The reference's MPI session runs RayKernels.Compute on each rank for the arrivals whose station
index satisfies `station % Size == Rank` (MpiSession.cs:101-106; table builds take the sources the
same way, :95-97), renumbers each rank's rows to their global arrival indices, and rank 0 collects
every rank's response, reports failures by rank, and orders the rows by arrival (Dispatch,
:76-87; Collect, :124-133).

Here each rank traces its share on its own device with ts_forward (its stations' tables and their
arrivals' rays); the only exchange is the final gather of the row blocks to the owner rank over
torch.distributed (NCCL between GPUs, gloo on CPU): one all-gather of the block sizes and of each
rank's status, then one gather of the padded blocks. No collective runs inside a solve.
"""
from __future__ import annotations

import dataclasses

import numpy as np


def station_share(n_stations: int, rank: int, world: int) -> np.ndarray:
    """The stations rank `rank` owns (MpiSession.cs:97: `i % Size == Rank`)."""
    return np.arange(rank, n_stations, world, dtype=np.int64)


def local_arrivals(arrivals: np.ndarray, rank: int, world: int) -> np.ndarray:
    """Indices of the arrivals traced on `rank` (MpiSession.cs:101: `Arrivals[i].Station % Size == Rank`);
    arrivals is (m, 3) int (event, station, phase)."""
    ar = np.asarray(arrivals).reshape(-1, 3)
    return np.nonzero(ar[:, 1] % world == rank)[0].astype(np.int64)


@dataclasses.dataclass
class RowBlock:
    """Jacobian rows of a set of arrivals: `arrival[r]` is row r's global arrival index; row r holds
    col/length[row_ptr[r]:row_ptr[r+1]]; tcg (n, 4) TCalc and the source gradient; ok: kept by the
    reference (0 = dropped, empty row); outside: RayRow.OutsideTime."""

    arrival: np.ndarray
    row_ptr: np.ndarray
    col: np.ndarray
    length: np.ndarray
    tcg: np.ndarray
    ok: np.ndarray
    outside: np.ndarray

    @property
    def n_rows(self) -> int:
        return len(self.arrival)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1]) if len(self.row_ptr) else 0

    @classmethod
    def empty(cls) -> "RowBlock":
        return cls(np.zeros(0, np.int64), np.zeros(1, np.int64), np.zeros(0, np.int32), np.zeros(0, np.float32),
                   np.zeros((0, 4)), np.zeros(0, np.uint8), np.zeros(0))

    @classmethod
    def of_rows(cls, rows, arrival: np.ndarray) -> "RowBlock":
        """From a tomostar_b200.rays.Rows result whose row r is arrival[r]."""
        outside = rows.outside if rows.outside is not None else np.zeros(rows.n_rows)
        return cls(np.asarray(arrival, np.int64), np.asarray(rows.row_ptr, np.int64), np.asarray(rows.col, np.int32),
                   np.asarray(rows.len, np.float32), np.asarray(rows.tcalc_grad, np.float64).reshape(-1, 4),
                   np.asarray(rows.ok, np.uint8), np.asarray(outside, np.float64))


def assemble(blocks: list, n_arrivals: int) -> RowBlock:
    """Every rank's block merged into arrival order (Dispatch's OrderBy(r => r.Arrival)). Each
    arrival must appear in exactly one block."""
    arrival = np.arange(n_arrivals, dtype=np.int64)
    counts = np.zeros(n_arrivals, np.int64)
    seen = np.zeros(n_arrivals, np.int32)
    for b in blocks:
        seen[b.arrival] += 1
        counts[b.arrival] = np.diff(b.row_ptr)
    if not np.all(seen == 1):
        raise ValueError("every arrival must come from exactly one rank")
    row_ptr = np.zeros(n_arrivals + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    col = np.empty(int(row_ptr[-1]), np.int32)
    length = np.empty(int(row_ptr[-1]), np.float32)
    tcg = np.empty((n_arrivals, 4))
    ok = np.empty(n_arrivals, np.uint8)
    outside = np.empty(n_arrivals)
    for b in blocks:
        if b.n_rows == 0:
            continue
        tcg[b.arrival] = b.tcg
        ok[b.arrival] = b.ok
        outside[b.arrival] = b.outside
        lens = np.diff(b.row_ptr)
        # Destination of each of the block's entries: its row's start in the merged rows plus its
        # position within the row.
        dst_start = np.repeat(row_ptr[b.arrival], lens)
        within = np.arange(b.nnz, dtype=np.int64) - np.repeat(b.row_ptr[:-1], lens)
        col[dst_start + within] = b.col
        length[dst_start + within] = b.length
    return RowBlock(arrival, row_ptr, col, length, tcg, ok, outside)


def _pack(b: RowBlock, max_rows: int, max_nnz: int):
    """The block as three fixed-size arrays (padded): int64 [arrival | row lengths], int32 col and
    float32 length bit patterns, float64 [tcg | outside | ok]."""
    ints = np.zeros(2 * max_rows, np.int64)
    ints[: b.n_rows] = b.arrival
    ints[max_rows: max_rows + b.n_rows] = np.diff(b.row_ptr)
    ent = np.zeros(2 * max_nnz, np.int32)
    ent[: b.nnz] = b.col
    ent[max_nnz: max_nnz + b.nnz] = np.asarray(b.length, np.float32).view(np.int32)
    flt = np.zeros(6 * max_rows)
    flt[: 4 * b.n_rows] = b.tcg.reshape(-1)
    flt[4 * max_rows: 4 * max_rows + b.n_rows] = b.outside
    flt[5 * max_rows: 5 * max_rows + b.n_rows] = b.ok
    return ints, ent, flt


def _unpack(ints, ent, flt, n_rows: int, nnz: int, max_rows: int, max_nnz: int) -> RowBlock:
    lens = ints[max_rows: max_rows + n_rows]
    row_ptr = np.zeros(n_rows + 1, np.int64)
    np.cumsum(lens, out=row_ptr[1:])
    return RowBlock(ints[:n_rows].copy(), row_ptr, ent[:nnz].copy(), ent[max_nnz: max_nnz + nnz].view(np.float32).copy(),
                    flt[: 4 * n_rows].reshape(-1, 4).copy(), flt[5 * max_rows: 5 * max_rows + n_rows].astype(np.uint8),
                    flt[4 * max_rows: 4 * max_rows + n_rows].copy())


def gather_rows(block: RowBlock | None, n_arrivals: int, dist, device: str = "cpu", dst: int = 0,
                error: str | None = None) -> RowBlock | None:
    """Collects every rank's rows on `dst` in arrival order (MpiSession.Collect + Dispatch). Every
    rank takes the same collective steps, also when its own part failed (`error` set, block None):
    then `dst` raises with each failing rank's message, as Dispatch does (MpiSession.cs:84-85), and
    the other ranks return None. `device` is where the transfer tensors live ("cuda:k" under NCCL).
    Returns the merged block on `dst`, None elsewhere."""
    import torch

    rank, world = dist.get_rank(), dist.get_world_size()
    if block is None:
        block = RowBlock.empty()
    status = [None] * world
    dist.all_gather_object(status, (error, block.n_rows, block.nnz))
    failures = [f"rank {r}: {s[0]}" for r, s in enumerate(status) if s[0] is not None]
    if failures:
        if rank == dst:
            raise RuntimeError("sharded forward step failed: " + "; ".join(failures))
        return None
    max_rows = max(1, max(s[1] for s in status))
    max_nnz = max(1, max(s[2] for s in status))
    parts = [torch.from_numpy(a).to(device) for a in _pack(block, max_rows, max_nnz)]
    got = []
    for t in parts:
        bufs = [torch.empty_like(t) for _ in range(world)] if rank == dst else None
        dist.gather(t, gather_list=bufs, dst=dst)
        got.append(bufs)
    if rank != dst:
        return None
    blocks = [_unpack(got[0][r].cpu().numpy(), got[1][r].cpu().numpy(), got[2][r].cpu().numpy(), status[r][1],
                      status[r][2], max_rows, max_nnz) for r in range(world)]
    return assemble(blocks, n_arrivals)


def forward_shard(kernels, slowness_fwd, stations, events, arrivals, rank: int, world: int,
                  precision: int | None = None, mode: int | None = None) -> RowBlock:
    """This rank's part of the forward step (MpiSession.RunLocal for "rays", MpiSession.cs:99-116):
    the arrivals of its stations traced with `kernels` (a tomostar_b200.rays.RayKernels on this
    rank's device), which builds only the tables of those stations, rows tagged with their global
    arrival indices."""
    from . import _lib as L

    idx = local_arrivals(arrivals, rank, world)
    if len(idx) == 0:
        return RowBlock.empty()
    rows = kernels.compute(slowness_fwd, stations, events, np.asarray(arrivals).reshape(-1, 3)[idx],
                           precision=precision, mode=L.MODE_FAST if mode is None else mode)
    return RowBlock.of_rows(rows, idx)
