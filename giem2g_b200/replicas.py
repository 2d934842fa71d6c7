"""Replica parallelism: independent (frequency x polarisation) IE solves spread over ranks.

The reference runs one frequency at a time over all MPI ranks and shards the operator in y
(giem2g.F90:336-373 loops frequencies and polarisations; Distributed_FFT.F90 transposes between
slabs).  On B200 one instance fits one GPU (128x128x32: 0.55 GB complex64 tensor), so the
instances themselves are the unit of parallelism: rank r of W takes instances r, r+W, r+2W, ...
of the row-major (frequency, polarisation) list, builds the Green's tensor of each of its
frequencies on its own GPU and solves; there is no collective on the data path.  The only
communication is the barrier around timed regions, the max over ranks of a device time, and the
final gather of the per-instance results to rank 0.
"""
from __future__ import annotations

from typing import Callable, Sequence


def instances(freqs: Sequence[float], pols: Sequence[int]) -> list[tuple[int, int]]:
    """Row-major (frequency index, polarisation) list, the order giem2g.F90:336-373 visits."""
    return [(fi, p) for fi in range(len(freqs)) for p in pols]


def shard(n: int, rank: int, world: int) -> list[int]:
    """Round-robin instance indices owned by `rank` (every index in exactly one rank)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return list(range(rank, n, world))


def max_over_ranks(x: float, device=None) -> float:
    """Max of a per-rank time over the default process group (identity without one)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_sweep(solve_one: Callable[[int, int], object], freqs: Sequence[float], pols: Sequence[int],
              rank: int = 0, world: int = 1) -> dict[tuple[int, int], object] | None:
    """Solve this rank's share of the sweep; rank 0 returns {(fi, pol): result} for all instances.

    `solve_one(fi, pol)` runs one instance on this rank's GPU and returns a picklable result.
    Frequencies are visited in order so a rank builds each of its tensors once.
    """
    import torch.distributed as dist
    todo = instances(freqs, pols)
    mine = {todo[i]: solve_one(*todo[i]) for i in shard(len(todo), rank, world)}
    if world == 1:
        return mine
    parts = [None] * world if rank == 0 else None
    dist.gather_object(mine, parts, dst=0)
    if rank != 0:
        return None
    out = {}
    for p in parts:
        out.update(p)
    return out
