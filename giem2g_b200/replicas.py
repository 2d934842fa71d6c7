"""Replica parallelism: independent (frequency x polarisation) IE solves spread over ranks.

The reference runs one frequency at a time over all MPI ranks and shards the operator in y
(giem2g.F90:336-373 loops frequencies and polarisations; Distributed_FFT.F90 transposes between
slabs).  On B200 one instance fits one GPU (128x128x32: 0.55 GB complex64 tensor), so the
frequencies themselves are the unit of parallelism: rank r of W takes frequencies r, r+W, r+2W, ...
and solves every polarisation of each of them, so the two polarisations of a frequency share one
Green's tensor build and, in the batched solver, every tensor read of their paired applies.  There
is no collective on the data path.  The only communication is the barrier around timed regions, the
max over ranks of a device time, and the final gather of the per-instance results to rank 0.
"""
from __future__ import annotations

from typing import Callable, Sequence


def instances(freqs: Sequence[float], pols: Sequence[int]) -> list[tuple[int, int]]:
    """Row-major (frequency index, polarisation) list, the order giem2g.F90:336-373 visits."""
    return [(fi, p) for fi in range(len(freqs)) for p in pols]


def shard(n: int, rank: int, world: int) -> list[int]:
    """Round-robin indices owned by `rank` (every index in exactly one rank)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError(f"bad rank {rank} of {world}")
    return list(range(rank, n, world))


def shard_instances(freqs: Sequence[float], pols: Sequence[int], rank: int, world: int) -> list[tuple[int, int]]:
    """The (frequency index, polarisation) instances of `rank`: its round-robin share of the frequencies, each
    with all of its polarisations, in the reference's visiting order."""
    mine = set(shard(len(freqs), rank, world))
    return [(fi, p) for fi, p in instances(freqs, pols) if fi in mine]


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

    `solve_one(fi, pol)` runs one instance on this rank's GPU and returns a picklable result.  A rank owns
    whole frequencies (all polarisations) and visits them in order, so it builds each of its tensors once.
    """
    import torch.distributed as dist
    mine = {key: solve_one(*key) for key in shard_instances(freqs, pols, rank, world)}
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
