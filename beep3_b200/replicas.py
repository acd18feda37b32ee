"""Multi-GPU execution as independent replicas.

The BEM matvec of one scenario does not shard (every GMRES step needs the
whole surface), so several GPUs run independent work items -- poses of a
rigid-body scan, requests of a stream -- one process per GPU, with no
collective on the data path.  This module splits a list of work items over
the ranks of a ``torch.distributed`` group and gathers the per-item results
(small host objects) on rank 0 after the work is done.
"""
from __future__ import annotations

from typing import Any, Callable, Sequence


def shard(items: Sequence[Any], rank: int, world: int) -> list[tuple[int, Any]]:
    """Round-robin split: rank r gets items r, r + world, ... with their index."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    return [(i, it) for i, it in enumerate(items) if i % world == rank]


def run_replicated(items: Sequence[Any], fn: Callable[[Any], Any], dist=None) -> list[Any] | None:
    """Runs ``fn`` over this rank's share and gathers all results on rank 0
    in item order (None on the other ranks).  ``dist`` is torch.distributed
    (already initialised) or None for a single process."""
    if dist is None or not dist.is_initialized():
        return [fn(it) for it in items]
    rank, world = dist.get_rank(), dist.get_world_size()
    mine = [(i, fn(it)) for i, it in shard(items, rank, world)]
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out: list[Any] = [None] * len(items)
    for part in gathered:
        for i, r in part:
            out[i] = r
    return out
