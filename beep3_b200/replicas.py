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


class ReplicaError(RuntimeError):
    """Raised on rank 0 when work items failed on some rank; ``failures``
    maps item index -> (rank, error text)."""

    def __init__(self, failures: dict[int, tuple[int, str]]):
        lines = [f"item {i} on rank {r}: {msg}" for i, (r, msg) in sorted(failures.items())]
        super().__init__("replicated work failed:\n  " + "\n  ".join(lines))
        self.failures = failures


def run_replicated(items: Sequence[Any], fn: Callable[[Any], Any], dist=None) -> list[Any] | None:
    """Runs ``fn`` over this rank's share and gathers all results on rank 0
    in item order (None on the other ranks).  ``dist`` is torch.distributed
    (already initialised) or None for a single process.

    An item whose ``fn`` raises does not take its rank out of the gather:
    the rank reports the error text instead of a result, the gather
    completes on every rank, and rank 0 raises ReplicaError naming the
    failed items.  (A rank that dies outright is caught by the process
    group's timeout, which the caller sets.)"""
    if dist is None or not dist.is_initialized():
        return [fn(it) for it in items]
    rank, world = dist.get_rank(), dist.get_world_size()
    mine = []
    for i, it in shard(items, rank, world):
        try:
            mine.append((i, True, fn(it)))
        except Exception as e:  # reported to rank 0, not raised here
            mine.append((i, False, f"{type(e).__name__}: {e}"))
    gathered = [None] * world if rank == 0 else None
    dist.gather_object(mine, gathered, dst=0)
    if rank != 0:
        return None
    out: list[Any] = [None] * len(items)
    failures: dict[int, tuple[int, str]] = {}
    for r, part in enumerate(gathered):
        for i, ok, v in part:
            if ok:
                out[i] = v
            else:
                failures[i] = (r, v)
    if failures:
        raise ReplicaError(failures)
    return out
