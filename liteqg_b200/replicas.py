"""Query sharding over replicated indexes (one process per GPU).

Queries are independent and an index fits one GPU, so N GPUs hold N copies of
the index and split the query stream; nothing on the data path crosses GPUs.
These helpers carry the host-side logic of that path:

* ``shard_bounds(m, rank, world)``: the contiguous query range of a rank;
* ``max_over_ranks(x)``: a timing taken on every rank reduced to its maximum
  (``torch.distributed`` all-reduce, any backend);
* ``search_sharded(search, queries, k)``: each rank searches its shard with
  ``search(q, k)`` and rank 0 receives all results in query order.
"""
from __future__ import annotations

import numpy as np


def shard_bounds(m: int, rank: int, world: int) -> tuple[int, int]:
    """[lo, hi) of rank's queries; the first m % world ranks take one more."""
    if world <= 0 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    base, extra = divmod(int(m), world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def _dist():
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return None
    return dist


def max_over_ranks(x: float, device=None) -> float:
    """The maximum of x over all ranks (x itself without a process group)."""
    dist = _dist()
    if dist is None:
        return float(x)
    import torch

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def search_sharded(search, queries: np.ndarray, k: int, dst: int = 0):
    """Runs ``search(shard, k)`` on this rank's shard; rank ``dst`` gets the
    results of all ranks concatenated in query order, the others None."""
    dist = _dist()
    if dist is None:
        return np.asarray(search(queries, k))
    rank, world = dist.get_rank(), dist.get_world_size()
    lo, hi = shard_bounds(len(queries), rank, world)
    mine = np.asarray(search(queries[lo:hi], k))
    parts = [None] * world if rank == dst else None
    dist.gather_object(mine, parts, dst=dst)
    if rank != dst:
        return None
    full = [p for p in parts if p is not None and len(p)]
    return np.concatenate(full, axis=0) if full else mine[:0]
