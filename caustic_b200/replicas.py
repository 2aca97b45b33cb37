"""Independent solves spread over the ranks of a job (one process per GPU).

One SDOT solve does not shard: every L-BFGS iteration needs global dot
products and a single evaluation needs the whole density.  What scales over
GPUs is a set of independent instances (batches of problems, data
generation for a warm start): each rank takes its share, solves it on its own
GPU, and the results are gathered on the host.  The only communication is
that gather (and barriers); there is no collective in the solve itself.
"""
from __future__ import annotations

from typing import Callable, List, Sequence


def shard(n_items: int, rank: int, world: int) -> List[int]:
    """Indices of the items this rank solves (round robin, so uneven
    instance sizes spread evenly)."""
    if world <= 0 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    return list(range(rank, n_items, world))


def solve_replicas(items: Sequence, solve: Callable, group=None) -> list:
    """Solve `items` across the ranks of `group` (torch.distributed, any
    backend) and return all results, in item order, on every rank.  Without
    an initialised process group everything runs locally."""
    import torch.distributed as dist

    if not (dist.is_available() and dist.is_initialized()):
        return [solve(x) for x in items]
    rank = dist.get_rank(group)
    world = dist.get_world_size(group)
    mine = {i: solve(items[i]) for i in shard(len(items), rank, world)}
    gathered = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    out = [None] * len(items)
    for part in gathered:
        for i, v in part.items():
            out[i] = v
    return out
