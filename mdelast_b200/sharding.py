"""Replicas across GPUs: independent cells, no exchange during a step.

The path does not shard within a cell (cells of up to ~10^5 atoms fit one GPU many times
over); several GPUs each advance their own batch of replicas. ``shard_replicas`` deals
replicas to ranks by size (largest first onto the least-loaded rank), deterministically,
and ``gather_observables`` collects per-replica results on every rank after a run (one
host-side all_gather; nothing on the step path).
"""

from __future__ import annotations


def shard_replicas(sizes, world: int) -> list[list[int]]:
    """Indices of the replicas each of `world` ranks advances; loads (atom counts) differ
    by at most the largest replica."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(sizes)), key=lambda k: (-sizes[k], k))
    load = [0] * world
    shards: list[list[int]] = [[] for _ in range(world)]
    for k in order:
        r = min(range(world), key=lambda q: (load[q], q))
        shards[r].append(k)
        load[r] += sizes[k]
    for s in shards:
        s.sort()
    return shards


def gather_observables(local: dict, group=None) -> dict:
    """Merge {replica index: observables} from every rank (torch.distributed)."""
    import torch.distributed as dist
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    out: dict = {}
    for p in parts:
        out.update(p)
    return out
