"""Many independent volumes over several GPUs: one process per GPU, volumes
assigned by node count, no collective while the loops run, one host gather of
the relaxed nodes at the end.

A single volume does not shard (every iteration reads neighbours' positions,
so a split needs a halo exchange per iteration); it runs as replicas. A batch
of independent volumes does: each rank relaxes its share with
relax_cl_batch on its own GPU.
"""
from __future__ import annotations

from typing import Callable, Sequence

from .types import Grid, Nodes, RelaxParams, RelaxStats


def assign_volumes(node_counts: Sequence[int], world: int) -> list[list[int]]:
    """Greedy longest-processing-time assignment: volumes by node count,
    largest first, each to the least-loaded rank (ties: the lower rank; equal
    counts keep their input order). Deterministic: every rank computes the same
    assignment from the same counts. Returns each rank's volume indices, ascending."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(node_counts)), key=lambda v: (-int(node_counts[v]), v))
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for v in order:
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(v)
        load[r] += int(node_counts[v])
    return [sorted(x) for x in out]


def relax_batch_distributed(grids: Sequence[Grid], prms: Sequence[RelaxParams], nodes: Sequence[Nodes],
                            device: int = -1, group=None,
                            relax_fn: Callable | None = None) -> list[RelaxStats]:
    """Relax every volume of the batch, each on one rank of the process group
    (torch.distributed, already initialised); on return every rank holds all
    relaxed nodes (updated in place) and all stats.

    relax_fn(grids, prms, nodes, device) -> stats relaxes one rank's share; the
    default is relax_cl_batch (one set of launches for the share)."""
    import torch.distributed as dist

    if relax_fn is None:
        from .relax import relax_cl_batch as relax_fn
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    mine = assign_volumes([nd.size() for nd in nodes], world)[rank]
    stats_mine = []
    if mine:
        stats_mine = relax_fn([grids[v] for v in mine], [prms[v] for v in mine], [nodes[v] for v in mine], device)
    payload = {v: (nodes[v].P, nodes[v].typ, nodes[v].part, st) for v, st in zip(mine, stats_mine)}
    gathered = [None] * world
    dist.all_gather_object(gathered, payload, group=group)
    stats: list[RelaxStats | None] = [None] * len(nodes)
    for part in gathered:
        for v, (P, typ, prt, st) in part.items():
            nodes[v].P[...] = P
            nodes[v].typ[...] = typ
            nodes[v].part[...] = prt
            stats[v] = st
    return stats
