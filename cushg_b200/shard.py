"""Splitting one batch of independent instances across ranks (one process per GPU).

The reference runs a parameter sweep as one process per point (src/cuSHG.sh:58-94).  The
instances never exchange data, so a batch shards with no collective on the data path: each
rank solves its share with shg_solve_batch_device, and only the scalars (SH powers) are
gathered at the end.  The split is greedy by cost N^2 * steps (longest first onto the least
loaded rank), deterministic, so every rank computes the same partition without talking.
"""
from __future__ import annotations

import numpy as np

from .params import ShgParams


def instance_cost(p: ShgParams) -> float:
    """Work of one instance: grid points times SSFM steps."""
    steps = p.nz if p.thermal else p.nz - 1
    return float(p.nx) * float(p.ny) * float(steps)


def partition(costs, world: int) -> list[list[int]]:
    """Greedy longest-first split of instances with the given costs over `world` ranks;
    returns each rank's instance indices in ascending order.  Ties go to the lower index and
    the lower rank, so every caller gets the same answer."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return [sorted(p) for p in parts]


def shard(ps: list[ShgParams], rank: int, world: int) -> tuple[list[int], list[ShgParams]]:
    """This rank's instance indices and parameter sets."""
    idx = partition([instance_cost(p) for p in ps], world)[rank]
    return idx, [ps[i] for i in idx]


def gather_powers(local_idx: list[int], local_powers, count: int, group=None) -> np.ndarray:
    """Collect every rank's (index, SH power) pairs into one array of `count` powers, in the
    batch's order, on every rank (torch.distributed all_gather_object: host scalars only)."""
    import torch.distributed as dist

    pairs = list(zip([int(i) for i in local_idx], [float(v) for v in local_powers]))
    world = dist.get_world_size(group)
    everything: list = [None] * world
    dist.all_gather_object(everything, pairs, group=group)
    out = np.full(count, np.nan)
    seen = np.zeros(count, dtype=bool)
    for part in everything:
        for i, v in part:
            if seen[i]:
                raise ValueError(f"instance {i} solved by two ranks")
            seen[i] = True
            out[i] = v
    if not seen.all():
        raise ValueError(f"instances {np.flatnonzero(~seen).tolist()} solved by no rank")
    return out
