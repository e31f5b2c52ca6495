"""Multi-GPU ensembles: whole members are dealt out to ranks, none is split.

A member's step costs in proportion to its grid points, so members are assigned
greedily, largest grid first, each to the rank with the least work so far (ties
to the lower rank).  The assignment is deterministic, so every rank computes the
same table without communicating.  There is no exchange on the data path; the
per-member diagnostics are gathered to rank 0 on the host afterwards.
"""
from __future__ import annotations

from typing import Dict, List, Sequence


def shard_members(cells: Sequence[int], world: int) -> List[List[int]]:
    """Member indices per rank (each list in ascending order) for members of
    `cells` grid points each."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    out: List[List[int]] = [[] for _ in range(world)]
    for m in sorted(range(len(cells)), key=lambda i: (-cells[i], i)):
        r = min(range(world), key=lambda k: (load[k], k))
        out[r].append(m)
        load[r] += cells[m]
    return [sorted(x) for x in out]


def gather_by_member(local: Dict[int, object], n_members: int, group=None):
    """Rank 0 receives every rank's {member: value} and returns the values in
    member order; other ranks return None.  Host-side (torch.distributed
    all_gather_object), outside any timed region."""
    import torch.distributed as dist

    if not dist.is_initialized() or dist.get_world_size(group) == 1:
        return [local[m] for m in range(n_members)]
    rank = dist.get_rank(group)
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)  # also supported by the NCCL backend
    if rank != 0:
        return None
    merged: Dict[int, object] = {}
    for p in parts:
        merged.update(p)
    if sorted(merged) != list(range(n_members)):
        raise RuntimeError("gathered members do not cover the ensemble")
    return [merged[m] for m in range(n_members)]
