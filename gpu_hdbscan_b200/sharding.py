"""Independent clustering instances over several GPUs, one process per GPU.

The instances of a batch (hdb_run_batched) share nothing, so they spread over
the ranks with no data exchange on the device: each rank clusters its own
subset in shared launches, and only the per-instance labels travel, on the
host, to the rank that wants them.  The assignment is greedy size balancing
(longest processing time first): instances in descending size, each to the
rank with the fewest points so far.  Its most loaded rank carries at most the
least loaded one's points plus one instance, and at most 4/3 of the best
possible maximum.
"""
from __future__ import annotations

import heapq
from typing import Sequence


def assign_instances(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Instance indices per rank: descending size (ties by index) to the rank
    with the fewest assigned points (ties by the lower rank).  Each rank's list
    is in ascending instance order, so its instances keep their batch order."""
    if world < 1:
        raise ValueError("assign_instances: world must be at least 1")
    heap = [(0, r) for r in range(world)]
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda j: (-int(sizes[j]), j)):
        load, r = heapq.heappop(heap)
        parts[r].append(i)
        heapq.heappush(heap, (load + int(sizes[i]), r))
    return [sorted(p) for p in parts]


def rank_loads(sizes: Sequence[int], parts: list[list[int]]) -> list[int]:
    """Points assigned to each rank."""
    return [sum(int(sizes[i]) for i in p) for p in parts]


def gather_labels(labels_local, parts: list[list[int]], rank: int, dst: int = 0):
    """Host gather of per-instance labels to rank `dst` (torch.distributed must
    be initialised; any backend).  labels_local: this rank's label arrays in the
    order of parts[rank].  Returns, on dst, every instance's labels in instance
    order (a list of numpy arrays); None on the other ranks."""
    import numpy as np
    import torch.distributed as dist

    mine = [np.asarray(x.cpu() if hasattr(x, "cpu") else x, dtype=np.int32) for x in labels_local]
    if len(mine) != len(parts[rank]):
        raise ValueError("gather_labels: one label array per assigned instance")
    world = dist.get_world_size()
    got = [None] * world if rank == dst else None
    dist.gather_object(mine, got, dst=dst)
    if rank != dst:
        return None
    out = [None] * sum(len(p) for p in parts)
    for r in range(world):
        if len(got[r]) != len(parts[r]):
            raise RuntimeError(f"gather_labels: rank {r} sent {len(got[r])} arrays, "
                               f"{len(parts[r])} expected")
        for i, lab in zip(parts[r], got[r]):
            out[i] = lab
    return out
