"""Replicas across GPUs for a list of spectra: one process per GPU, each
searching its own share of the list; no device collective on the data path.

The reference splits a file list over processes or CUDA devices
(python/parallel_search.py:18, 71-76, 209-218).  Here the list is
partitioned longest-processing-time first by trial count, so the ranks'
loads are even; each rank searches its files (e.g. with a Batch); the
candidate lists come back to every rank through one host-side object
all-gather (torch.distributed, gloo or nccl), reassembled in list order.
"""
from __future__ import annotations

from typing import Callable, Sequence


def lpt_partition(costs: Sequence[float], nparts: int) -> list[list[int]]:
    """Indices of `costs` split into `nparts` lists, largest first onto the
    least-loaded part; each list is returned in ascending index order."""
    if nparts < 1:
        raise ValueError("nparts must be >= 1")
    loads = [0.0] * nparts
    parts: list[list[int]] = [[] for _ in range(nparts)]
    for i in sorted(range(len(costs)), key=lambda i: (-costs[i], i)):
        k = min(range(nparts), key=lambda j: (loads[j], j))
        parts[k].append(i)
        loads[k] += costs[i]
    return [sorted(p) for p in parts]


def search_list(costs: Sequence[float], search: Callable[[list[int]], dict], dist=None) -> list:
    """Run `search(indices) -> {index: result}` on this rank's share and
    return every result in list order on every rank.  `dist` is an
    initialised torch.distributed module, or None for one process."""
    rank, world = (dist.get_rank(), dist.get_world_size()) if dist is not None else (0, 1)
    parts = lpt_partition(costs, world)
    mine = search(parts[rank])
    if set(mine) != set(parts[rank]):
        raise RuntimeError(f"rank {rank} returned results for the wrong files")
    if world == 1:
        merged = mine
    else:
        gathered: list = [None] * world
        dist.all_gather_object(gathered, mine)
        merged = {}
        for g in gathered:
            merged.update(g)
    return [merged[i] for i in range(len(costs))]
