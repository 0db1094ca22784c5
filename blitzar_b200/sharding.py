"""Multi-GPU layout for the gravity path: ranks own independent systems.

A single periodic or isolated system runs on one GPU (its force evaluation does not shard in
this engine); several GPUs run independent replicas or independent ensemble members, one
process per GPU, with no collective on the data path.  This module holds the host logic for
that layout: a longest-processing-time assignment of systems (e.g. star clusters of uneven
size) to ranks, and the end-of-run gather of per-rank diagnostics over torch.distributed.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_partition(costs, nranks: int):
    """Assign items with the given costs to nranks bins, largest first, each to the currently
    lightest bin (ties by lowest rank).  Deterministic; returns a list of index lists."""
    costs = np.asarray(costs, dtype=np.float64)
    if nranks <= 0:
        raise ValueError("nranks must be positive")
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    heap = [(0.0, r) for r in range(nranks)]
    heapq.heapify(heap)
    bins = [[] for _ in range(nranks)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + float(costs[i]), r))
    return [sorted(b) for b in bins]


def partition_loads(costs, bins):
    costs = np.asarray(costs, dtype=np.float64)
    return [float(costs[b].sum()) if len(b) else 0.0 for b in bins]


def gather_diagnostics(local: dict, group=None):
    """All-gather one small dict per rank (rank order).  Without an initialised process group
    returns [local]."""
    import torch.distributed as dist

    if not dist.is_available() or not dist.is_initialized():
        return [local]
    out = [None] * dist.get_world_size(group)
    dist.all_gather_object(out, local, group=group)
    return out


def particle_steps_per_second(particles_per_rank, steps: int, seconds_per_rank):
    """Whole-job throughput: all ranks' particle-steps over the slowest rank's time."""
    return float(np.sum(particles_per_rank)) * steps / float(np.max(seconds_per_rank))
