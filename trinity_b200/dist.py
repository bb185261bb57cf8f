"""Multi-GPU plumbing for independent meshes (no collective on the data path).

A single mesh is adapted on one GPU: its updates are made conflict-free by
global independent sets, matchings and colorings, and the reference never
decomposes the domain. Several GPUs therefore run replicas or disjoint sets of
meshes; the only communication is the end-of-run reduction of timings and
counts, done here with torch.distributed (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

import numpy as np


def shard_meshes(sizes, world: int) -> list[list[int]]:
    """Assign mesh indices to ranks, largest first, each to the least loaded
    rank (ties to the lower rank): deterministic and balanced by size."""
    load = [0] * world
    out: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-sizes[k], k)):
        r = min(range(world), key=lambda q: (load[q], q))
        out[r].append(i)
        load[r] += sizes[i]
    for lst in out:
        lst.sort()
    return out


def reduce_stats(stats, sum_idx, max_idx, device="cpu"):
    """All-reduce a vector of per-rank statistics: entries in ``sum_idx`` are
    summed over ranks (work done), entries in ``max_idx`` take the maximum
    (time: the job ends with its slowest rank). Returns a numpy array."""
    import torch
    import torch.distributed as dist
    v = np.asarray(stats, dtype=np.float64)
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return v.copy()
    t = torch.tensor(v, device=device)
    s, m = t.clone(), t.clone()
    dist.all_reduce(s, op=dist.ReduceOp.SUM)
    dist.all_reduce(m, op=dist.ReduceOp.MAX)
    out = v.copy()
    for i in sum_idx:
        out[i] = s[i].item()
    for i in max_idx:
        out[i] = m[i].item()
    return out
