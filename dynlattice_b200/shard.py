"""Sharding of independent lattices over the ranks of one node (batched
impact workloads): each rank steps its own Batch with no collective in the
data path; results and timings are reduced on the host side at the end."""
from __future__ import annotations

from typing import List, Sequence


def partition_by_elements(sizes: Sequence[int], n_parts: int) -> List[List[int]]:
    """Longest-processing-time greedy: lattices by decreasing element count,
    each to the currently lightest part (ties: lower part index).  Returns the
    lattice indices of each part, ascending.  Deterministic."""
    if n_parts <= 0:
        raise ValueError("n_parts must be positive")
    order = sorted(range(len(sizes)), key=lambda i: (-int(sizes[i]), i))
    load = [0] * n_parts
    parts: List[List[int]] = [[] for _ in range(n_parts)]
    for i in order:
        p = min(range(n_parts), key=lambda q: (load[q], q))
        parts[p].append(i)
        load[p] += int(sizes[i])
    return [sorted(p) for p in parts]


def shard_for_rank(specs, rank: int, world: int):
    """(indices, specs) of the lattices this rank steps."""
    parts = partition_by_elements([s.n_elems for s in specs], world)
    idx = parts[rank]
    return idx, [specs[i] for i in idx]


def max_over_ranks(value: float) -> float:
    """Maximum of a host float over the default process group (any backend)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def sum_over_ranks(value: float) -> float:
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(value)
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(value)], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM)
    return float(t.item())
