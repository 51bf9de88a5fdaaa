"""Batched instances split across GPUs, one process per GPU.

The batched workload is a list of independent QPs, so it partitions with
no data exchange during the solve: every rank takes a bin of instances,
solves it with its own persistent batched kernel on its own GPU's memory
(``pdhcg_b200_solve_batch``), and the only collective is the gather of the
results to rank 0 at the end.  Bins are balanced by the instances' nonzero
counts (the batched kernel's work per iteration is proportional to them),
with the longest-processing-time rule: instances in decreasing weight,
each to the currently lightest bin (ties: lowest rank).  The partition is a
pure function of the weights, so every rank computes the same one without
communicating.

The reference has no batched solver; its distributed path
(``solve_qp_problem_distributed``) splits ONE problem over a 2-D process
grid with an NCCL all-reduce per product, which this library does not
implement (single-instance solves run as replicas).
"""
from __future__ import annotations

import heapq
from typing import Callable, Sequence


def partition(weights: Sequence[float], parts: int) -> list[list[int]]:
    """Indices 0..len(weights)-1 split into ``parts`` bins of nearly equal
    total weight; each bin lists its indices in increasing order."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(weights)), key=lambda i: (-float(weights[i]), i))
    heap = [(0.0, r) for r in range(parts)]
    bins: list[list[int]] = [[] for _ in range(parts)]
    for i in order:
        load, r = heapq.heappop(heap)
        bins[r].append(i)
        heapq.heappush(heap, (load + float(weights[i]), r))
    for b in bins:
        b.sort()
    return bins


def gather_results(local: dict, rank: int, world: int, count: int, group=None) -> list | None:
    """Collect {global index: result} from every rank on rank 0 and return
    the results in the batch's order (None on the other ranks).  Every
    index must arrive exactly once."""
    import torch.distributed as dist
    parts = [None] * world if rank == 0 else None
    if world > 1:
        dist.gather_object(local, parts, dst=0, group=group)
    else:
        parts = [local]
    if rank != 0:
        return None
    out: list = [None] * count
    seen = 0
    for part in parts:
        for i, res in part.items():
            if out[i] is not None:
                raise RuntimeError(f"instance {i} was solved on two ranks")
            out[i] = res
            seen += 1
    if seen != count:
        raise RuntimeError(f"{count - seen} instances were not solved")
    return out


def solve_batch_sharded(weights: Sequence[float], build: Callable[[list[int]], list], params: dict | None = None,
                        solver: Callable | None = None, rank: int = 0, world: int = 1, group=None) -> list | None:
    """Solve one batch split across ``world`` ranks.

    ``weights[i]`` is instance i's weight (its nonzero count); ``build(idx)``
    returns the problems with global indices ``idx`` (each rank builds only
    its own bin); ``solver(problems, params)`` returns one result per
    problem (default: ``native.solve_batch``, the persistent batched kernel
    on this rank's current device).  Returns the results of the whole batch
    in order on rank 0, None elsewhere."""
    if solver is None:
        from . import native
        solver = native.solve_batch
    bins = partition(weights, world)
    mine = bins[rank]
    results = solver(build(mine), params) if mine else []
    return gather_results(dict(zip(mine, results)), rank, world, len(weights), group)
