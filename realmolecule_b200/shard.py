"""Batched instances over several GPUs: one process per GPU, instances partitioned by cost.

Independent instances (molecules or clusters of one batch) share nothing while they are solved,
so the multi-GPU path has no data-path collective: every rank builds a ``Batch`` of its own
share on its own GPU, solves it, and the per-instance results are gathered to every rank with
one ``all_gather_object`` at the end.  The partition balances the estimated cost of a share,
the instance's voxel count (every kernel of a step streams the whole grid), by longest
processing time first: instances in decreasing cost, each to the currently lightest rank, ties
to the lowest rank -- deterministic, so every rank computes the same partition without talking.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

import numpy as np


def instance_cost(inst: dict) -> int:
    """Voxels of the instance's grid, (NN+1)^3."""
    return (int(inst["NN"]) + 1) ** 3


def partition(costs: Sequence[float], parts: int) -> List[List[int]]:
    """Longest-processing-time partition of instance indices into ``parts`` lists.

    Each list is in increasing index order.  Raises ValueError for parts < 1."""
    if parts < 1:
        raise ValueError("parts must be >= 1")
    order = sorted(range(len(costs)), key=lambda q: (-costs[q], q))
    load = [0.0] * parts
    out: List[List[int]] = [[] for _ in range(parts)]
    for q in order:
        r = min(range(parts), key=lambda x: (load[x], x))
        out[r].append(q)
        load[r] += costs[q]
    return [sorted(x) for x in out]


def my_share(instances: Sequence[dict], rank: int, world: int) -> List[int]:
    """Indices of the instances rank ``rank`` of ``world`` solves."""
    if not 0 <= rank < world:
        raise ValueError(f"rank {rank} outside [0, {world})")
    return partition([instance_cost(i) for i in instances], world)[rank]


def batch_solver(precision: str = "mixed", tol_dE: float = 1e-6, max_steps: int = 40000, check_interval: int = 100,
                 stream: Optional[int] = None, **opts) -> Callable[[Sequence[dict]], Tuple[np.ndarray, np.ndarray]]:
    """A solve function for ``solve_sharded``: one ``Batch`` of the share, initialise, solve."""
    def solve(share: Sequence[dict]):
        from .batch import Batch
        b = Batch(share, precision=precision, **opts)
        try:
            if stream is not None:
                b.set_stream(stream)
            b.initialize()
            return b.solve(tol_dE, max_steps, check_interval)
        finally:
            b.close()
    return solve


def solve_sharded(instances: Sequence[dict], solve: Callable[[Sequence[dict]], Tuple[np.ndarray, np.ndarray]],
                  group=None) -> Tuple[np.ndarray, np.ndarray]:
    """Solve ``instances`` split over the ranks of ``group`` (torch.distributed, any backend).

    ``solve(share)`` returns (steps to converge, energies) for the share, in share order.  Every
    rank returns the full arrays in instance order.  Without an initialised process group the
    whole list is solved here."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        conv, E = solve(list(instances))
        return np.asarray(conv), np.asarray(E, dtype=np.float64)
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    idx = my_share(instances, rank, world)
    conv, E = solve([instances[q] for q in idx]) if idx else (np.zeros(0, np.int32), np.zeros(0))
    mine = (idx, np.asarray(conv).tolist(), np.asarray(E, dtype=np.float64).tolist())
    gathered: List = [None] * world
    dist.all_gather_object(gathered, mine, group=group)
    conv_all = np.full(len(instances), -1, np.int32)
    E_all = np.full(len(instances), np.nan)
    for ids, c, e in gathered:
        conv_all[ids] = c
        E_all[ids] = e
    return conv_all, E_all
