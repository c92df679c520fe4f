"""Multi-GPU plumbing of the batched form: whole cases are assigned to ranks
(one process per GPU) by cell count, each rank runs its own batch with no
collective during the iterations, and the end-of-run figures are reduced on
the host side of ``torch.distributed`` (NCCL on GPUs, gloo in the CPU tests).

A single mesh is not split: its LU-SGS sweeps are one Gauss-Seidel order,
which a domain decomposition would turn into block Jacobi.
"""
from __future__ import annotations

from typing import Sequence


def assign_cases(cells: Sequence[int], world: int) -> list[int]:
    """Rank of every case: cases in decreasing cell count (ties: lower case
    index first), each to the least-loaded rank (ties: lower rank).  The
    largest load then exceeds the mean by less than the largest case."""
    if world < 1:
        raise ValueError("world size must be at least 1")
    load = [0] * world
    owner = [0] * len(cells)
    for k in sorted(range(len(cells)), key=lambda i: (-int(cells[i]), i)):
        r = min(range(world), key=lambda j: (load[j], j))
        owner[k] = r
        load[r] += int(cells[k])
    return owner


def rank_cases(cells: Sequence[int], world: int, rank: int) -> list[int]:
    """Indices of the cases of `rank`, in case order."""
    owner = assign_cases(cells, world)
    return [k for k, r in enumerate(owner) if r == rank]


def _reduce(value: float, dist, device, op_name: str) -> float:
    if dist is None:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=getattr(dist.ReduceOp, op_name))
    return float(t.item())


def reduce_max(value: float, dist=None, device="cpu") -> float:
    """Largest value over the ranks (device times: the job ends with its
    slowest rank)."""
    return _reduce(value, dist, device, "MAX")


def reduce_sum(value: float, dist=None, device="cpu") -> float:
    """Sum over the ranks (cells, cell-updates)."""
    return _reduce(value, dist, device, "SUM")
