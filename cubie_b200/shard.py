"""Runs across GPUs: one process per GPU, each integrating its own shard.

Runs are independent, so a batch shards along the run axis with no
exchange during integration (the reference's equivalent is chunking the
run axis on one device, ``BatchSolverKernel._execute_run``,
src/cubie/batchsolving/BatchSolverKernel.py:606-754).  The only
collectives are after the launch: the slowest rank's time and the sum of
per-rank counts, so that a whole-job rate is total work / slowest rank.
"""

from __future__ import annotations

from typing import Optional, Sequence, Tuple

import numpy as np


def shard_bounds(n_total: int, rank: int, world: int) -> Tuple[int, int]:
    """Contiguous run range ``[start, stop)`` of ``rank``; sizes differ by at
    most one and the ranges tile ``[0, n_total)``."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    base, extra = divmod(int(n_total), int(world))
    start = rank * base + min(rank, extra)
    return start, start + base + (1 if rank < extra else 0)


def shard_columns(arrays: Sequence, rank: int, world: int) -> list:
    """The run columns of ``rank`` of every ``[rows, n_runs]`` array (or
    1-D per-run array) in ``arrays`` (None entries pass through)."""
    n = None
    for a in arrays:
        if a is not None:
            n = a.shape[-1]
            break
    if n is None:
        return list(arrays)
    lo, hi = shard_bounds(n, rank, world)
    return [None if a is None else a[..., lo:hi] for a in arrays]


def aggregate(ms: float, count: float, group=None, device=None) -> Tuple[float, float]:
    """(max over ranks of ``ms``, sum over ranks of ``count``) with
    ``torch.distributed``; the local pair when no process group is up."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()):
        return float(ms), float(count)
    t = torch.tensor([float(ms), float(count)], dtype=torch.float64, device=device)
    tm = t[:1].clone()
    ts = t[1:].clone()
    dist.all_reduce(tm, op=dist.ReduceOp.MAX, group=group)
    dist.all_reduce(ts, op=dist.ReduceOp.SUM, group=group)
    return float(tm[0]), float(ts[0])
