"""Runs across GPUs: one process per GPU, each integrating its own shard.

Runs are independent, so a batch shards along the run axis with no
exchange during integration (the reference's equivalent is chunking the
run axis on one device, ``BatchSolverKernel._execute_run``,
src/cubie/batchsolving/BatchSolverKernel.py:606-754).  The only
collectives are after the launch: the slowest rank's time and the sum of
per-rank counts, so that a whole-job rate is total work / slowest rank.
"""

from __future__ import annotations

from typing import Callable, Dict, Optional, Sequence, Tuple

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


def interleaved_runs(n_total: int, rank: int, world: int) -> np.ndarray:
    """Run indices ``rank, rank + world, ...`` of a strided split: every
    rank gets the same mix of short and long runs (and, for a batch that
    concatenates several systems, of every system)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("rank must be in [0, world)")
    return np.arange(rank, int(n_total), world, dtype=np.int64)


def _take_runs(x, idx):
    if x is None:
        return None
    if hasattr(x, "index_select") and hasattr(x, "device"):
        import torch
        return x.index_select(x.dim() - 1, torch.as_tensor(idx, device=x.device, dtype=torch.long))
    return np.asarray(x)[..., idx]


def distributed_solve(solve: Callable, initial_values, parameters, per_run: Optional[Dict] = None,
                      group=None):
    """Integrate a batch across the ranks of a ``torch.distributed`` group,
    one process per GPU: each rank integrates its interleaved share of the
    runs with ``solve(inits, params, **per_run_share)`` (a SolveResult), and
    every rank returns the whole batch's SolveResult in the caller's run
    order.  The integration exchanges nothing; the results are gathered
    once at the end (``all_gather_object``: over NCCL or gloo).  Without an
    initialised group (or with one rank) it is ``solve`` itself."""
    import torch.distributed as dist
    per_run = dict(per_run or {})
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return solve(initial_values, parameters, **per_run)
    from .solveresult import merge_results
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    n = int(initial_values.shape[-1])
    idx = interleaved_runs(n, rank, world)
    share = {k: _take_runs(v, idx) for k, v in per_run.items()}
    local = solve(_take_runs(initial_values, idx), _take_runs(parameters, idx), **share)
    parts = [None] * world
    dist.all_gather_object(parts, local, group=group)
    return merge_results([(r, interleaved_runs(n, k, world)) for k, r in enumerate(parts)])
