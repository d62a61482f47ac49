"""Run-axis chunking and host staging for batches larger than the device
memory budget.

The reference sizes chunks from its memory manager's VRAM share
(``mem_manager.py:1850-2133``: ``allocate_queue``, ``get_chunk_parameters``)
and runs one launch per chunk with host staging and a write-back thread
(``BatchSolverKernel._execute_run``, ``BatchSolverKernel.py:606-773``;
``writeback_watcher.py``).  Here:

* :func:`plan_chunks` turns the per-run device footprint of a prepared
  launch (inputs, per-run arrays, every output) and a byte budget into a
  chunk size (a multiple of 32 runs);
* :func:`device_budget` is the budget: ``mem_proportion`` of the device's
  total memory (the reference's manual proportion) or, with
  ``mem_proportion=None``, 90 % of what is free, never more than is free;
* :func:`run_chunked` integrates the batch chunk by chunk with two buffer
  slots on two streams: while one slot's kernel runs, the other slot's
  outputs come back and its next inputs go up, through pinned staging
  buffers.  Results land in host arrays of the full batch, or, above
  ``host_spill_threshold`` bytes, in memory-mapped files (the reference's
  host spill).  Runs are independent, so a chunked solve returns exactly
  the unchunked result.
"""

from __future__ import annotations

import math
import os
import tempfile
from dataclasses import dataclass
from typing import Any, Dict, List, Optional, Tuple

import numpy as np

@dataclass
class ChunkPlan:
    n_runs: int
    chunk_runs: int
    bytes_per_run: int
    budget: int

    @property
    def n_chunks(self) -> int:
        return max(1, math.ceil(self.n_runs / self.chunk_runs)) if self.n_runs else 1

    def bounds(self) -> List[Tuple[int, int]]:
        return [(c0, min(c0 + self.chunk_runs, self.n_runs)) for c0 in range(0, self.n_runs, self.chunk_runs)]


def output_shapes(solver, prep, n_runs: int) -> Dict[str, Tuple[Tuple[int, ...], Any]]:
    """Shape and numpy dtype of every output array of a launch of
    ``n_runs`` runs (the layout ``Solver.allocate_outputs`` creates)."""
    spec = prep["spec"]
    p = np.dtype(solver.precision)
    n_save, n_summ = prep["n_save"], prep["n_summ"]
    width = (len(spec.saved_state_indices) if spec.save_state else 0) + (1 if spec.save_time else 0)
    per_var = spec.summary.output_per_var if spec.summary else 0
    shapes: Dict[str, Tuple[Tuple[int, ...], Any]] = {}
    if width:
        shapes["state"] = ((n_save, width, n_runs), p)
    if spec.save_observables:
        shapes["obs"] = ((n_save, len(spec.saved_observable_indices), n_runs), p)
    if spec.summarised_state_indices and per_var:
        shapes["state_sum"] = ((n_summ, len(spec.summarised_state_indices) * per_var, n_runs), p)
    if spec.summarised_observable_indices and per_var:
        shapes["obs_sum"] = ((n_summ, len(spec.summarised_observable_indices) * per_var, n_runs), p)
    if spec.save_counters:
        shapes["counters"] = ((n_save, 4, n_runs), np.dtype(np.int32))
    shapes["status"] = ((n_runs,), np.dtype(np.int32))
    return shapes


def bytes_per_run(solver, prep, per_run_arrays: int = 0) -> int:
    """Device bytes one run needs: initial values, parameters, every output
    and ``per_run_arrays`` float64 per-run inputs (horizon, tolerance
    scale) plus the int64 claim order."""
    itemsize = np.dtype(solver.precision).itemsize
    sysm = solver.system
    total = (sysm.num_states + max(sysm.num_parameters, 1)) * itemsize
    total += 8 * per_run_arrays + (8 if per_run_arrays else 0)
    for shape, dt in output_shapes(solver, prep, 1).values():
        total += int(np.prod(shape)) * np.dtype(dt).itemsize
    return total


def device_budget(device: int, mem_proportion: Optional[float]) -> int:
    """Bytes a solve may hold on ``device``."""
    import torch
    free, total = torch.cuda.mem_get_info(device)
    if mem_proportion is None:
        return int(0.9 * free)
    return int(min(float(mem_proportion) * total, free))


def plan_chunks(n_runs: int, per_run: int, budget: int, max_chunk_runs: Optional[int] = None) -> ChunkPlan:
    """One chunk when the whole batch fits ``budget`` (and
    ``max_chunk_runs``); otherwise the largest chunk, a multiple of 32 runs
    and at least 32, of which two (the two slots in flight) fit."""
    if per_run <= 0:
        raise ValueError("per-run footprint must be positive")
    cap = None if max_chunk_runs is None else max(32, (int(max_chunk_runs) + 31) // 32 * 32)
    if n_runs * per_run <= budget and (cap is None or n_runs <= cap):
        return ChunkPlan(n_runs=n_runs, chunk_runs=max(n_runs, 1), bytes_per_run=per_run, budget=budget)
    fit = max(32, (budget // (2 * per_run)) // 32 * 32)
    if cap is not None:
        fit = min(fit, cap)
    chunk = min(fit, max(n_runs, 1))
    return ChunkPlan(n_runs=n_runs, chunk_runs=max(chunk, 1), bytes_per_run=per_run, budget=budget)


def host_outputs(shapes, spill_threshold: Optional[int], spill_dir: Optional[str]) -> Dict[str, np.ndarray]:
    """Full-batch host arrays for the outputs; memory-mapped files in
    ``spill_dir`` when their total exceeds ``spill_threshold`` bytes."""
    total = sum(int(np.prod(s)) * np.dtype(dt).itemsize for s, dt in shapes.values())
    spill = spill_threshold is not None and total > int(spill_threshold)
    out: Dict[str, np.ndarray] = {}
    if spill:
        root = tempfile.mkdtemp(prefix="cubie_b200_spill_", dir=spill_dir)
    for key, (shape, dt) in shapes.items():
        if spill:
            path = os.path.join(root, f"{key}.bin")
            arr = np.memmap(path, dtype=dt, mode="w+", shape=shape)
            arr.spill_path = path
            out[key] = arr
        else:
            out[key] = np.zeros(shape, dtype=dt)
    return out


class _Slot:
    """Device buffers, pinned staging and a stream for one chunk in flight."""

    def __init__(self, solver, prep, chunk_runs, dev, tdtype, n_states, n_params, per_run_flags, coeff_t):
        import torch
        self.stream = torch.cuda.Stream(device=dev)
        self.done = torch.cuda.Event()
        self.bufs = solver.allocate_outputs(prep, chunk_runs, dev, tdtype)
        self.inits_d = torch.zeros((n_states, chunk_runs), dtype=tdtype, device=dev)
        self.params_d = torch.zeros((n_params, chunk_runs), dtype=tdtype, device=dev)
        self.inits_h = torch.zeros((n_states, chunk_runs), dtype=tdtype).pin_memory()
        self.params_h = torch.zeros((n_params, chunk_runs), dtype=tdtype).pin_memory()
        self.dur_d = self.dur_h = self.tol_d = self.tol_h = None
        if per_run_flags[0]:
            self.dur_d = torch.zeros((chunk_runs,), dtype=torch.float64, device=dev)
            self.dur_h = torch.zeros((chunk_runs,), dtype=torch.float64).pin_memory()
        if per_run_flags[1]:
            self.tol_d = torch.ones((chunk_runs,), dtype=torch.float64, device=dev)
            self.tol_h = torch.ones((chunk_runs,), dtype=torch.float64).pin_memory()
        self.out_h = {k: torch.zeros(tuple(v.shape), dtype=v.dtype).pin_memory()
                      for k, v in self.bufs.items() if v is not None and k != "work"}
        self.coeff_t = coeff_t
        self.pending: Optional[Tuple[int, int]] = None


def run_chunked(solver, prep, inits, params, coeff_t, plan: ChunkPlan, duration, settling_time, t0,
                durations=None, tol_scale=None, nan_error_trajectories=True):
    """Integrate ``plan.n_runs`` runs chunk by chunk (see the module
    docstring) and return the full :class:`SolveResult`."""
    import torch
    dev = torch.device("cuda", solver.device)
    tdtype = torch.float32 if solver.precision == np.float32 else torch.float64
    n_runs, chunk = plan.n_runs, plan.chunk_runs
    n_states = solver.system.num_states
    n_params = max(solver.system.num_parameters, 1)

    def host_input(x, rows):
        if x is None:
            return np.zeros((rows, n_runs), dtype=solver.precision)
        if torch.is_tensor(x):
            return x  # device or host tensor; sliced per chunk below
        return np.asarray(x, dtype=solver.precision)

    inits_src = host_input(inits, n_states)
    params_src = host_input(params, n_params) if (params is not None and np.size(params)) else \
        np.zeros((n_params, n_runs), dtype=solver.precision)
    dur_src = None if durations is None else (durations if torch.is_tensor(durations)
                                              else np.asarray(durations, dtype=np.float64).reshape(-1))
    tol_src = None if tol_scale is None else (tol_scale if torch.is_tensor(tol_scale)
                                              else np.asarray(tol_scale, dtype=np.float64).reshape(-1))
    flags = (dur_src is not None, tol_src is not None)
    slots = [_Slot(solver, prep, chunk, dev, tdtype, n_states, n_params, flags, coeff_t) for _ in range(2)]
    host = host_outputs(output_shapes(solver, prep, n_runs), solver.host_spill_threshold, solver.spill_dir)
    totals = np.zeros(4, dtype=np.int64)

    def stage(dst_h, src, c0, c1):
        m = c1 - c0
        if torch.is_tensor(src):
            dst_h[..., :m].copy_(src[..., c0:c1])
        else:
            dst_h.numpy()[..., :m] = src[..., c0:c1]

    kernel_ms = [0.0]

    def drain(slot):
        if slot.pending is None:
            return
        slot.done.synchronize()
        e0, e1 = slot.timing
        kernel_ms[0] += e0.elapsed_time(e1)
        c0, c1 = slot.pending
        m = c1 - c0
        for key, h in slot.out_h.items():
            if key == "totals":
                continue
            if key in host:
                host[key][..., c0:c1] = h.numpy()[..., :m]
        totals[:] += slot.out_h["totals"].numpy()
        slot.pending = None

    for ci, (c0, c1) in enumerate(plan.bounds()):
        slot = slots[ci % 2]
        drain(slot)
        m = c1 - c0
        stage(slot.inits_h, inits_src, c0, c1)
        stage(slot.params_h, params_src, c0, c1)
        if slot.dur_h is not None:
            stage(slot.dur_h, dur_src, c0, c1)
        if slot.tol_h is not None:
            stage(slot.tol_h, tol_src, c0, c1)
        with torch.cuda.stream(slot.stream):
            slot.inits_d.copy_(slot.inits_h, non_blocking=True)
            slot.params_d.copy_(slot.params_h, non_blocking=True)
            dur_t = tol_t = None
            if slot.dur_d is not None:
                slot.dur_d.copy_(slot.dur_h, non_blocking=True)
                dur_t = slot.dur_d[:m]
            if slot.tol_d is not None:
                slot.tol_d.copy_(slot.tol_h, non_blocking=True)
                tol_t = slot.tol_d
            slot.bufs["totals"].zero_()
            order = solver.run_order(dur_t, tol_t[:m] if tol_t is not None else None) \
                if dur_t is not None else None
            args = solver.make_args(prep, slot.bufs, slot.inits_d, slot.params_d, coeff_t, m, duration,
                                    settling_time, t0, slot.dur_d if dur_t is not None else None, tol_t,
                                    order_t=order, run_stride=chunk)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(slot.stream)
            prep["module"].launch(args, solver.launch_kind, solver.block_size, 0, slot.stream.cuda_stream)
            e1.record(slot.stream)
            for key, h in slot.out_h.items():
                h.copy_(slot.bufs[key], non_blocking=True)
            slot.done.record(slot.stream)
        slot.pending = (c0, c1)
        slot.timing = (e0, e1)
    for slot in slots:
        drain(slot)
    host["totals"] = totals
    solver.chunks = plan.n_chunks
    solver.last_kernel_ms = kernel_ms[0]
    return solver.collect(prep, None, n_runs, duration, settling_time, t0, nan_error_trajectories,
                          on_device=False, host_arrays=host)
