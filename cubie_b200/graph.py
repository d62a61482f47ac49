"""Repeated solves of one batch shape as a single CUDA graph replay.

A :class:`GraphSolve` owns pinned host staging buffers and device buffers
for one ``(solver, n_runs, duration)`` and captures, once:

    host -> device copies of the initial values, parameters and (optional)
    per-run horizons and tolerance scales; zeroing of the work counter and
    iteration totals; the integration launch (persistent by default, with a
    fixed grid); device -> host copies of the saved states, summaries and
    status words.

Each call then writes new inputs into the pinned buffers, replays the graph
and waits for it: one submission per solve, no allocation, no Python-side
launch work.  This replaces the reference's per-chunk sequence of
transfers and launches (``BatchSolverKernel._execute_run``,
src/cubie/batchsolving/BatchSolverKernel.py:606-754) for callers that solve
the same batch shape repeatedly.  The module is compiled and loaded before
capture, so nothing is compiled, loaded or allocated while capturing.
"""

from __future__ import annotations

from typing import Optional

import numpy as np

from .solver import Solver, _torch


class GraphSolve:
    """Captured solve of ``n_runs`` runs over ``duration`` with ``solver``."""

    def __init__(self, solver: Solver, n_runs: int, duration: float, settling_time: float = 0.0,
                 t0: float = 0.0, per_run_durations: bool = False, per_run_tol_scale: bool = False,
                 kernel: Optional[str] = None, block: Optional[int] = None):
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("cubie_b200 needs a CUDA device: no GPU is visible")
        from . import _native
        self.solver = solver
        self.n_runs = int(n_runs)
        self.duration = float(duration)
        dev = torch.device("cuda", solver.device)
        self.device = dev
        p = solver.precision
        tdt = torch.float32 if p == np.float32 else torch.float64
        n, npar = solver.system.num_states, max(solver.system.num_parameters, 1)
        self.prep = prep = solver.prepare(duration, settling_time, t0,
                                          durations=np.zeros(1) if per_run_durations else None)
        self.kernel = solver.launch_kind if kernel is None else (1 if kernel == "persistent" else 0)
        self.block = int(block or solver.block_size)
        if self.kernel == 3:
            per_sm = prep["module"].occupancy(3, self.block)
            sms = _native.device_info(solver.device)["sm_count"]
            self.grid = max(1, min(max(per_sm, 1) * sms, (self.n_runs + self.block // 32 - 1) // (self.block // 32)))
        elif self.kernel == 1:
            per_sm = prep["module"].occupancy(1, self.block)
            sms = _native.device_info(solver.device)["sm_count"]
            self.grid = max(1, min(max(per_sm, 1) * sms, (self.n_runs + self.block - 1) // self.block))
        else:
            self.grid = (self.n_runs + self.block - 1) // self.block
        # pinned host staging and device buffers
        # staging starts zeroed: horizons of 0 end every run at once
        self.inits_h = torch.zeros((n, self.n_runs), dtype=tdt).pin_memory()
        self.params_h = torch.zeros((npar, self.n_runs), dtype=tdt).pin_memory()
        self.inits_d = torch.zeros((n, self.n_runs), dtype=tdt, device=dev)
        self.params_d = torch.zeros((npar, self.n_runs), dtype=tdt, device=dev)
        self.dur_h = torch.zeros((self.n_runs,), dtype=torch.float64).pin_memory() if per_run_durations else None
        self.dur_d = torch.zeros((self.n_runs,), dtype=torch.float64, device=dev) if per_run_durations else None
        self.tol_h = torch.ones((self.n_runs,), dtype=torch.float64).pin_memory() if per_run_tol_scale else None
        self.tol_d = torch.ones((self.n_runs,), dtype=torch.float64, device=dev) if per_run_tol_scale else None
        self.bufs = bufs = solver.allocate_outputs(prep, self.n_runs, dev, tdt)
        self.out_h = {k: torch.zeros(tuple(v.shape), dtype=v.dtype).pin_memory()
                      for k, v in bufs.items() if v is not None and k not in ("work",)}
        self.args = solver.make_args(prep, bufs, self.inits_d, self.params_d, None, self.n_runs, duration,
                                     settling_time, t0, self.dur_d, self.tol_d)
        self.graph = torch.cuda.CUDAGraph()
        stream = torch.cuda.Stream(device=dev)
        # One eager pass on the capture stream first, so the kernel and the
        # copy paths are loaded before capture; it takes at most one step
        # per run, whatever the staging buffers hold.
        warm = _native.SolveArgs.from_buffer_copy(self.args)
        warm.max_steps = 1
        with torch.cuda.stream(stream):
            self._body(stream, warm)
        stream.synchronize()
        with torch.cuda.graph(self.graph, stream=stream):
            self._body(stream, self.args)
        torch.cuda.synchronize(dev)

    def _body(self, stream, args):
        self.inits_d.copy_(self.inits_h, non_blocking=True)
        self.params_d.copy_(self.params_h, non_blocking=True)
        if self.dur_d is not None:
            self.dur_d.copy_(self.dur_h, non_blocking=True)
        if self.tol_d is not None:
            self.tol_d.copy_(self.tol_h, non_blocking=True)
        self.bufs["work"].zero_()
        self.bufs["totals"].zero_()
        self.prep["module"].launch(args, self.kernel, self.block, self.grid, stream.cuda_stream)
        for k, h in self.out_h.items():
            h.copy_(self.bufs[k], non_blocking=True)

    def __call__(self, inits=None, params=None, durations=None, tol_scale=None):
        """Copy the given inputs into the pinned staging buffers (skip any
        argument already written there in place), replay, wait; returns
        the pinned host outputs (``state``, ``status``, ``totals``, ...),
        valid until the next call."""
        torch = _torch()
        for src, dst in ((inits, self.inits_h), (params, self.params_h), (durations, self.dur_h),
                         (tol_scale, self.tol_h)):
            if src is not None:
                if dst is None:
                    raise ValueError("this graph was captured without that per-run input")
                dst.copy_(torch.as_tensor(np.asarray(src) if not torch.is_tensor(src) else src).reshape(dst.shape))
        self.graph.replay()
        torch.cuda.synchronize(self.device)
        return self.out_h
