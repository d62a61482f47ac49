"""Batches of different systems in one persistent work-stealing launch.

The reference builds and launches one kernel per system and solver
configuration (``BatchSolverKernel``; src/cubie/batchsolving/
BatchSolverKernel.py:851-1011).  :class:`HeteroSolver` takes several
configured :class:`~cubie_b200.solver.Solver` objects ("families": any mix of
systems, algorithms, precisions, tolerances and outputs) and integrates all
their runs with one launch of ``cbx_integrate_hetero``
(``csrc/device/cbx_hetero.cuh``): warps drain one family at a time and
move on to the next family that still has runs, so a family of short runs
and a family of long runs share the GPU without a tail where only the long
family is still running.  Each family keeps its own inputs, outputs,
per-run horizons and tolerance scales, and returns its own
:class:`~cubie_b200.solveresult.SolveResult`.  :meth:`HeteroSolver.setup`
prepares a launch once for repeated or graph-captured replays.
"""

from __future__ import annotations

from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from . import _native
from .kernelgen import generate_hetero_kernel
from .solver import Solver, _is_tensor, _torch
from .solveresult import merge_results

_HETERO_MODULES: Dict[tuple, "_native.Module"] = {}


# Relative tolerance below which FP32 stepping cannot honour a run's
# tolerance: an FP32 state carries about 6e-8 relative rounding per
# operation, and the reference's own gate rejects FP32 results below about
# 1e-6 (tests/integrated_numerical_tests/julia_reference/ne_gate.py:38-41).
FP32_RTOL_FLOOR = 1e-6
# The same for the mixed-precision path (FP32 stages, FP64 time and control,
# compensated state update): its state accumulates increments at FP64-like
# accuracy, and on the mixed three-system batch its runs at rtol down to
# 1e-8 match the error of the same method stepped in FP64; the floor sits a
# decade below that.
MIXED_RTOL_FLOOR = 1e-9


def _take(x, idx):
    """Columns ``idx`` (runs) of an array or tensor ``[..., n]``."""
    if x is None:
        return None
    if _is_tensor(x):
        torch = _torch()
        return x.index_select(x.dim() - 1, torch.as_tensor(idx, device=x.device, dtype=torch.long))
    return np.asarray(x)[..., idx]


class HeteroSolver:
    """One launch over the runs of several solvers.

    ``fp32_floor`` / ``mixed_floor``: runs of an FP32 (or a
    mixed-precision) family whose tightest relative tolerance (``rtol`` x
    the run's ``tol_scale``) lies below it are integrated by an
    FP64-stepping twin of that family, added to the same launch; the
    family's results come back merged in the caller's run order (in FP64
    when any run was routed).  ``None`` turns the routing off."""

    def __init__(self, solvers: Sequence[Solver], block_size: Optional[int] = None,
                 fp32_floor: Optional[float] = FP32_RTOL_FLOOR, mixed_floor: Optional[float] = MIXED_RTOL_FLOOR):
        if not 1 <= len(solvers) <= _native.HeteroArgs.MAX_FAMILIES:
            raise ValueError(f"one to {_native.HeteroArgs.MAX_FAMILIES} solvers per launch")
        devices = {s.device for s in solvers}
        if len(devices) != 1:
            raise ValueError("all solvers must use the same device")
        self.user_solvers = list(solvers)
        self.solvers = list(solvers)
        self.device = devices.pop()
        self.block_size = int(block_size or solvers[0].block_size)
        self.fp32_floor = fp32_floor
        self.mixed_floor = mixed_floor
        self.last_kernel_ms = None
        self._twins: Dict[int, Solver] = {}

    def route(self, batches: Sequence[Dict[str, Any]]):
        """Split each FP32 family's batch at the floor: returns the launch's
        (solver, batch) families and, per caller family, a list of
        ``(launch family, run indices)``."""
        fams, routes = [], []
        for k, (s, b) in enumerate(zip(self.user_solvers, batches)):
            iv = b["initial_values"]
            n = int(iv.shape[1]) if hasattr(iv, "shape") and len(iv.shape) == 2 else None
            low = None
            floor = self.mixed_floor if s.mixed_precision else self.fp32_floor
            if floor is not None and s.precision == np.float32 and n is not None:
                ts = b.get("tol_scale")
                scale = np.ones(n) if ts is None else np.asarray(
                    ts.detach().cpu().numpy() if _is_tensor(ts) else ts, dtype=np.float64).reshape(-1)
                low = float(np.min(s.rtol)) * scale < floor
            if low is None or not low.any():
                routes.append([(len(fams), None)])
                fams.append((s, b))
                continue
            hi_idx, lo_idx = np.where(~low)[0], np.where(low)[0]
            twin = self._twins.get(k)
            if twin is None:
                twin = self._twins[k] = s.with_precision(np.float64)
            route = []
            for solver, idx in ((s, hi_idx), (twin, lo_idx)):
                if idx.size == 0:
                    continue
                sub = dict(b)
                for key in ("initial_values", "parameters", "durations", "tol_scale"):
                    if b.get(key) is not None:
                        sub[key] = _take(b[key], idx)
                route.append((len(fams), idx))
                fams.append((solver, sub))
            routes.append(route)
        if len(fams) > _native.HeteroArgs.MAX_FAMILIES:
            raise ValueError(f"{len(fams)} families after FP64 routing; at most {_native.HeteroArgs.MAX_FAMILIES}")
        return fams, routes

    def _module(self, preps):
        fams = []
        for s, prep in zip(self.solvers, preps):
            fams.append((s.system, prep["spec"], prep["gen"].system))
        src = generate_hetero_kernel(fams)
        import hashlib
        key = (hashlib.sha256(src.encode()).hexdigest(), self.device)
        mod = _HETERO_MODULES.get(key)
        if mod is None:
            cubin, log = _native.compile_cubin(src, _native.default_options(fast_math=self.solvers[0].fast_math))
            mod = _native.Module(cubin, self.device, log)
            _HETERO_MODULES[key] = mod
        return mod, src

    def setup(self, batches: Sequence[Dict[str, Any]]) -> "HeteroLaunch":
        """Allocate the outputs and build the launch arguments for
        ``batches`` (``batches[k]`` for ``solvers[k]``: a dict with
        ``initial_values`` and ``parameters`` (arrays ``[n_states, n_runs]``
        / ``[n_params, n_runs]`` or tensors), ``duration`` and optionally
        ``durations``, ``tol_scale``, ``settling_time``, ``t0``)."""
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("cubie_b200 needs a CUDA device: no GPU is visible")
        if len(batches) != len(self.user_solvers):
            raise ValueError("one batch per solver")
        fams, routes = self.route(batches)
        self.solvers = [f[0] for f in fams]
        batches = [f[1] for f in fams]
        dev = torch.device("cuda", self.device)
        preps, bufs, args, keep = [], [], [], []
        first = [0]
        for s, b in zip(self.solvers, batches):
            duration = float(b["duration"])
            durs = b.get("durations")
            prep = s.prepare(duration, b.get("settling_time", 0.0), b.get("t0", 0.0), durations=durs, load=False)
            tdt = torch.float32 if s.precision == np.float32 else torch.float64
            iv, pv = b["initial_values"], b.get("parameters")
            if not (_is_tensor(iv) and _is_tensor(pv)):
                iv, pv = s.build_grid(iv, pv, "verbatim")
            it = torch.as_tensor(iv).to(device=dev, dtype=tdt).contiguous()
            pt = torch.as_tensor(pv).to(device=dev, dtype=tdt).contiguous()
            n = int(it.shape[1])
            if pt.numel() == 0:
                pt = torch.zeros((1, max(n, 1)), device=dev, dtype=tdt)
            bf = s.allocate_outputs(prep, n, dev, tdt)
            dt = None if durs is None else torch.as_tensor(durs).to(device=dev, dtype=torch.float64).contiguous()
            ts = b.get("tol_scale")
            tt = None if ts is None else torch.as_tensor(ts).to(device=dev, dtype=torch.float64).contiguous()
            # runs claimed by decreasing estimated work within each family
            order = s.run_order(dt, tt) if dt is not None else None
            a = s.make_args(prep, bf, it, pt, None, n, duration, b.get("settling_time", 0.0), b.get("t0", 0.0),
                            dt, tt, order_t=order)
            keep.append(order)
            preps.append(prep)
            bufs.append(bf)
            args.append(a)
            keep += [it, pt, dt, tt]
            first.append(first[-1] + n)
        mod, _ = self._module(preps)
        h = _native.HeteroArgs()
        for k, a in enumerate(args):
            h.family[k] = a
        for k in range(_native.HeteroArgs.MAX_FAMILIES + 1):
            h.first_run[k] = first[min(k, len(first) - 1)]
        work = torch.zeros((_native.HeteroArgs.MAX_FAMILIES,), device=dev, dtype=torch.int64)
        h.work_counter = work.data_ptr()
        h.n_families = len(self.solvers)
        per_sm = mod.occupancy(2, self.block_size)
        sms = _native.device_info(self.device)["sm_count"]
        grid = max(1, min(max(per_sm, 1) * sms, (first[-1] + self.block_size - 1) // self.block_size))
        launch = HeteroLaunch(self, batches, mod, h, work, preps, bufs, keep, grid)
        launch.routes = routes
        return launch

    def solve(self, batches: Sequence[Dict[str, Any]], nan_error_trajectories: bool = True,
              on_device: bool = False, stream=None, distributed: bool = False) -> List:
        """Integrate every family's batch with one launch; one SolveResult
        per family.  ``distributed=True`` splits every family's runs across
        the ranks of the initialised ``torch.distributed`` group
        (interleaved, so each rank's launch holds the same mix of families
        and horizons); every rank returns the whole batch's results."""
        import torch.distributed as dist
        if distributed and dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
            from .shard import interleaved_runs
            rank, world = dist.get_rank(), dist.get_world_size()
            sizes = [int(b["initial_values"].shape[-1]) for b in batches]
            local = []
            for b, n in zip(batches, sizes):
                idx = interleaved_runs(n, rank, world)
                sub = dict(b)
                for key in ("initial_values", "parameters", "durations", "tol_scale"):
                    if b.get(key) is not None:
                        sub[key] = _take(b[key], idx)
                local.append(sub)
            mine = self.solve(local, nan_error_trajectories, False, stream)
            parts = [None] * world
            dist.all_gather_object(parts, mine)
            return [merge_results([(parts[r][k], interleaved_runs(n, r, world)) for r in range(world)])
                    for k, n in enumerate(sizes)]
        run = self.setup(batches)
        self.last_kernel_ms = run.timed_launch(stream)
        return run.collect(nan_error_trajectories, on_device)


class HeteroLaunch:
    """Buffers and arguments of one heterogeneous batch, ready to launch
    (repeatedly, or as a captured CUDA graph)."""

    def __init__(self, owner, batches, module, hargs, work, preps, bufs, keep, grid):
        self.owner, self.batches, self.module, self.hargs = owner, batches, module, hargs
        self.work, self.preps, self.bufs, self._keep, self.grid = work, preps, bufs, keep, grid

    def launch(self, stream, hargs=None) -> None:
        """Zero the run counters and iteration totals, then launch, on
        ``stream`` (capturable: no allocation, no synchronisation)."""
        self.work.zero_()
        for bf in self.bufs:
            bf["totals"].zero_()
        self.module.launch_hetero(hargs or self.hargs, self.owner.block_size, self.grid, stream.cuda_stream)

    def timed_launch(self, stream=None) -> float:
        torch = _torch()
        s0 = stream if stream is not None else torch.cuda.current_stream(torch.device("cuda", self.owner.device))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(s0)
        self.launch(s0)
        e1.record(s0)
        e1.synchronize()
        return e0.elapsed_time(e1)

    def graph(self):
        """The launch captured as a CUDA graph (``.replay()`` to run)."""
        torch = _torch()
        dev = torch.device("cuda", self.owner.device)
        stream = torch.cuda.Stream(device=dev)
        # eager pass first (kernel loaded before capture), at most one step per run
        warm = _native.HeteroArgs.from_buffer_copy(self.hargs)
        for k in range(self.hargs.n_families):
            warm.family[k].max_steps = 1
        with torch.cuda.stream(stream):
            self.launch(stream, warm)
        stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            self.launch(stream)
        torch.cuda.synchronize(dev)
        return g

    def collect(self, nan_error_trajectories: bool = True, on_device: bool = False) -> List:
        """One SolveResult per caller family, in the caller's run order."""
        per_launch = []
        for s, b, prep, bf in zip(self.owner.solvers, self.batches, self.preps, self.bufs):
            s.last_kernel_ms = self.owner.last_kernel_ms
            per_launch.append(s.collect(prep, bf, int(bf["status"].shape[0]), float(b["duration"]),
                                        b.get("settling_time", 0.0), b.get("t0", 0.0), nan_error_trajectories,
                                        on_device))
        routes = getattr(self, "routes", None) or [[(k, None)] for k in range(len(per_launch))]
        out = []
        for route in routes:
            if len(route) == 1 and route[0][1] is None:
                out.append(per_launch[route[0][0]])
            else:
                if on_device:
                    raise ValueError("routed families are merged on the host (on_device=False)")
                out.append(merge_results([(per_launch[f], idx) for f, idx in route]))
        return out
