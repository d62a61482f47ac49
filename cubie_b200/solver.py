"""User-facing batch solver: ``Solver`` and ``solve_ivp``.

Keeps the reference's public surface (``batchsolving/solver.py:215-751``):
``solve_ivp(system, y0, parameters, drivers, method, duration,
settling_time, t0, save_variables, summarise_variables, grid_type, ...)``
and ``Solver(system, algorithm, ..., **kwargs).solve(...)``, the keyword
routing into step-control, algorithm, output and loop settings, the
per-family controller defaults (``SingleIntegratorRunCore.py:180-205``),
the inner-tolerance defaults (``SingleIntegratorRunCore.py:353-415``) and
the save/summary timing rules (``SingleIntegratorRunCore.py:250-352``).

Underneath, the configuration becomes one generated CUDA translation unit
(:mod:`cubie_b200.kernelgen`) compiled by NVRTC for sm_100a and launched
through the C ABI (:mod:`cubie_b200._native`).  Device buffers are torch
tensors; the library only receives their pointers.

Additions beyond the reference are opt-in keywords:
``mixed_precision`` (FP32 stepping with FP64 time, step size, error-norm
reduction and Newton norms, the gain's powers in FP32, and a compensated
state update), ``kernel`` (``"persistent"`` work-stealing launch
or the ``"plain"`` one-thread-per-run launch), ``linear_correction_type=
"gmres"``, per-run ``durations`` and ``tol_scale`` arrays, ``max_steps``.
"""

from __future__ import annotations

import itertools
import math
import time
import warnings
from dataclasses import replace
from typing import Any, Dict, Iterable, List, Optional, Sequence, Tuple, Union

import numpy as np

from . import _native
from .codegen import generate_system
from .kernelgen import KernelSpec, generate_kernel
from .outputs import (SummaryPlan, output_length, parse_output_types, save_stop_time,
                      summaries_length, summary_stop_time)
from .solveresult import SolveResult, SolveSpec
from .symbolic import SymbolicODE, create_ODE_system
from .tableaus import ADAPTIVE_DEFAULTS, ROSENBROCK, Tableau, resolve_algorithm

STEP_CONTROL_KEYS = {"step_controller", "dt", "dt_min", "dt_max", "atol", "rtol", "kp", "ki", "kd",
                     "safety", "min_gain", "max_gain", "deadband_min", "deadband_max",
                     "newton_target_iters"}
ALGORITHM_KEYS = {"linear_correction_type", "krylov_atol", "krylov_rtol", "krylov_max_iters",
                  "krylov_residual_reduction", "krylov_residual_floor", "newton_atol", "newton_rtol",
                  "newton_max_iters", "preconditioner_order", "preconditioner_type",
                  "attempt_dense_prediction", "gmres_restart"}
OUTPUT_KEYS = {"output_types", "saved_state_indices", "saved_observable_indices",
               "summarised_state_indices", "summarised_observable_indices",
               "save_variables", "summarise_variables"}
LOOP_KEYS = {"save_every", "summarise_every", "sample_summaries_every"}
# largest operator (states, or stages x states for fully implicit tableaus)
# the register-resident direct solve forms
DIRECT_MAX_WIDTH = 16
EXECUTION_KEYS = {"mixed_precision", "kernel", "block_size", "min_blocks_per_sm", "max_steps", "device", "fast_math",
                  "precision", "adjoint", "layout", "schedule", "mem_proportion", "host_spill_threshold",
                  "spill_dir", "max_chunk_runs", "scratch_placement", "max_registers"}
IGNORED_KEYS = {"memory_settings", "cache", "auto_memory", "lineinfo", "time_logging_level",
                "profileCUDA", "cache_settings"}
RENAMED = {"dt_save": "save_every", "dt_summarise": "summarise_every",
           "dt_update_summaries": "sample_summaries_every"}

_MODULE_CACHE: Dict[Tuple[str, int], "_native.Module"] = {}


def _torch():
    import torch
    return torch


def _is_tensor(value) -> bool:
    return type(value).__module__.startswith("torch") and hasattr(value, "data_ptr")


def _as_tol(value, n) -> np.ndarray:
    arr = np.asarray(value, dtype=np.float64).reshape(-1)
    if arr.size == 1:
        arr = np.full(n, float(arr[0]))
    if arr.size != n:
        raise ValueError(f"tolerance vector has {arr.size} entries; expected 1 or {n}")
    if not np.all(np.isfinite(arr)) or np.any(arr < 0):
        raise ValueError("tolerances must be finite and non-negative")
    return arr


class Solver:
    """Batch solver for one system and one integrator configuration."""

    def __init__(self, system: SymbolicODE, algorithm: Union[str, Tableau] = "euler",
                 lineinfo: Optional[bool] = None,
                 step_control_settings: Optional[Dict[str, Any]] = None,
                 algorithm_settings: Optional[Dict[str, Any]] = None,
                 output_settings: Optional[Dict[str, Any]] = None,
                 memory_settings: Optional[Dict[str, Any]] = None,
                 loop_settings: Optional[Dict[str, Any]] = None,
                 time_logging_level: Optional[str] = None,
                 cache: Any = True, auto_memory: bool = True, **kwargs: Any) -> None:
        renamed = [k for k in kwargs if k in RENAMED]
        if renamed:
            raise KeyError("Renamed keyword argument(s): " +
                           ", ".join(f"'{k}' is now '{RENAMED[k]}'" for k in renamed))
        self.system = system
        self.precision = np.dtype(system.precision).type
        self.algorithm = algorithm if isinstance(algorithm, str) else getattr(algorithm, "name", "custom")
        step = dict(step_control_settings or {})
        algo = dict(algorithm_settings or {})
        out = dict(output_settings or {})
        loop = dict(loop_settings or {})
        execution: Dict[str, Any] = {}
        unknown = []
        for k, v in kwargs.items():
            if k in STEP_CONTROL_KEYS:
                step[k] = v
            elif k in ALGORITHM_KEYS:
                algo[k] = v
            elif k in OUTPUT_KEYS:
                out[k] = v
            elif k in LOOP_KEYS:
                loop[k] = v
            elif k in EXECUTION_KEYS:
                execution[k] = v
            elif k in IGNORED_KEYS:
                continue
            else:
                unknown.append(k)
        if unknown:
            raise KeyError(f"Unrecognized keyword arguments: {set(unknown)}")
        self.tableau = resolve_algorithm(algorithm)
        self.mixed_precision = bool(execution.get("mixed_precision", False))
        self.kernel_kind = execution.get("kernel", "persistent")
        if self.kernel_kind not in ("plain", "persistent"):
            raise ValueError("kernel must be 'plain' or 'persistent'")
        bs = execution.get("block_size", 128)
        self.autotune_pending = isinstance(bs, str) and bs == "auto"
        self.block_size = 128 if self.autotune_pending else int(bs)
        self.min_blocks_per_sm = int(execution.get("min_blocks_per_sm", 1))
        self.adjoint = bool(execution.get("adjoint", False))
        # "thread": one run per thread; "warp": one run per warp, for large
        # systems (diagonally implicit tableaus); "auto": warp from 64 states
        layout = execution.get("layout", "thread")
        if layout == "auto":
            layout = "warp" if (system.num_states >= 64 and self.tableau.kind == "dirk") else "thread"
        if layout not in ("thread", "warp"):
            raise ValueError("layout must be 'thread', 'warp' or 'auto'")
        self.layout = layout
        if getattr(system, "mass", None) is not None:
            # SingleIntegratorRunCore.py:765-780
            if self.tableau.kind == "erk":
                raise ValueError("The system defines a mass matrix and requires an implicit algorithm; "
                                 f"'{self.algorithm}' does not consume a mass matrix and would integrate the "
                                 "constraint residuals as derivatives.")
            if layout == "warp":
                raise NotImplementedError("the warp-per-system layout takes systems without a mass matrix")
            if execution.get("adjoint"):
                raise NotImplementedError("the discrete adjoint takes systems without a mass matrix")
        # warp layout: stage-solve scratch vectors in "shared" memory,
        # "local" (the lanes' arrays in local memory, cached in L1; the
        # fastest on the 256-state cable at 65,536 runs) or "registers"
        # (passed by value, more registers per thread); "auto" lets the
        # autotuner pick
        sp_ = str(execution.get("scratch_placement", "local"))
        if sp_ not in ("shared", "local", "registers", "auto"):
            raise ValueError("scratch_placement must be 'shared', 'local', 'registers' or 'auto'")
        self.placement_pending = sp_ == "auto"
        self.scratch_placement = "shared" if sp_ == "auto" else sp_
        # register cap per thread for the compiler (0: its default); the
        # warp layout's out-of-line stage solve otherwise stays at 128
        self.max_registers = int(execution.get("max_registers", 0))
        # claim order of persistent launches: "auto" / "longest_first" sort
        # runs by decreasing per-run horizon when horizons are given
        self.schedule = str(execution.get("schedule", "auto"))
        if self.schedule not in ("auto", "longest_first", "index"):
            raise ValueError("schedule must be 'auto', 'longest_first' or 'index'")
        self.max_steps = int(execution.get("max_steps", 0))
        # memory: share of device memory a solve may hold (None: 90 % of
        # free), outputs above host_spill_threshold bytes go to memory-mapped
        # files in spill_dir, max_chunk_runs caps the runs per launch
        mp = execution.get("mem_proportion")
        self.mem_proportion = None if mp is None else float(mp)
        if self.mem_proportion is not None and not 0.0 < self.mem_proportion <= 1.0:
            raise ValueError("mem_proportion must be in (0, 1]")
        hst = execution.get("host_spill_threshold")
        self.host_spill_threshold = None if hst is None else int(hst)
        self.spill_dir = execution.get("spill_dir")
        mcr = execution.get("max_chunk_runs")
        self.max_chunk_runs = None if mcr is None else int(mcr)
        self.chunks = 1
        self.device = int(execution.get("device", 0))
        self.fast_math = bool(execution.get("fast_math", True))
        self._resolve_step_control(step)
        self._resolve_algorithm_settings(algo)
        self._resolve_outputs(out)
        self._user_timing = {k: loop.get(k) for k in LOOP_KEYS}
        self._modules: Dict[str, Any] = {}
        self.last_kernel_ms: Optional[float] = None

    # ------------------------------------------------------------------
    # settings resolution
    # ------------------------------------------------------------------
    def _resolve_step_control(self, user: Dict[str, Any]) -> None:
        tab = self.tableau
        n = self.system.num_states
        if tab.has_error_estimate:
            settings = dict(ADAPTIVE_DEFAULTS[tab.kind])
        else:
            settings = {"step_controller": "fixed"}
        settings.update(user)
        ctl = str(settings.pop("step_controller")).lower()
        if ctl not in ("fixed", "i", "pi", "pid", "gustafsson"):
            raise ValueError(f"Unknown controller type: {ctl}")
        if ctl != "fixed" and not tab.has_error_estimate:
            warnings.warn(f"Adaptive step controller '{ctl}' cannot be used with fixed-step algorithm "
                          f"'{self.algorithm}'. Replacing with fixed-step controller.", UserWarning)
            ctl = "fixed"
        self.controller = ctl
        self.atol = _as_tol(settings.pop("atol", 1e-6), n)
        self.rtol = _as_tol(settings.pop("rtol", 1e-6), n)
        dt = settings.pop("dt", None)
        dt_min = settings.pop("dt_min", None)
        dt_max = settings.pop("dt_max", None)
        if ctl == "fixed":
            self.dt = float(dt) if dt is not None else 1e-3
            self.dt_min = self.dt_max = self.dt
        else:
            # BaseAdaptiveStepController._resolve_step_params / _ensure_sane_bounds
            user_min, user_max = dt_min is not None, dt_max is not None
            if dt is not None:
                dt_min = dt_min if user_min else dt / 100.0
                dt_max = dt_max if user_max else dt * 100.0
            dt_min = 1e-6 if dt_min is None else float(dt_min)
            dt_max = 1.0 if dt_max is None else float(dt_max)
            if dt is None:
                dt = math.sqrt(dt_min * dt_max)
            dt = float(dt)
            if dt_max < dt_min and user_min and user_max:
                raise ValueError(f"dt_max ({dt_max}) < dt_min ({dt_min}).")
            if dt < dt_min and user_min:
                raise ValueError(f"dt ({dt}) < dt_min ({dt_min}).")
            if dt > dt_max and user_max:
                raise ValueError(f"dt ({dt}) > dt_max ({dt_max}).")
            if dt_max < dt_min and not user_max:
                dt_max = dt_min * 100
            if dt_max < dt_min and not user_min:
                dt_min = dt_max / 100
            if dt < dt_min and not user_min:
                dt_min = dt / 100
            if dt > dt_max and not user_max:
                dt_max = dt * 100
            self.dt, self.dt_min, self.dt_max = dt, dt_min, dt_max
        self.kp = float(settings.pop("kp", 0.7))
        self.ki = float(settings.pop("ki", -0.4))
        self.kd = float(settings.pop("kd", 0.0))
        self.safety = float(settings.pop("safety", 0.9))
        self.min_gain = float(settings.pop("min_gain", 0.3))
        self.max_gain = float(settings.pop("max_gain", 2.0))
        self.deadband_min = float(settings.pop("deadband_min", 1.0))
        self.deadband_max = float(settings.pop("deadband_max", 1.2))
        self.newton_target_iters = int(settings.pop("newton_target_iters", 20))

    def _resolve_algorithm_settings(self, user: Dict[str, Any]) -> None:
        n = self.system.num_states
        tab = self.tableau
        eps = float(np.finfo(self.precision).eps)
        lin = user.get("linear_correction_type", "minimal_residual")
        if lin not in ("steepest_descent", "minimal_residual", "bicgstab", "gmres", "direct"):
            raise ValueError("linear_correction_type must be one of 'steepest_descent', "
                             f"'minimal_residual', 'bicgstab', 'gmres', 'direct'; got '{lin}'.")
        if lin == "direct":
            # direct solve in registers: one system per thread, small operators
            width = n * (tab.stage_count if tab.kind == "firk" else 1)
            if self.layout != "thread":
                raise ValueError("linear_correction_type='direct' needs layout='thread'")
            if width > DIRECT_MAX_WIDTH:
                raise ValueError(f"linear_correction_type='direct' forms the {width}x{width} operator; "
                                 f"at most {DIRECT_MAX_WIDTH} is supported")
        self.linear_correction_type = lin
        implicit = tab.kind != "erk"
        # inner tolerances derived from the controller unless given
        self.krylov_atol = _as_tol(user["krylov_atol"], n) if user.get("krylov_atol") is not None else self.atol.copy()
        self.krylov_rtol = _as_tol(user["krylov_rtol"], n) if user.get("krylov_rtol") is not None else self.rtol.copy()
        self.newton_atol = _as_tol(user["newton_atol"], n) if user.get("newton_atol") is not None else self.atol / 10.0
        self.newton_rtol = _as_tol(user["newton_rtol"], n) if user.get("newton_rtol") is not None else self.rtol / 10.0
        if user.get("krylov_residual_reduction") is not None:
            self.krylov_residual_reduction = float(user["krylov_residual_reduction"])
        else:
            floor = float(self.rtol.min())
            if implicit and self.controller != "fixed" and floor > 0.0:
                if tab.kind == ROSENBROCK:
                    floor *= 0.01
                self.krylov_residual_reduction = floor
            else:
                self.krylov_residual_reduction = eps
            if self.mixed_precision:
                # FP32 Krylov vectors cannot represent a residual reduction
                # finer than a few float32 ulps; the derived default (0.01 rtol
                # for Rosenbrock steps) would otherwise leave every solve at
                # its iteration cap.
                self.krylov_residual_reduction = max(self.krylov_residual_reduction,
                                                     8.0 * float(np.finfo(np.float32).eps))
        self.krylov_residual_floor = float(user.get("krylov_residual_floor") or math.sqrt(eps))
        self.krylov_max_iters = int(user.get("krylov_max_iters", 100))
        self.newton_max_iters = int(user.get("newton_max_iters", 100))
        self.preconditioner_order = int(user.get("preconditioner_order", 2))
        ptype = user.get("preconditioner_type", "neumann")
        if ptype not in ("neumann", None, "none"):
            raise NotImplementedError(f"preconditioner_type '{ptype}' is not supported")
        self.preconditioned = ptype == "neumann"
        self.attempt_dense_prediction = bool(user.get("attempt_dense_prediction", True))
        self.gmres_restart = int(user.get("gmres_restart", 8))

    def _resolve_outputs(self, out: Dict[str, Any]) -> None:
        sysm = self.system
        output_types = out.get("output_types", ["state"])
        if isinstance(output_types, str):
            output_types = [output_types]
        self.output_types = list(output_types)
        flags, summary_req = parse_output_types(self.output_types)
        self.flags = flags
        self.summary_plan = SummaryPlan.from_request(summary_req)

        def resolve(labels, s_idx, o_idx):
            if labels is None and s_idx is None and o_idx is None:
                return list(range(sysm.num_states)), list(range(sysm.num_observables))
            st, ob = set(), set()
            for lab in labels or []:
                if lab in sysm.state_names:
                    st.add(sysm.state_names.index(lab))
                elif lab in sysm.observable_names:
                    ob.add(sysm.observable_names.index(lab))
                else:
                    raise ValueError(f"Variable '{lab}' is not a state or observable")
            st |= set(int(i) for i in (s_idx if s_idx is not None else []))
            ob |= set(int(i) for i in (o_idx if o_idx is not None else []))
            return sorted(st), sorted(ob)

        self.saved_state_indices, self.saved_observable_indices = resolve(
            out.get("save_variables"), out.get("saved_state_indices"), out.get("saved_observable_indices"))
        if (out.get("summarise_variables") is None and out.get("summarised_state_indices") is None
                and out.get("summarised_observable_indices") is None):
            self.summarised_state_indices = list(self.saved_state_indices)
            self.summarised_observable_indices = list(self.saved_observable_indices)
        else:
            self.summarised_state_indices, self.summarised_observable_indices = resolve(
                out.get("summarise_variables"), out.get("summarised_state_indices"),
                out.get("summarised_observable_indices"))
        for i in self.saved_state_indices + self.summarised_state_indices:
            if not 0 <= i < sysm.num_states:
                raise ValueError(f"state index {i} out of range")
        for i in self.saved_observable_indices + self.summarised_observable_indices:
            if not 0 <= i < sysm.num_observables:
                raise ValueError(f"observable index {i} out of range")

    # ------------------------------------------------------------------
    def _timing(self, duration: float) -> Dict[str, Any]:
        """Loop timing (SingleIntegratorRunCore.py:250-352)."""
        f = self.flags
        time_domain = (f["state"] and len(self.saved_state_indices) > 0) or \
                      (f["observables"] and len(self.saved_observable_indices) > 0) or \
                      f["time"] or f["iteration_counters"]
        summaries = bool(self.summary_plan.metrics) and \
            (len(self.summarised_state_indices) + len(self.summarised_observable_indices) > 0)
        save_every = self._user_timing.get("save_every")
        summarise_every = self._user_timing.get("summarise_every")
        sample_every = self._user_timing.get("sample_summaries_every")
        save_last = bool(time_domain and save_every is None)
        if summaries:
            if summarise_every is None:
                warnings.warn("Summary metrics were requested with no summarise_every or "
                              "sample_summaries_every timing. Sample_summaries_every was set to "
                              "duration / 100 by default.", UserWarning)
                summarise_every = duration
                sample_every = duration / 100.0
            elif sample_every is None:
                sample_every = summarise_every / 10.0
        else:
            summarise_every = sample_every = None
        samples_per_summary = 0
        if summarise_every is not None and sample_every is not None:
            p = self.precision
            ratio = float(p(summarise_every)) / float(p(sample_every))
            samples_per_summary = int(round(ratio))
            if abs(ratio - samples_per_summary) > 0.01:
                raise ValueError(f"summarise_every ({summarise_every}) must be an integer multiple of "
                                 f"sample_summaries_every ({sample_every}).")
        return dict(save_every=save_every if time_domain else None, summarise_every=summarise_every,
                    sample_every=sample_every, samples_per_summary=samples_per_summary,
                    save_last=save_last, save_regularly=bool(save_every is not None and time_domain),
                    summarise_regularly=bool(summarise_every is not None and summaries),
                    time_domain=time_domain, summaries=summaries)

    def kernel_spec(self, timing: Dict[str, Any], driver_meta: Optional[dict] = None) -> KernelSpec:
        f = self.flags
        dm = driver_meta or {}
        return KernelSpec(
            precision=self.precision, tableau=self.tableau, controller=self.controller,
            dt=self.dt, dt_min=self.dt_min, dt_max=self.dt_max, atol=self.atol, rtol=self.rtol,
            kp=self.kp, ki=self.ki, kd=self.kd, safety=self.safety, min_gain=self.min_gain,
            max_gain=self.max_gain, deadband_min=self.deadband_min, deadband_max=self.deadband_max,
            newton_target_iters=self.newton_target_iters,
            linear_correction_type=self.linear_correction_type,
            krylov_atol=self.krylov_atol, krylov_rtol=self.krylov_rtol,
            krylov_max_iters=self.krylov_max_iters,
            krylov_residual_reduction=self.krylov_residual_reduction,
            krylov_residual_floor=self.krylov_residual_floor,
            newton_atol=self.newton_atol, newton_rtol=self.newton_rtol,
            newton_max_iters=self.newton_max_iters, preconditioner_order=self.preconditioner_order,
            preconditioned=self.preconditioned, gmres_restart=self.gmres_restart,
            save_state=bool(f["state"] and self.saved_state_indices),
            save_observables=bool(f["observables"] and self.saved_observable_indices),
            save_time=bool(f["time"]), save_counters=bool(f["iteration_counters"]),
            saved_state_indices=tuple(self.saved_state_indices) if f["state"] else (),
            saved_observable_indices=tuple(self.saved_observable_indices) if f["observables"] else (),
            summarised_state_indices=tuple(self.summarised_state_indices) if timing["summaries"] else (),
            summarised_observable_indices=tuple(self.summarised_observable_indices) if timing["summaries"] else (),
            summary=self.summary_plan if timing["summaries"] else SummaryPlan.empty(),
            save_every=timing["save_every"], sample_summaries_every=timing["sample_every"],
            samples_per_summary=timing["samples_per_summary"], save_last=timing["save_last"],
            save_regularly=timing["save_regularly"], summarise_regularly=timing["summarise_regularly"],
            driver_order=dm.get("order", 3), driver_num_segments=dm.get("num_segments", 1),
            driver_eval_start=dm.get("eval_start", 0.0), driver_inv_resolution=dm.get("inv_resolution", 1.0),
            driver_wrap=dm.get("wrap", False),
            mixed_precision=self.mixed_precision, block_size=self.block_size,
            min_blocks_per_sm=self.min_blocks_per_sm, adjoint=self.adjoint, layout=self.layout,
            dense_prediction=None if self.attempt_dense_prediction else False,
            scratch_placement=self.scratch_placement, max_registers=self.max_registers,
        )

    def _generate(self, spec: KernelSpec):
        """Kernel source for ``spec``; the symbolic system part (SymPy CSE,
        the costly step) is generated once per solver."""
        second = bool(spec.adjoint and spec.tableau.kind == "rosenbrock")
        cache = self.__dict__.setdefault("_system_code", {})
        key = "stub" if spec.layout == "warp" else second
        gen = cache.get(key)
        if gen is None:
            if spec.layout == "warp":
                from .codegen import system_stub
                gen = cache[key] = system_stub(self.system)
            else:
                gen = cache[key] = generate_system(self.system, second_order=second)
        warp = None
        if spec.layout == "warp":
            warp = cache.get("warp")
            if warp is None:
                from .warpgen import generate_warp_system
                warp = cache["warp"] = generate_warp_system(self.system)
        return generate_kernel(self.system, spec, gen=gen, warp_code=warp)

    def compile_for(self, spec: KernelSpec):
        """NVRTC-compile ``spec`` (no device needed; safe to call from
        several threads at once).  Returns ``(gk, cubin, log)``, or
        ``(gk, None, None)`` when the module is already loaded."""
        gk = self._generate(spec)
        if (gk.key, self.device) in _MODULE_CACHE:
            return gk, None, None
        opts = _native.default_options(fast_math=self.fast_math)
        if spec.max_registers:
            opts.append(f"--maxrregcount={int(spec.max_registers)}")
        cubin, log = _native.compile_cubin(gk.source, opts)
        return gk, cubin, log

    def module_for(self, spec: KernelSpec, compiled=None):
        """Compile (or fetch) the NVRTC module for ``spec`` on this device;
        ``compiled`` is a result of :meth:`compile_for` to load instead."""
        gk, cubin, log = compiled if compiled is not None else self.compile_for(spec)
        key = (gk.key, self.device)
        mod = _MODULE_CACHE.get(key)
        if mod is None:
            if cubin is None:
                gk, cubin, log = self.compile_for(spec)
            mod = _native.Module(cubin, self.device, log)
            _MODULE_CACHE[key] = mod
        return mod, gk

    # ------------------------------------------------------------------
    def build_grid(self, initial_values, parameters, grid_type: str = "verbatim") -> Tuple[np.ndarray, np.ndarray]:
        """Return (inits[n_states, n_runs], params[n_params, n_runs])."""
        sysm = self.system
        p = self.precision
        if not isinstance(initial_values, dict) and not isinstance(parameters, dict):
            inits = np.asarray(initial_values, dtype=p)
            if inits.ndim == 1:
                inits = inits[:, None]
            if parameters is None:
                params = np.repeat(sysm.default_parameters()[:, None], inits.shape[1], axis=1)
            else:
                params = np.asarray(parameters, dtype=p)
                if params.ndim == 1:
                    params = params[:, None]
            if params.shape[1] == 1 and inits.shape[1] > 1:
                params = np.repeat(params, inits.shape[1], axis=1)
            if inits.shape[1] == 1 and params.shape[1] > 1:
                inits = np.repeat(inits, params.shape[1], axis=1)
            if inits.shape[0] != sysm.num_states or params.shape[0] != sysm.num_parameters:
                raise ValueError(f"expected inits ({sysm.num_states}, n_runs) and params "
                                 f"({sysm.num_parameters}, n_runs); got {inits.shape} and {params.shape}")
            if inits.shape[1] != params.shape[1]:
                raise ValueError("inits and params must have the same number of runs")
            return np.ascontiguousarray(inits), np.ascontiguousarray(params)
        # dictionary inputs: build a grid (BatchInputHandler.py:210-330)
        req: List[Tuple[str, int, np.ndarray]] = []
        for kind, spec in (("state", initial_values), ("param", parameters)):
            if spec is None:
                continue
            if not isinstance(spec, dict):
                arr = np.asarray(spec, dtype=np.float64).reshape(-1)
                names = sysm.state_names if kind == "state" else sysm.parameter_names
                spec = {nm: arr[i] for i, nm in enumerate(names)}
            for k, v in spec.items():
                names = sysm.state_names if kind == "state" else sysm.parameter_names
                idx = names.index(k) if isinstance(k, str) else int(k)
                req.append((kind, idx, np.atleast_1d(np.asarray(v, dtype=np.float64))))
        if grid_type == "combinatorial":
            vals = [list(dict.fromkeys(r[2].tolist())) for r in req]
            combos = np.array(list(itertools.product(*vals))).T if vals else np.zeros((0, 1))
            n_runs = combos.shape[1] if vals else 1
        elif grid_type == "verbatim":
            lens = {r[2].size for r in req if r[2].size > 1}
            if len(lens) > 1:
                raise ValueError("verbatim grids need equal-length inputs")
            n_runs = lens.pop() if lens else 1
            combos = np.array([np.broadcast_to(r[2], (n_runs,)) for r in req]) if req else np.zeros((0, n_runs))
        else:
            raise ValueError("grid_type must be 'combinatorial' or 'verbatim'")
        inits = np.repeat(sysm.default_initial_values()[:, None], n_runs, axis=1).astype(p)
        params = np.repeat(sysm.default_parameters()[:, None], n_runs, axis=1).astype(p)
        for row, (kind, idx, _) in enumerate(req):
            (inits if kind == "state" else params)[idx, :] = combos[row]
        return inits, params

    # ------------------------------------------------------------------
    def solve(self, initial_values, parameters=None, drivers=None, duration: float = 1.0,
              settling_time: float = 0.0, t0: float = 0.0, blocksize: Optional[int] = None,
              grid_type: str = "verbatim", nan_error_trajectories: bool = True,
              on_device: bool = False, durations=None, tol_scale=None, stream=None,
              distributed: bool = False, **kwargs) -> SolveResult:
        """``distributed=True`` splits the runs across the ranks of the
        initialised ``torch.distributed`` group (one process per GPU, each
        solver on its own device): every rank integrates an interleaved
        share and returns the whole batch's result (no exchange during the
        integration; the outputs are gathered once at the end)."""
        if kwargs:
            raise KeyError(f"Unrecognized keyword arguments: {set(kwargs)}")
        if distributed:
            if on_device:
                raise ValueError("a distributed solve returns host arrays (on_device=False)")
            from .shard import distributed_solve
            if not (_is_tensor(initial_values) and _is_tensor(parameters)):
                initial_values, parameters = self.build_grid(initial_values, parameters, grid_type)

            def local(iv, pv, durations=None, tol_scale=None):
                return self.solve(iv, pv, drivers=drivers, duration=duration, settling_time=settling_time, t0=t0,
                                  blocksize=blocksize, nan_error_trajectories=nan_error_trajectories,
                                  durations=durations, tol_scale=tol_scale, stream=stream)

            return distributed_solve(local, initial_values, parameters,
                                     {k: v for k, v in (("durations", durations), ("tol_scale", tol_scale))
                                      if v is not None})
        if drivers is not None or self.system.num_drivers > 0:
            from .interpolator import ArrayInterpolator
            interp = ArrayInterpolator.from_system(self.system, drivers, self.precision)
        else:
            interp = None
        if _is_tensor(initial_values) and _is_tensor(parameters):
            # pre-built [n_states, n_runs] / [n_params, n_runs] tensors (host,
            # possibly pinned, or device): no grid building, no host copies
            inits, params = initial_values, parameters
        else:
            inits, params = self.build_grid(initial_values, parameters, grid_type)
        return self.run(inits, params, interp, duration, settling_time, t0,
                        nan_error_trajectories=nan_error_trajectories, on_device=on_device,
                        durations=durations, tol_scale=tol_scale, stream=stream,
                        block=blocksize)

    def prepare(self, duration: float, settling_time: float = 0.0, t0: float = 0.0,
                interp=None, durations=None, load: bool = True) -> Dict[str, Any]:
        """Compile (and with ``load``, load) the module and compute output
        sizes for a launch."""
        if duration <= 0:
            raise ValueError("duration must be positive")
        key = None
        if interp is None:
            key = (float(duration), float(settling_time), float(t0), durations is None, bool(load))
            hit = self.__dict__.setdefault("_prepared", {}).get(key)
            if hit is not None:
                return hit
        timing = self._timing(float(duration))
        if durations is not None and (timing["save_regularly"] or timing["summarise_regularly"]):
            raise ValueError("per-run durations need end-of-run saving only (no save_every or summaries)")
        driver_meta = interp.device_meta() if interp is not None else None
        spec = self.kernel_spec(timing, driver_meta)
        if load:
            mod, gk = self.module_for(spec)
        else:
            mod, gk = None, self._generate(spec)
        p = self.precision
        n_save = output_length(duration, timing["save_every"], timing["save_last"], p) if timing["time_domain"] else 0
        n_summ = summaries_length(duration, timing["sample_every"], timing["samples_per_summary"], p) \
            if timing["summaries"] else 0
        save_stop = save_stop_time(duration, settling_time, t0, timing["save_every"], p)
        summ_stop = summary_stop_time(duration, settling_time, t0, timing["sample_every"], p)
        prep = dict(timing=timing, spec=spec, module=mod, gen=gk, n_save=n_save, n_summ=n_summ,
                    save_stop=save_stop, summary_stop=summ_stop)
        if key is not None:
            self._prepared[key] = prep
        return prep

    def run(self, inits: np.ndarray, params: np.ndarray, interp=None, duration: float = 1.0,
            settling_time: float = 0.0, t0: float = 0.0, nan_error_trajectories: bool = True,
            on_device: bool = False, durations=None, tol_scale=None, stream=None, block=None) -> SolveResult:
        """The seam the reference's ``BatchSolverKernel.run`` occupies
        (``BatchSolverKernel.py:525-604``): allocate, launch, collect."""
        torch = _torch()
        if not torch.cuda.is_available():
            raise RuntimeError("cubie_b200 needs a CUDA device: no GPU is visible")
        if self.autotune_pending or self.placement_pending:
            from .autotune import autotune, default_candidates
            cands = default_candidates(self)
            if not self.autotune_pending:
                # placement only: keep the caller's launch shape
                cands = [c for c in cands if c[0] == self.block_size] or cands
            tuned = autotune(self, inits, params, duration, durations=durations, candidates=cands, interp=interp)
            self.block_size, self.min_blocks_per_sm = int(tuned["block"]), int(tuned["min_blocks"])
            if tuned.get("placement"):
                self.scratch_placement = tuned["placement"]
            if tuned.get("max_registers") is not None:
                self.max_registers = int(tuned["max_registers"])
            self.autotune_result = tuned
            self.autotune_pending = self.placement_pending = False
            self.__dict__["_prepared"] = {}
        prep = self.prepare(duration, settling_time, t0, interp, durations)
        spec: KernelSpec = prep["spec"]
        dev = torch.device("cuda", self.device)
        tdtype = torch.float32 if self.precision == np.float32 else torch.float64
        n_runs = int(inits.shape[1])
        # run-axis chunking when the batch does not fit the memory budget
        from . import chunking
        plan = chunking.plan_chunks(
            n_runs, chunking.bytes_per_run(self, prep, int(durations is not None) + int(tol_scale is not None)),
            chunking.device_budget(self.device, self.mem_proportion), self.max_chunk_runs)
        if plan.n_chunks > 1:
            if on_device:
                raise ValueError("a chunked run cannot return device arrays (on_device=True); raise "
                                 "mem_proportion or solve fewer runs at a time")
            coeff = None
            if interp is not None:
                coeff = torch.as_tensor(interp.coefficients.astype(self.precision), device=dev).contiguous()
            return chunking.run_chunked(self, prep, inits, params, coeff, plan, duration, settling_time, t0,
                                        durations, tol_scale, nan_error_trajectories)
        self.chunks = 1
        inits_t = inits if isinstance(inits, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(inits), device=dev)
        params_t = params if isinstance(params, torch.Tensor) else torch.as_tensor(np.ascontiguousarray(params), device=dev)
        inits_t = inits_t.to(device=dev, dtype=tdtype, non_blocking=True).contiguous()
        params_t = params_t.to(device=dev, dtype=tdtype, non_blocking=True).contiguous()
        if params_t.numel() == 0:
            params_t = torch.zeros((1, max(n_runs, 1)), device=dev, dtype=tdtype)
        bufs = self.allocate_outputs(prep, n_runs, dev, tdtype)
        def per_run(values, name):
            if values is None:
                return None
            if _is_tensor(values):
                t = values.to(device=dev, dtype=torch.float64, non_blocking=True).reshape(-1).contiguous()
            else:
                t = torch.as_tensor(np.asarray(values, dtype=np.float64).reshape(-1), device=dev)
            if t.numel() != n_runs:
                raise ValueError(f"{name} must have one entry per run")
            return t

        dur_t = per_run(durations, "durations")
        tol_t = per_run(tol_scale, "tol_scale")
        coeff_t = None
        if interp is not None:
            coeff_t = torch.as_tensor(interp.coefficients.astype(self.precision), device=dev).contiguous()
        order_t = self.run_order(dur_t, tol_t)
        args = self.make_args(prep, bufs, inits_t, params_t, coeff_t, n_runs, duration, settling_time, t0,
                              dur_t, tol_t, order_t=order_t)
        kernel = self.launch_kind
        s = stream if stream is not None else torch.cuda.current_stream(dev)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        prep["module"].launch(args, kernel, int(block or self.block_size), 0, s.cuda_stream)
        e1.record(s)
        e1.synchronize()
        self.last_kernel_ms = e0.elapsed_time(e1)
        return self.collect(prep, bufs, n_runs, duration, settling_time, t0, nan_error_trajectories, on_device)

    @property
    def launch_kind(self) -> int:
        """C-ABI kernel kind of this solver's launch (CBX_KERNEL_*)."""
        if self.layout == "warp":
            return 3
        return 1 if self.kernel_kind == "persistent" else 0

    def graph(self, n_runs: int, duration: float, **kwargs):
        """A :class:`~cubie_b200.graph.GraphSolve`: this solve captured as
        one CUDA graph (transfers, launch, read-back) for repeated calls."""
        from .graph import GraphSolve
        return GraphSolve(self, n_runs, duration, **kwargs)

    def allocate_outputs(self, prep, n_runs: int, dev, tdtype) -> Dict[str, Any]:
        torch = _torch()
        spec: KernelSpec = prep["spec"]
        n_save, n_summ = prep["n_save"], prep["n_summ"]
        width = (len(spec.saved_state_indices) if spec.save_state else 0) + (1 if spec.save_time else 0)
        per_var = spec.summary.output_per_var if spec.summary else 0
        bufs = {
            "state": torch.zeros((n_save, width, n_runs), device=dev, dtype=tdtype) if width else None,
            "obs": torch.zeros((n_save, len(spec.saved_observable_indices), n_runs), device=dev, dtype=tdtype)
            if spec.save_observables else None,
            "state_sum": torch.zeros((n_summ, len(spec.summarised_state_indices) * per_var, n_runs), device=dev,
                                     dtype=tdtype) if spec.summarised_state_indices and per_var else None,
            "obs_sum": torch.zeros((n_summ, len(spec.summarised_observable_indices) * per_var, n_runs), device=dev,
                                   dtype=tdtype) if spec.summarised_observable_indices and per_var else None,
            "counters": torch.zeros((n_save, 4, n_runs), device=dev, dtype=torch.int32) if spec.save_counters else None,
            "status": torch.zeros((n_runs,), device=dev, dtype=torch.int32),
            "work": torch.zeros((2,), device=dev, dtype=torch.int64),
            "totals": torch.zeros((4,), device=dev, dtype=torch.int64),
        }
        return bufs

    def run_order(self, dur_t, tol_t=None):
        """Claim order of a persistent launch: with per-run horizons and
        ``schedule='longest_first'`` (the default ``'auto'`` when horizons
        are given), the runs sorted by decreasing estimated work, as a
        device int64 permutation; otherwise None (claim in index order).
        The estimate is the horizon, times tol_scale^(-1/(q+1)) for an
        adaptive method of order q when per-run tolerance scales are given
        (an error-controlled step shrinks as the (q+1)-th root of the
        tolerance), so a long, tight run is not claimed after shorter,
        cheaper ones and left running alone at the end of the launch.
        Each run's result does not depend on the order."""
        if dur_t is None or self.schedule == "index" or self.launch_kind == 0:
            return None
        torch = _torch()
        cost = dur_t
        if tol_t is not None and self.controller != "fixed":
            q = max(int(getattr(self.tableau, "order", 1) or 1), 1)
            cost = dur_t * torch.clamp(tol_t, min=1e-300) ** (-1.0 / (q + 1))
        return torch.argsort(cost, descending=True).to(torch.int64).contiguous()

    def make_args(self, prep, bufs, inits_t, params_t, coeff_t, n_runs, duration, settling_time, t0,
                  dur_t=None, tol_t=None, max_steps=None, order_t=None,
                  run_stride=None) -> "_native.SolveArgs":
        def ptr(t):
            return t.data_ptr() if t is not None else None
        a = _native.SolveArgs()
        a.inits = ptr(inits_t)
        a.params = ptr(params_t)
        a.driver_coeffs = ptr(coeff_t)
        a.state_out = ptr(bufs["state"])
        a.obs_out = ptr(bufs["obs"])
        a.state_sum_out = ptr(bufs["state_sum"])
        a.obs_sum_out = ptr(bufs["obs_sum"])
        a.counters_out = ptr(bufs["counters"])
        a.status_out = ptr(bufs["status"])
        a.durations = ptr(dur_t)
        a.tol_scale = ptr(tol_t)
        bufs["work"].zero_()
        a.work_counter = ptr(bufs["work"])
        a.totals = ptr(bufs["totals"])
        a.abort_flag = None
        a.run_order = ptr(order_t)
        a.n_runs = n_runs
        a.run_stride = n_runs if run_stride is None else int(run_stride)
        a.max_steps = int(self.max_steps if max_steps is None else max_steps)
        a.duration = float(duration)
        a.warmup = float(settling_time)
        a.t0 = float(t0)
        a.save_stop = float(prep["save_stop"])
        a.summary_stop = float(prep["summary_stop"])
        a.n_save_rows = int(prep["n_save"])
        a.n_summary_rows = int(prep["n_summ"])
        return a

    def collect(self, prep, bufs, n_runs, duration, settling_time, t0, nan_error_trajectories=True,
                on_device=False, host_arrays=None) -> SolveResult:
        """Build the :class:`SolveResult` from the device buffers of a
        launch (``bufs``), or from outputs already on the host
        (``host_arrays``, same keys; the chunked path)."""
        spec: KernelSpec = prep["spec"]
        keys = ("state", "obs", "state_sum", "obs_sum", "counters", "status", "totals")
        if host_arrays is not None:
            out = {k: host_arrays.get(k) for k in keys}
        elif on_device:
            out = {k: bufs.get(k) for k in keys}
        else:
            # one batch of asynchronous copies into pinned host memory (the
            # host caching allocator reuses the blocks across calls), then a
            # single wait: pageable copies would be staged through a bounce
            # buffer one output at a time
            torch = _torch()
            pinned = {}
            for key in keys:
                t = bufs.get(key)
                if t is not None:
                    pinned[key] = torch.empty(tuple(t.shape), dtype=t.dtype, pin_memory=True)
                    pinned[key].copy_(t, non_blocking=True)
            torch.cuda.current_stream(bufs["status"].device).synchronize()
            out = {k: (pinned[k].numpy() if k in pinned else None) for k in keys}
        res = SolveResult(
            state=out["state"], observables=out["obs"],
            state_summaries=out["state_sum"], observable_summaries=out["obs_sum"],
            iteration_counters=out["counters"], status_codes=out["status"],
            save_time=spec.save_time,
        )
        tot = out["totals"].cpu().numpy() if (on_device and host_arrays is None) else out["totals"]
        res.totals = dict(steps=int(tot[0]), rejections=int(tot[1]), newton=int(tot[2]), krylov=int(tot[3]))
        res.kernel_ms = self.last_kernel_ms
        sysm = self.system
        legend = {}
        k = 0
        if spec.save_state:
            for i in spec.saved_state_indices:
                legend[k] = sysm.state_names[i]
                k += 1
        if spec.save_observables:
            for i in spec.saved_observable_indices:
                legend[k] = sysm.observable_names[i]
                k += 1
        res.time_domain_legend = legend
        sl = {}
        k = 0
        names = spec.summary.legend() if spec.summary else []
        for i in spec.summarised_state_indices:
            for nm in names:
                sl[k] = f"{sysm.state_names[i]} {nm}"
                k += 1
        for i in spec.summarised_observable_indices:
            for nm in names:
                sl[k] = f"{sysm.observable_names[i]} {nm}"
                k += 1
        res.summaries_legend = sl
        timing = prep["timing"]
        res.solve_settings = SolveSpec(
            algorithm=self.algorithm, duration=float(duration), warmup=float(settling_time), t0=float(t0),
            dt=self.dt, dt_min=self.dt_min, dt_max=self.dt_max, save_every=timing["save_every"],
            summarise_every=timing["summarise_every"], sample_summaries_every=timing["sample_every"],
            atol=self.atol, rtol=self.rtol, output_types=self.output_types,
            saved_states=[sysm.state_names[i] for i in spec.saved_state_indices],
            saved_observables=[sysm.observable_names[i] for i in spec.saved_observable_indices],
            summarised_states=[sysm.state_names[i] for i in spec.summarised_state_indices],
            summarised_observables=[sysm.observable_names[i] for i in spec.summarised_observable_indices],
            precision=self.precision, mixed_precision=self.mixed_precision, kernel=self.kernel_kind)
        if nan_error_trajectories and not on_device:
            res.mask_error_runs()
        return res

    def with_precision(self, precision) -> "Solver":
        """A solver with the same settings stepping the same system at
        ``precision`` throughout (no mixed precision)."""
        import copy
        twin = copy.copy(self)
        twin.system = self.system.with_precision(precision)
        twin.precision = np.dtype(precision).type
        twin.mixed_precision = False
        for key in ("_system_code", "_prepared"):
            twin.__dict__.pop(key, None)
        twin._modules = {}
        return twin

    def close(self) -> None:
        pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def solve_ivp(system, y0, parameters=None, drivers=None, method: str = "euler", duration: float = 1.0,
              settling_time: float = 0.0, t0: float = 0.0, save_variables: Optional[List[str]] = None,
              summarise_variables: Optional[List[str]] = None, grid_type: str = "combinatorial",
              time_logging_level: Optional[str] = None, nan_error_trajectories: bool = True,
              **kwargs: Any) -> SolveResult:
    """Solve a batch of initial value problems (``solver.py:215-347``)."""
    if not isinstance(system, SymbolicODE):
        if parameters is not None and not isinstance(parameters, dict):
            raise TypeError("When equations are supplied directly to solve_ivp, parameters must be a "
                            "dict mapping names to values so the system's parameters can be declared.")
        states = None
        if isinstance(y0, dict):
            states = {k: float(np.asarray(v).flat[0]) for k, v in y0.items()}
        pdefs = None
        if isinstance(parameters, dict):
            pdefs = {k: float(np.asarray(v).flat[0]) for k, v in parameters.items()}
        create_kwargs = {}
        if "precision" in kwargs:
            create_kwargs["precision"] = kwargs.pop("precision")
        system = create_ODE_system(system, states=states, parameters=pdefs, drivers=drivers, **create_kwargs)
    if save_variables is not None:
        kwargs.setdefault("save_variables", save_variables)
    if summarise_variables is not None:
        kwargs.setdefault("summarise_variables", summarise_variables)
    blocksize = kwargs.pop("blocksize", None)
    solver = Solver(system, algorithm=method, **kwargs)
    try:
        return solver.solve(y0, parameters, drivers=drivers, duration=duration, settling_time=settling_time,
                            t0=t0, grid_type=grid_type, nan_error_trajectories=nan_error_trajectories,
                            blocksize=blocksize)
    finally:
        solver.close()
