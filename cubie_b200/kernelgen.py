"""Assemble the CUDA source of one integrator configuration.

A configuration (system, tableau, controller, solver and output settings,
precision policy) becomes a single translation unit: the generated system
``struct`` (:mod:`cubie_b200.codegen`), a tableau ``struct`` with
``constexpr`` accessors, ``__constant__`` tolerance and index tables, a
generated summary-metric ``struct`` and a ``Cfg`` struct of compile-time
switches, followed by the hand-written integrator headers under
``csrc/device``.  The result is compiled by NVRTC for sm_100a through the
C ABI (:mod:`cubie_b200._native`).

This replaces the reference's chain of CUDAFactory closures that Numba
inlines into one kernel per configuration (``BatchSolverKernel.py:851-1011``
and the factories it pulls in).
"""

from __future__ import annotations

import hashlib
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

from .codegen import GeneratedSystem, generate_system
from .outputs import SummaryPlan
from .symbolic import TIME, SymbolicODE
from .tableaus import DIRK, ERK, FIRK, ROSENBROCK, Tableau

ALGO_IDS = {ERK: "cbx::ALGO_ERK", DIRK: "cbx::ALGO_DIRK", FIRK: "cbx::ALGO_FIRK", ROSENBROCK: "cbx::ALGO_ROSENBROCK"}
STEP_TYPES = {ERK: "cbx::ErkStep<Cfg>", DIRK: "cbx::DirkStep<Cfg>", FIRK: "cbx::FirkStep<Cfg>",
              ROSENBROCK: "cbx::RosenbrockStep<Cfg>"}
LIN_IDS = {"minimal_residual": "cbx::LIN_MR", "steepest_descent": "cbx::LIN_SD",
           "bicgstab": "cbx::LIN_BICGSTAB", "gmres": "cbx::LIN_GMRES", "direct": "cbx::LIN_DIRECT"}
ADJOINT_FAMILIES = {ERK, ROSENBROCK}
CTRL_IDS = {"fixed": "cbx::CTRL_FIXED", "i": "cbx::CTRL_I", "pi": "cbx::CTRL_PI",
            "pid": "cbx::CTRL_PID", "gustafsson": "cbx::CTRL_GUSTAFSSON"}


@dataclass
class KernelSpec:
    """Everything that fixes the compiled integrator for one solver."""

    precision: type
    tableau: Tableau
    controller: str
    dt: float
    dt_min: float
    dt_max: float
    atol: np.ndarray
    rtol: np.ndarray
    kp: float = 0.7
    ki: float = -0.4
    kd: float = 0.0
    safety: float = 0.9
    min_gain: float = 0.3
    max_gain: float = 2.0
    deadband_min: float = 1.0
    deadband_max: float = 1.2
    newton_target_iters: int = 20
    linear_correction_type: str = "minimal_residual"
    krylov_atol: Optional[np.ndarray] = None
    krylov_rtol: Optional[np.ndarray] = None
    krylov_max_iters: int = 100
    krylov_residual_reduction: float = 0.0
    krylov_residual_floor: float = 0.0
    newton_atol: Optional[np.ndarray] = None
    newton_rtol: Optional[np.ndarray] = None
    newton_max_iters: int = 100
    preconditioner_order: int = 2
    preconditioned: bool = True
    gmres_restart: int = 8
    # outputs
    save_state: bool = False
    save_observables: bool = False
    save_time: bool = False
    save_counters: bool = False
    saved_state_indices: Tuple[int, ...] = ()
    saved_observable_indices: Tuple[int, ...] = ()
    summarised_state_indices: Tuple[int, ...] = ()
    summarised_observable_indices: Tuple[int, ...] = ()
    summary: Optional[SummaryPlan] = None
    # loop schedule
    save_every: Optional[float] = None
    sample_summaries_every: Optional[float] = None
    samples_per_summary: int = 0
    save_last: bool = False
    save_regularly: bool = False
    summarise_regularly: bool = False
    # drivers
    driver_order: int = 3
    driver_num_segments: int = 1
    driver_eval_start: float = 0.0
    driver_inv_resolution: float = 1.0
    driver_wrap: bool = False
    # execution policy
    mixed_precision: bool = False
    block_size: int = 128
    min_blocks_per_sm: int = 1
    dense_prediction: Optional[bool] = None
    # discrete adjoint kernels (forward with checkpoints, reverse sweep)
    adjoint: bool = False
    # "thread": one run per thread; "warp": one run per warp (large systems)
    layout: str = "thread"
    # where the warp layout keeps its stage-solve scratch vectors (stage
    # base, step start, BiCGSTAB shadow residual): "shared" memory of the
    # warp, "local" (the lane's arrays, passed by address into the
    # out-of-line stage solve, so in local memory) or "registers" (passed
    # and returned by value)
    scratch_placement: str = "local"
    # register cap per thread passed to the compiler (0: its default)
    max_registers: int = 0

    @property
    def adaptive(self) -> bool:
        return self.controller != "fixed"


def _lit(x: float) -> str:
    x = float(x)
    if np.isnan(x):
        return "__builtin_nan(\"\")"
    if np.isinf(x):
        return "(1.0/0.0)" if x > 0 else "(-1.0/0.0)"
    return repr(x)


def _table_fn(name: str, values: np.ndarray) -> str:
    """constexpr accessor over a (possibly 2-D/3-D) table of doubles."""
    arr = np.asarray(values, dtype=float)
    if arr.ndim == 1:
        body = ", ".join(_lit(v) for v in arr) if arr.size else "0.0"
        n = max(arr.size, 1)
        return (f"    static __host__ __device__ constexpr double {name}(int i) {{\n"
                f"        constexpr double v[{n}] = {{{body}}};\n        return v[i];\n    }}\n")
    if arr.ndim == 2:
        rows = ", ".join("{" + ", ".join(_lit(v) for v in row) + "}" for row in arr)
        return (f"    static __host__ __device__ constexpr double {name}(int i, int j) {{\n"
                f"        constexpr double v[{arr.shape[0]}][{arr.shape[1]}] = {{{rows}}};\n"
                f"        return v[i][j];\n    }}\n")
    flat = ", ".join(_lit(v) for v in arr.reshape(-1))
    p, s1, s2 = arr.shape
    return (f"    static __host__ __device__ constexpr double {name}(int q, int i, int j) {{\n"
            f"        constexpr double v[{p * s1 * s2}] = {{{flat}}};\n"
            f"        return v[(q * {s1} + i) * {s2} + j];\n    }}\n")


def tableau_struct(tab: Tableau, precision, dense: bool) -> str:
    s = tab.stage_count
    a = tab.a_matrix()
    d = np.asarray(tab.d if tab.d is not None else np.zeros(s))
    out = ["struct Tab {",
           f"    static constexpr int S = {s};",
           f"    static constexpr bool FSAL = {str(tab.first_same_as_last).lower()};",
           f"    static constexpr bool HAS_ERR = {str(tab.has_error_estimate).lower()};",
           f"    static constexpr bool ACC_OUT = {str(tab.accumulates_output).lower()};",
           f"    static constexpr bool ACC_ERR = {str(tab.accumulates_error).lower()};",
           f"    static constexpr int B_ROW = {tab.b_row if tab.b_row is not None else -1};",
           f"    static constexpr int BHAT_ROW = {tab.b_hat_row if tab.b_hat_row is not None else -1};",
           f"    static constexpr double GAMMA = {_lit(tab.gamma)};",
           f"    static constexpr bool DENSE_PRED = {str(bool(dense)).lower()};",
           f"    static constexpr double PRED_RATIO_LIMIT = {_lit(tab.dense_ratio_limit(precision))};",
           ]
    first_explicit = tab.first_stage_explicit
    diag = np.diag(a)
    later_explicit = bool(np.any(diag[1:] == 0.0)) if s > 1 else False
    out.append(f"    static constexpr bool HAS_LATER_EXPLICIT = {str(later_explicit).lower()};")
    out.append(f"    static constexpr bool EULER_GUESS = {str(bool(tab.euler_guess)).lower()};")
    out.append(f"    static __host__ __device__ constexpr bool need_f(int i) {{ constexpr bool v[{s}] = {{"
               + ", ".join(str(tab.stage_derivative_needed(i)).lower() for i in range(s)) + "}; return v[i]; }")
    out.append(f"    static constexpr int PRED_FIRST = {1 if first_explicit else 0};")
    if dense:
        coeffs = tab.prediction_coefficients()
        out.append(f"    static constexpr int PRED_POWERS = {coeffs.shape[0]};")
        out.append(_table_fn("pred", coeffs))
    else:
        out.append("    static constexpr int PRED_POWERS = 1;")
        out.append(_table_fn("pred", np.zeros((1, s, s))))
    src = np.asarray(tab.prediction_source_stages, dtype=float)
    out.append(f"    static __host__ __device__ constexpr int pred_source(int i) {{ constexpr int v[{s}] = {{"
               + ", ".join(str(int(x)) for x in src) + "}; return v[i]; }")
    out.append(_table_fn("a", a))
    out.append(_table_fn("b", np.asarray(tab.b)))
    out.append(_table_fn("c", np.asarray(tab.c)))
    out.append(_table_fn("d", d))
    Cm = np.zeros((s, s))
    if tab.C is not None:
        for i, row in enumerate(tab.C):
            Cm[i, : len(row)] = row
    out.append(_table_fn("Cm", Cm))
    gs = np.asarray(tab.gamma_stages if tab.gamma_stages is not None else np.zeros(s))
    out.append(_table_fn("gs", gs))
    out.append("};")
    return "\n".join(out)


def _const_array(name: str, ctype: str, values) -> str:
    vals = list(values)
    if not vals:
        vals = [0]
    body = ", ".join(_lit(v) if ctype != "int" else str(int(v)) for v in vals)
    return f"__constant__ {ctype} {name}[{len(vals)}] = {{{body}}};"


@dataclass
class GeneratedKernel:
    source: str
    system: GeneratedSystem
    spec: KernelSpec

    @property
    def key(self) -> str:
        return hashlib.sha256(self.source.encode()).hexdigest()[:24]


DEVICE_INCLUDES = ['#include "cbx_common.cuh"', '#include "cbx_args.h"', '#include "cbx_steps.cuh"',
                   '#include "cbx_control.cuh"', '#include "cbx_loop.cuh"']


def family_block(system: SymbolicODE, spec: KernelSpec, gen: GeneratedSystem, ns: str,
                 warp_source: Optional[str] = None) -> List[str]:
    """The generated pieces of one configuration (system struct, tolerance
    tables, index tables, tableau, summary metrics and ``Cfg``), to be
    placed inside namespace ``ns``; ``warp_source`` (the class-grouped
    system of the warp-per-system layout) adds ``Cfg::WSys``."""
    tab = spec.tableau
    n = system.num_states
    rtype = "float" if np.dtype(spec.precision) == np.float32 else "double"
    ctype = "double" if (spec.mixed_precision or rtype == "double") else "float"
    dense = spec.dense_prediction
    if dense is None:
        dense = tab.kind in (FIRK, DIRK) and tab.dense_prediction(spec.precision)
    ctl = spec.controller
    order = tab.order
    if ctl == "i":
        e1, e2, e3 = 1.0 / (2 * (1 + order)), 0.0, 0.0
    elif ctl in ("pi", "pid"):
        e1 = spec.kp / ((order + 1) * 2)
        e2 = spec.ki / ((order + 1) * 2)
        e3 = spec.kd / ((order + 1) * 2)
    elif ctl == "gustafsson":
        e1, e2, e3 = 1.0 / (2 * (order + 1)), 0.0, 0.0
    else:
        e1 = e2 = e3 = 0.0
    katol = spec.krylov_atol if spec.krylov_atol is not None else spec.atol
    krtol = spec.krylov_rtol if spec.krylov_rtol is not None else spec.rtol
    natol = spec.newton_atol if spec.newton_atol is not None else spec.atol / 10.0
    nrtol = spec.newton_rtol if spec.newton_rtol is not None else spec.rtol / 10.0
    summ = spec.summary or SummaryPlan.empty()
    summarise = bool(summ.metrics) and (len(spec.summarised_state_indices) + len(spec.summarised_observable_indices) > 0)

    def castp(v):
        # tolerances and schedule values are held at the precision the
        # control arithmetic runs in (the reference casts them to the
        # system precision; the mixed path keeps float64)
        if ctype == "float":
            return float(np.float32(v))
        return float(v)

    lines: List[str] = [gen.source]
    if warp_source is not None:
        lines.append(warp_source)
    tol_arrays = [("atol", spec.atol), ("rtol", spec.rtol), ("katol", katol), ("krtol", krtol), ("natol", natol),
                  ("nrtol", nrtol)]
    # A tolerance that is the same for every component becomes a literal;
    # otherwise a table: __constant__ where each lane reads one entry at a
    # time (thread layout), global memory where the lanes of a warp read
    # different entries at once (warp layout; the constant cache would
    # serialise those reads).
    accessors = []
    for name, vals in tol_arrays:
        cv = [castp(v) for v in np.broadcast_to(vals, (n,))]
        if all(v == cv[0] for v in cv):
            accessors.append(f"    static __device__ __forceinline__ C {name}(int) {{ return C({_lit(cv[0])}); }}")
            continue
        decl = _const_array(f"cbx_{name}", ctype, cv)
        if warp_source is not None:
            decl = "__device__ const " + decl[len("__constant__ "):]
        lines.append(decl)
        accessors.append(f"    static __device__ __forceinline__ C {name}(int i) {{ return cbx_{name}[i]; }}")
    idx_fns = []
    for fname, vals in (("saved_state", spec.saved_state_indices), ("saved_obs", spec.saved_observable_indices),
                        ("summ_state", spec.summarised_state_indices), ("summ_obs", spec.summarised_observable_indices)):
        vv = [int(v) for v in vals] or [0]
        step = vv[1] - vv[0] if len(vv) > 1 else 0
        if all(v == vv[0] + step * k for k, v in enumerate(vv)):
            # an affine selection (the common ranges) needs no table, which a
            # lane-dependent index would otherwise rebuild in local memory
            idx_fns.append(f"    static __host__ __device__ constexpr int {fname}(int k) {{ "
                           f"return {vv[0]} + {step} * k; }}")
        else:
            idx_fns.append(f"    static __host__ __device__ constexpr int {fname}(int k) {{ constexpr int v[{len(vv)}] = "
                           f"{{{', '.join(str(v) for v in vv)}}}; return v[k]; }}")
    lines.append("struct Idx {\n" + "\n".join(idx_fns) + "\n};")
    lines.append(tableau_struct(tab, spec.precision, dense))
    save_every = castp(spec.save_every) if spec.save_every is not None else 0.0
    sample_every = castp(spec.sample_summaries_every) if spec.sample_summaries_every is not None else 0.0
    lines.append(summ.device_struct(sample_every))
    cfg = [
        "struct Cfg {",
        f"    using Sys = {ns}::System;",
        f"    using R = {rtype};",
        f"    using C = {ctype};",
        f"    using G = {'float' if spec.mixed_precision else ctype};",
        f"    using Tab = {ns}::Tab;",
        f"    using Summ = {ns}::Summ;",
        f"    using Idx = {ns}::Idx;",
        f"    static constexpr int N = Sys::N, NP = Sys::NP, ND = Sys::ND, NO = Sys::NO, S = Tab::S;",
        f"    static constexpr int ALGO = {ALGO_IDS[tab.kind]};",
        f"    static constexpr int CTRL = {CTRL_IDS[ctl]};",
        f"    static constexpr bool ADAPTIVE = {str(spec.adaptive).lower()};",
        f"    static constexpr bool MIXED = {str(bool(spec.mixed_precision)).lower()};",
        f"    static constexpr double DT0 = {_lit(castp(spec.dt))};",
        f"    static constexpr double DT_MIN = {_lit(castp(spec.dt_min))};",
        f"    static constexpr double DT_MAX = {_lit(castp(spec.dt_max))};",
        f"    static constexpr double CTL_E1 = {_lit(castp(e1))};",
        f"    static constexpr double CTL_E2 = {_lit(castp(e2))};",
        f"    static constexpr double CTL_E3 = {_lit(castp(e3))};",
        f"    static constexpr double CTL_SAFETY = {_lit(castp(spec.safety))};",
        f"    static constexpr double CTL_MIN_GAIN = {_lit(castp(spec.min_gain))};",
        f"    static constexpr double CTL_MAX_GAIN = {_lit(castp(spec.max_gain))};",
        f"    static constexpr double CTL_DEADBAND_MIN = {_lit(castp(spec.deadband_min))};",
        f"    static constexpr double CTL_DEADBAND_MAX = {_lit(castp(spec.deadband_max))};",
        f"    static constexpr double CTL_INV_N = {_lit(castp(1.0 / n))};",
        f"    static constexpr int CTL_NEWTON_TARGET = {int(spec.newton_target_iters)};",
        f"    static constexpr int LIN = {LIN_IDS[spec.linear_correction_type]};",
        f"    static constexpr int KRYLOV_MAX_ITERS = {int(spec.krylov_max_iters)};",
        f"    static constexpr int NEWTON_MAX_ITERS = {int(spec.newton_max_iters)};",
        f"    static constexpr double KRYLOV_REDUCTION = {_lit(castp(spec.krylov_residual_reduction))};",
        f"    static constexpr double KRYLOV_FLOOR = {_lit(castp(spec.krylov_residual_floor))};",
        f"    static constexpr int PRECOND_ORDER = {int(spec.preconditioner_order)};",
        f"    static constexpr bool PRECONDITIONED = {str(bool(spec.preconditioned)).lower()};",
        f"    static constexpr int GMRES_RESTART = {int(spec.gmres_restart)};",
        f"    static constexpr bool SAVE_STATE = {str(spec.save_state).lower()};",
        f"    static constexpr bool SAVE_OBS = {str(spec.save_observables).lower()};",
        f"    static constexpr bool SAVE_TIME = {str(spec.save_time).lower()};",
        f"    static constexpr bool SAVE_COUNTERS = {str(spec.save_counters).lower()};",
        f"    static constexpr int N_SAVED_STATES = {len(spec.saved_state_indices) if spec.save_state else 0};",
        f"    static constexpr int N_SAVED_OBS = {len(spec.saved_observable_indices) if spec.save_observables else 0};",
        f"    static constexpr bool SUMMARISE = {str(summarise).lower()};",
        f"    static constexpr int N_SUMM_STATES = {len(spec.summarised_state_indices) if summarise else 0};",
        f"    static constexpr int N_SUMM_OBS = {len(spec.summarised_observable_indices) if summarise else 0};",
        f"    static constexpr int SAMPLES_PER_SUMMARY = {max(int(spec.samples_per_summary), 1)};",
        f"    static constexpr double SAVE_EVERY = {_lit(save_every)};",
        f"    static constexpr double SAMPLE_EVERY = {_lit(sample_every)};",
        f"    static constexpr bool SAVE_LAST = {str(spec.save_last).lower()};",
        f"    static constexpr bool SAVE_REG = {str(spec.save_regularly).lower()};",
        f"    static constexpr bool SUMM_REG = {str(spec.summarise_regularly).lower()};",
        f"    static constexpr int DRV_ORDER = {int(spec.driver_order)};",
        f"    static constexpr int DRV_NSEG = {max(int(spec.driver_num_segments), 1)};",
        f"    static constexpr double DRV_EVAL_START = {_lit(spec.driver_eval_start)};",
        f"    static constexpr double DRV_INV_RESOLUTION = {_lit(spec.driver_inv_resolution)};",
        f"    static constexpr bool DRV_WRAP = {str(spec.driver_wrap).lower()};",
        f"    static constexpr int BLOCK = {int(spec.block_size)};",
        f"    static constexpr int MIN_BLOCKS = {max(int(spec.min_blocks_per_sm), 1)};",
        f"    static constexpr bool SHARED_SCRATCH = "
        f"{str(spec.layout == 'warp' and spec.scratch_placement == 'shared').lower()};",
        f"    static constexpr bool REG_SCRATCH = "
        f"{str(spec.layout == 'warp' and spec.scratch_placement == 'registers').lower()};",
        f"    using Step = {STEP_TYPES[tab.kind]};",
        *([f"    using WSys = {ns}::WarpSystem;"] if warp_source is not None else []),
        *accessors,
        "};",
    ]
    lines.append("\n".join(cfg))
    return lines


def generate_kernel(system: SymbolicODE, spec: KernelSpec, gen: Optional[GeneratedSystem] = None,
                    warp_code=None) -> GeneratedKernel:
    """Return the complete CUDA translation unit for ``spec``: the device
    headers, then the configuration's generated pieces in namespace
    ``cbxsys``, then the kernels instantiated for ``cbxsys::Cfg``."""
    gen = gen or generate_system(system, second_order=spec.adjoint and spec.tableau.kind == ROSENBROCK)
    tab = spec.tableau
    if spec.layout == "warp":
        return _generate_warp_kernel(system, spec, gen, warp_code)
    lines = ["// generated by cubie_b200.kernelgen; do not edit"]
    if int(spec.min_blocks_per_sm) > 1:
        lines.append("#define CBX_LAUNCH_BOUNDS(CFG) __launch_bounds__(CFG::BLOCK, CFG::MIN_BLOCKS)")
    lines += DEVICE_INCLUDES
    if spec.adjoint:
        lines.append('#include "cbx_adjoint.cuh"')
    lines.append("namespace cbxsys {")
    lines += family_block(system, spec, gen, "cbxsys")
    lines.append("}  // namespace cbxsys")
    lines.append("CBX_DEFINE_KERNELS(cbxsys::Cfg)")
    if spec.adjoint:
        if tab.kind not in ADJOINT_FAMILIES:
            raise NotImplementedError(f"no discrete adjoint for the {tab.kind} family "
                                      f"(available: {sorted(ADJOINT_FAMILIES)})")
        if tab.kind == ROSENBROCK and (system.num_drivers > 0 or any(
                TIME in e.free_symbols for e in system.rhs_expressions())):
            raise NotImplementedError("the Rosenbrock adjoint needs an autonomous system without drivers")
        lines.append("CBX_DEFINE_ADJOINT_KERNELS(cbxsys::Cfg)")
    return GeneratedKernel(source="\n".join(lines) + "\n", system=gen, spec=spec)


def generate_hetero_kernel(families: Sequence[Tuple[SymbolicODE, KernelSpec, GeneratedSystem]]) -> str:
    """One translation unit holding several configurations (namespaces
    ``cbxfam0``, ``cbxfam1``, ...) and the heterogeneous persistent kernel
    over all of them (``csrc/device/cbx_hetero.cuh``).  All families share
    the first family's block size."""
    if not 1 <= len(families) <= 8:
        raise ValueError("one to eight families per heterogeneous launch")
    block = int(families[0][1].block_size)
    lines = ["// generated by cubie_b200.kernelgen (heterogeneous batch); do not edit"]
    lines += DEVICE_INCLUDES
    lines.append('#include "cbx_hetero.cuh"')
    names = []
    for k, (system, spec, gen) in enumerate(families):
        ns = f"cbxfam{k}"
        names.append(f"{ns}::Cfg")
        lines.append(f"namespace {ns} {{")
        lines += family_block(system, replace(spec, block_size=block, adjoint=False), gen, ns)
        lines.append(f"}}  // namespace {ns}")
    lines.append(f"CBX_DEFINE_HETERO_KERNEL({block}, {', '.join(names)})")
    return "\n".join(lines) + "\n"


def _generate_warp_kernel(system: SymbolicODE, spec: KernelSpec, gen: GeneratedSystem, warp_code=None):
    """Translation unit of the warp-per-system layout (``cbx_integrate_warp``)."""
    from .warpgen import generate_warp_system
    tab = spec.tableau
    if tab.kind != DIRK:
        raise NotImplementedError("the warp-per-system layout runs diagonally implicit RK tableaus")
    if spec.save_observables or spec.summarised_observable_indices:
        raise NotImplementedError("the warp-per-system layout saves and summarises states only")
    if spec.adjoint:
        raise NotImplementedError("no adjoint on the warp-per-system layout")
    if spec.block_size % 32:
        raise ValueError("block size must be a multiple of 32")
    warp_code = warp_code or generate_warp_system(system)
    spec = replace(spec, dense_prediction=False)
    lines = ["// generated by cubie_b200.kernelgen (warp-per-system layout); do not edit",
             f"// register cap: {int(spec.max_registers)}"]
    lines += DEVICE_INCLUDES
    lines.append('#include "cbx_warp.cuh"')
    lines.append("namespace cbxsys {")
    lines += family_block(system, spec, gen, "cbxsys", warp_source=warp_code.source)
    lines.append("}  // namespace cbxsys")
    lines.append("CBX_DEFINE_WARP_KERNEL(cbxsys::Cfg)")
    return GeneratedKernel(source="\n".join(lines) + "\n", system=gen, spec=spec)
