"""Launch-shape autotuner for the integration kernels.

For one solver configuration it compiles the kernel at a set of launch
shapes (block size, i.e. warps per block, and a minimum of resident blocks
per SM, which caps registers per thread) and, for the warp-per-system
layout, scratch placements (the stage solve's scratch vectors in the warp's
shared memory, in the lanes' local memory, or passed in registers; the reference
makes the same shared-versus-local choice per buffer with a fixed table,
src/cubie/integrators/memory_heuristics.py:99-116), times the persistent
launch of each on a sample of the caller's batch with CUDA events, and
keeps the fastest.  Results are
cached on disk per configuration and GPU (``CUBIE_B200_CACHE_DIR``, default
``~/.cache/cubie_b200``, file ``autotune.json``), so a configuration is
tuned once per machine.  The reference picks its block size by a
shared-memory limit only (``limit_blocksize``,
src/cubie/batchsolving/BatchSolverKernel.py:780-830).

``Solver(..., block_size="auto")`` (shapes) and
``Solver(..., layout="warp", scratch_placement="auto")`` (shapes and
placements) run it on the first solve.
"""

from __future__ import annotations

import copy
import hashlib
import json
import os
from pathlib import Path
from typing import Callable, Dict, Iterable, List, Optional, Sequence, Tuple

import numpy as np

DEFAULT_CANDIDATES: Tuple[Tuple[int, int], ...] = ((128, 1), (64, 1), (256, 1), (32, 1), (128, 4), (128, 6),
                                                    (64, 8), (256, 2))


# warp-per-system layout: fewer shapes (each compile of a large system is
# costly), each with the scratch placements; the register cap matters for
# the placements that pass vectors by address (with "registers" the call
# keeps them live and the compiler takes what it needs)
WARP_CANDIDATES: Tuple[Tuple[int, int, str, int], ...] = tuple(
    (b, 1, p, r) for b in (128, 64) for p in ("shared", "local") for r in (0, 168)) + tuple(
    (b, 1, "registers", 0) for b in (128, 64))


# runs of the caller's batch timed per candidate
SAMPLE_RUNS = 8192


def default_candidates(solver) -> List[Tuple]:
    if solver.layout == "warp":
        if getattr(solver, "placement_pending", False):
            return list(WARP_CANDIDATES)
        return [(b, 1, solver.scratch_placement, r) for b in (128, 64) for r in (0, 168)]
    return list(DEFAULT_CANDIDATES)


def _cache_path() -> Path:
    d = os.environ.get("CUBIE_B200_CACHE_DIR")
    p = Path(d) if d else Path.home() / ".cache" / "cubie_b200"
    p.mkdir(parents=True, exist_ok=True)
    return p / "autotune.json"


def config_key(solver, duration: float, gpu_name: str) -> str:
    """Configuration identity without the launch shape."""
    variant = copy.copy(solver)
    variant.block_size, variant.min_blocks_per_sm = 128, 1
    variant.scratch_placement = "shared"
    variant.max_registers = 0
    variant.__dict__["_prepared"] = {}
    src = variant.prepare(duration, load=False)["gen"].source
    # the device headers are included by path: their contents are part of
    # the configuration's identity too
    from . import _native
    return hashlib.sha256((src + _native._headers_digest() + gpu_name).encode()).hexdigest()[:24]


def choose(timings: Dict[Tuple, float]) -> Tuple:
    """Fastest shape; ties go to the earlier candidate (stable order)."""
    best = None
    for shape, ms in timings.items():
        if ms is None or not np.isfinite(ms):
            continue
        if best is None or ms < timings[best]:
            best = shape
    if best is None:
        raise RuntimeError("no launch shape could be timed")
    return best


def variant(solver, block: int, min_blocks: int, placement: Optional[str] = None,
            max_registers: Optional[int] = None):
    v = copy.copy(solver)
    v.block_size = int(block)
    v.min_blocks_per_sm = int(min_blocks)
    if placement is not None:
        v.scratch_placement = placement
    if max_registers is not None:
        v.max_registers = int(max_registers)
    v.__dict__["_prepared"] = {}
    return v


def _label(shape: Tuple) -> str:
    return "x".join(str(x) for x in shape)


def autotune(solver, inits, params, duration: float, durations=None, candidates: Optional[Sequence] = None,
             repeats: int = 2, timer: Optional[Callable] = None, use_cache: bool = True, interp=None) -> Dict:
    """Time the persistent launch at each candidate shape on the given
    batch (device tensors or arrays ``[n_states, n]``, ``[n_params, n]``)
    and return ``{"block", "min_blocks", "timings_ms", "cached"}``.

    ``timer(variant_solver) -> ms`` replaces the GPU measurement (tests)."""
    cands = [tuple(c) for c in (candidates or default_candidates(solver))]
    gpu = "cpu-test" if timer is not None else _gpu_name(solver.device)
    key = config_key(solver, duration, gpu)
    store = {}
    path = _cache_path()
    if use_cache and path.exists():
        try:
            store = json.loads(path.read_text())
        except ValueError:
            store = {}
    key = key + "".join(f"|{_label(c)}" for c in cands)
    if use_cache and key in store:
        hit = store[key]
        return dict(block=hit["block"], min_blocks=hit["min_blocks"], placement=hit.get("placement"),
                    max_registers=hit.get("max_registers"), timings_ms=hit["timings_ms"], cached=True)
    measure = timer or _gpu_timer(inits, params, duration, durations, repeats, interp)
    if timer is None:
        _precompile([variant(solver, *c) for c in cands], duration, durations, interp)
    timings = {}
    for shape in cands:
        try:
            timings[shape] = float(measure(variant(solver, *shape)))
        except Exception:  # a shape that cannot compile or launch is skipped
            timings[shape] = float("nan")
    best = choose(timings)
    result = dict(block=best[0], min_blocks=best[1], placement=best[2] if len(best) > 2 else None,
                  max_registers=best[3] if len(best) > 3 else None,
                  timings_ms={_label(c): t for c, t in timings.items()})
    if use_cache:
        store[key] = result
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        tmp.write_text(json.dumps(store, indent=1, sort_keys=True))
        os.replace(tmp, path)
    return dict(result, cached=False)


def _precompile(variants, duration, durations, interp) -> None:
    """Compile every candidate at once on the host's cores (NVRTC releases
    the interpreter lock), then load the modules one by one; the timing
    loop then finds them loaded."""
    from concurrent.futures import ThreadPoolExecutor
    specs = []
    for v in variants:
        timing = v._timing(float(duration))
        specs.append(v.kernel_spec(timing, interp.device_meta() if interp is not None else None))
    if variants:
        variants[0]._generate(specs[0])   # the symbolic part once, shared by every variant
    workers = max(1, min(len(variants), os.cpu_count() or 1))

    def build(pair):
        v, spec = pair
        try:
            return v.compile_for(spec)
        except Exception:  # the timing loop reports the candidate as failed
            return None

    with ThreadPoolExecutor(workers) as ex:
        results = list(ex.map(build, zip(variants, specs)))
    for v, spec, res in zip(variants, specs, results):
        if res is not None:
            try:
                v.module_for(spec, compiled=res)
            except Exception:
                pass


def _gpu_name(device: int) -> str:
    torch = __import__("torch")
    return torch.cuda.get_device_name(device)


def _gpu_timer(inits, params, duration, durations, repeats, interp=None):
    """Best of ``repeats`` persistent launches of a variant on the caller's
    batch (driven systems with the caller's driver table)."""
    torch = __import__("torch")

    def measure(v) -> float:
        dev = torch.device("cuda", v.device)
        tdt = torch.float32 if v.precision == np.float32 else torch.float64
        # a sample of the batch (a few resident waves) is timed
        k = min(int(inits.shape[1]), SAMPLE_RUNS)
        it = torch.as_tensor(inits[:, :k], device=dev).to(tdt).contiguous()
        pt = torch.as_tensor(params[:, :k], device=dev).to(tdt).contiguous()
        dt = torch.as_tensor(np.asarray(durations)[:k] if not hasattr(durations, "device") else durations[:k],
                             device=dev, dtype=torch.float64) if durations is not None else None
        n = int(it.shape[1])
        prep = v.prepare(duration, interp=interp, durations=durations)
        coeff = None
        if interp is not None:
            coeff = torch.as_tensor(interp.coefficients.astype(v.precision), device=dev).contiguous()
        elif v.system.num_drivers > 0:
            raise ValueError("a driven system is tuned with its driver table")
        bufs = v.allocate_outputs(prep, n, dev, tdt)
        stream = torch.cuda.current_stream(dev)
        best = float("inf")
        for _ in range(max(1, repeats)):
            a = v.make_args(prep, bufs, it, pt, coeff, n, duration, 0.0, 0.0, dt)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prep["module"].launch(a, v.launch_kind, v.block_size, 0, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    return measure
