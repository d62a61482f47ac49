"""Launch-shape autotuner for the integration kernels.

For one solver configuration it compiles the kernel at a set of launch
shapes (block size, and a minimum of resident blocks per SM, which caps
registers per thread), times the persistent launch of each on a sample of
the caller's batch with CUDA events, and keeps the fastest.  Results are
cached on disk per configuration and GPU (``CUBIE_B200_CACHE_DIR``, default
``~/.cache/cubie_b200``, file ``autotune.json``), so a configuration is
tuned once per machine.  The reference picks its block size by a
shared-memory limit only (``limit_blocksize``,
src/cubie/batchsolving/BatchSolverKernel.py:780-830).

``Solver(..., block_size="auto")`` runs it on the first solve.
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


def _cache_path() -> Path:
    d = os.environ.get("CUBIE_B200_CACHE_DIR")
    p = Path(d) if d else Path.home() / ".cache" / "cubie_b200"
    p.mkdir(parents=True, exist_ok=True)
    return p / "autotune.json"


def config_key(solver, duration: float, gpu_name: str) -> str:
    """Configuration identity without the launch shape."""
    variant = copy.copy(solver)
    variant.block_size, variant.min_blocks_per_sm = 128, 1
    variant.__dict__["_prepared"] = {}
    src = variant.prepare(duration, load=False)["gen"].source
    return hashlib.sha256((src + gpu_name).encode()).hexdigest()[:24]


def choose(timings: Dict[Tuple[int, int], float]) -> Tuple[int, int]:
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


def variant(solver, block: int, min_blocks: int):
    v = copy.copy(solver)
    v.block_size = int(block)
    v.min_blocks_per_sm = int(min_blocks)
    v.__dict__["_prepared"] = {}
    return v


def autotune(solver, inits, params, duration: float, durations=None, candidates: Optional[Sequence] = None,
             repeats: int = 2, timer: Optional[Callable] = None, use_cache: bool = True) -> Dict:
    """Time the persistent launch at each candidate shape on the given
    batch (device tensors or arrays ``[n_states, n]``, ``[n_params, n]``)
    and return ``{"block", "min_blocks", "timings_ms", "cached"}``.

    ``timer(variant_solver) -> ms`` replaces the GPU measurement (tests)."""
    cands = [tuple(c) for c in (candidates or DEFAULT_CANDIDATES)]
    gpu = "cpu-test" if timer is not None else _gpu_name(solver.device)
    key = config_key(solver, duration, gpu)
    store = {}
    path = _cache_path()
    if use_cache and path.exists():
        try:
            store = json.loads(path.read_text())
        except ValueError:
            store = {}
    if use_cache and key in store:
        hit = store[key]
        return dict(block=hit["block"], min_blocks=hit["min_blocks"], timings_ms=hit["timings_ms"], cached=True)
    measure = timer or _gpu_timer(inits, params, duration, durations, repeats)
    timings = {}
    for block, minb in cands:
        try:
            timings[(block, minb)] = float(measure(variant(solver, block, minb)))
        except Exception:  # a shape that cannot compile or launch is skipped
            timings[(block, minb)] = float("nan")
    block, minb = choose(timings)
    result = dict(block=block, min_blocks=minb, timings_ms={f"{b}x{m}": t for (b, m), t in timings.items()})
    if use_cache:
        store[key] = result
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        tmp.write_text(json.dumps(store, indent=1, sort_keys=True))
        os.replace(tmp, path)
    return dict(result, cached=False)


def _gpu_name(device: int) -> str:
    torch = __import__("torch")
    return torch.cuda.get_device_name(device)


def _gpu_timer(inits, params, duration, durations, repeats):
    torch = __import__("torch")

    def measure(v) -> float:
        dev = torch.device("cuda", v.device)
        tdt = torch.float32 if v.precision == np.float32 else torch.float64
        it = torch.as_tensor(inits, device=dev).to(tdt).contiguous()
        pt = torch.as_tensor(params, device=dev).to(tdt).contiguous()
        dt = torch.as_tensor(durations, device=dev, dtype=torch.float64) if durations is not None else None
        n = int(it.shape[1])
        prep = v.prepare(duration, durations=durations)
        bufs = v.allocate_outputs(prep, n, dev, tdt)
        stream = torch.cuda.current_stream(dev)
        best = float("inf")
        for _ in range(max(1, repeats)):
            a = v.make_args(prep, bufs, it, pt, None, n, duration, 0.0, 0.0, dt)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            prep["module"].launch(a, 1, v.block_size, 0, stream.cuda_stream)
            e1.record(stream)
            e1.synchronize()
            best = min(best, e0.elapsed_time(e1))
        return best

    return measure
