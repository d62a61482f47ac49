"""Run a generated integrator translation unit on the CPU (test harness).

The generated CUDA source is compiled by g++ with ``cbx_host_emu.h`` forced
in front, plus a small driver that loops over (block, thread) and calls the
kernel body for each emulated thread.  Inputs and outputs are numpy arrays
whose pointers go into the same ``cbx_solve_args`` struct the GPU launch
uses.
"""

import ctypes
import hashlib
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
DEVICE = ROOT / "cubie_b200" / "csrc" / "device"

DRIVER = r"""
cbx_dim3 threadIdx, blockIdx, blockDim, gridDim;
extern "C" void emu_launch(cbx_solve_args* a, int kernel, int grid, int block) {
    blockDim = {(unsigned)block, 1, 1};
    gridDim = {(unsigned)grid, 1, 1};
    for (int b = 0; b < grid; ++b) {
        for (int t = 0; t < block; ++t) {
            blockIdx = {(unsigned)b, 0, 0};
            threadIdx = {(unsigned)t, 0, 0};
            if (kernel == 0) cbx_integrate_plain(*a);
            else cbx_integrate_persistent(*a);
        }
    }
}
"""

ADJOINT_DRIVER = r"""
extern "C" void emu_adjoint(cbx_solve_args* a, cbx_adjoint_args* g, int phase, int grid, int block) {
    blockDim = {(unsigned)block, 1, 1};
    gridDim = {(unsigned)grid, 1, 1};
    for (int b = 0; b < grid; ++b) {
        for (int t = 0; t < block; ++t) {
            blockIdx = {(unsigned)b, 0, 0};
            threadIdx = {(unsigned)t, 0, 0};
            if (phase == 0) cbx_adjoint_forward(*a, *g);
            else cbx_adjoint_backward(*a, *g);
        }
    }
}
extern "C" long long emu_lane_bytes() { return (long long)sizeof(cbx_lane_probe); }
extern "C" long long emu_record_bytes() { return (long long)sizeof(cbx_seg_record_probe); }
extern "C" long long emu_tape_bytes() { return (long long)sizeof(cbx_tape_probe); }
"""

HETERO_DRIVER = r"""
cbx_dim3 threadIdx, blockIdx, blockDim, gridDim;
extern "C" void emu_hetero(cbx_hetero_args* h, int grid, int block) {
    blockDim = {(unsigned)block, 1, 1};
    gridDim = {(unsigned)grid, 1, 1};
    for (int b = 0; b < grid; ++b) {
        for (int t = 0; t < block; ++t) {
            blockIdx = {(unsigned)b, 0, 0};
            threadIdx = {(unsigned)t, 0, 0};
            cbx_integrate_hetero(*h);
        }
    }
}
"""

_cache = {}


def compile_emulated(source: str):
    h = hashlib.sha256((source + (HERE / "cbx_host_emu.h").read_text() + DRIVER + ADJOINT_DRIVER +
                        HETERO_DRIVER).encode())
    for f in sorted(Path(DEVICE).glob("*")):
        h.update(f.read_bytes())
    key = h.hexdigest()[:20]
    if key in _cache:
        return _cache[key]
    d = Path(tempfile.gettempdir()) / "cbx_emu"
    d.mkdir(exist_ok=True)
    src = d / f"{key}.cpp"
    so = d / f"{key}.so"
    if not so.exists():
        hetero = "CBX_DEFINE_HETERO_KERNEL(" in source
        src.write_text(source + ("" if hetero else DRIVER) + (HETERO_DRIVER if hetero else "") +
                       (ADJOINT_DRIVER if "CBX_DEFINE_ADJOINT_KERNELS(" in source else ""))
        cmd = ["g++", "-O1", "-std=c++17", "-shared", "-fPIC", "-include", str(HERE / "cbx_host_emu.h"),
               f"-I{DEVICE}", "-x", "c++", str(src), "-o", str(so)]
        subprocess.run(cmd, check=True, capture_output=True, text=True)
    lib = ctypes.CDLL(str(so))
    if "CBX_DEFINE_HETERO_KERNEL(" in source:
        lib.emu_hetero.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
    else:
        lib.emu_launch.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
    if "CBX_DEFINE_ADJOINT_KERNELS" in source:
        lib.emu_adjoint.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        lib.emu_lane_bytes.restype = ctypes.c_longlong
        lib.emu_record_bytes.restype = ctypes.c_longlong
        lib.emu_tape_bytes.restype = ctypes.c_longlong
    _cache[key] = lib
    return lib


def run_emulated(solver, inits, params, duration, settling_time=0.0, t0=0.0, kernel="plain",
                 durations=None, tol_scale=None, drivers=None):
    """Integrate with the solver's generated kernel on the CPU; returns a dict
    of output arrays laid out like ``SolveResult``."""
    from cubie_b200 import _native
    interp = None
    coeffs = None
    if drivers is not None:
        from cubie_b200.interpolator import ArrayInterpolator
        interp = ArrayInterpolator.from_system(solver.system, drivers, solver.precision)
        coeffs = np.ascontiguousarray(interp.coefficients, dtype=solver.precision)
    prep = solver.prepare(duration, settling_time, t0, interp, durations, load=False)
    spec = prep["spec"]
    gk = prep["gen"]
    lib = compile_emulated(gk.source)
    p = solver.precision
    n_runs = inits.shape[1]
    inits = np.ascontiguousarray(inits, dtype=p)
    params = np.ascontiguousarray(params, dtype=p) if params.size else np.zeros((1, n_runs), p)
    n_save, n_summ = prep["n_save"], prep["n_summ"]
    width = (len(spec.saved_state_indices) if spec.save_state else 0) + (1 if spec.save_time else 0)
    per_var = spec.summary.output_per_var if spec.summary else 0
    bufs = {
        "state": np.zeros((n_save, width, n_runs), p) if width else None,
        "obs": np.zeros((n_save, len(spec.saved_observable_indices), n_runs), p) if spec.save_observables else None,
        "state_sum": np.zeros((n_summ, len(spec.summarised_state_indices) * per_var, n_runs), p)
        if spec.summarised_state_indices and per_var else None,
        "obs_sum": np.zeros((n_summ, len(spec.summarised_observable_indices) * per_var, n_runs), p)
        if spec.summarised_observable_indices and per_var else None,
        "counters": np.zeros((n_save, 4, n_runs), np.int32) if spec.save_counters else None,
        "status": np.zeros((n_runs,), np.int32),
        "work": np.zeros((2,), np.int64),
        "totals": np.zeros((4,), np.int64),
    }
    dur = np.ascontiguousarray(durations, dtype=np.float64) if durations is not None else None
    tsc = np.ascontiguousarray(tol_scale, dtype=np.float64) if tol_scale is not None else None

    class _P:
        def __init__(self, arr):
            self.arr = arr

        def data_ptr(self):
            return self.arr.ctypes.data

    wrap = {k: (_P(v) if v is not None else None) for k, v in bufs.items()}

    class _W(dict):
        def __getitem__(self, k):
            return dict.__getitem__(self, k)

    wb = _W(wrap)
    wb["work"] = _P(bufs["work"])
    # make_args zeroes the work counter through .zero_(); emulate that
    bufs["work"][:] = 0
    wb["work"].zero_ = lambda: None
    args = solver.make_args(prep, wb, _P(inits), _P(params), _P(coeffs) if coeffs is not None else None, n_runs,
                            duration, settling_time, t0,
                            _P(dur) if dur is not None else None, _P(tsc) if tsc is not None else None)
    block = 32
    grid = (n_runs + block - 1) // block
    lib.emu_launch(ctypes.byref(args), 0 if kernel == "plain" else 1, grid, block)
    bufs["n_save"] = n_save
    bufs["n_summ"] = n_summ
    return bufs


def run_emulated_adjoint(solver, inits, params, duration, grad_state_fn, ckpt_every=64, max_ckpts=64,
                         drivers=None):
    """Forward with checkpoints and the reverse sweep of the adjoint kernels
    on the CPU.  ``grad_state_fn(state)`` returns dL/d(state rows) for the
    forward's state output.  Returns (state, status, grad_inits, grad_params)."""
    from cubie_b200 import _native
    interp = None
    coeffs = None
    if drivers is not None:
        from cubie_b200.interpolator import ArrayInterpolator
        interp = ArrayInterpolator.from_system(solver.system, drivers, solver.precision)
        coeffs = np.ascontiguousarray(interp.coefficients, dtype=solver.precision)
    prep = solver.prepare(duration, 0.0, 0.0, interp, None, load=False)
    spec = prep["spec"]
    lib = compile_emulated(prep["gen"].source)
    p = solver.precision
    n_runs = inits.shape[1]
    n = inits.shape[0]
    inits = np.ascontiguousarray(inits, dtype=p)
    params = np.ascontiguousarray(params, dtype=p) if params.size else np.zeros((1, n_runs), p)
    npar = solver.system.num_parameters
    n_save = prep["n_save"]
    width = (len(spec.saved_state_indices) if spec.save_state else 0) + (1 if spec.save_time else 0)
    state = np.zeros((n_save, width, n_runs), p)
    status = np.zeros((n_runs,), np.int32)
    work = np.zeros((2,), np.uint64)
    lane = int(lib.emu_lane_bytes())
    words = lane // 4
    ckpt = np.zeros((n_runs * max_ckpts * words,), np.uint32)
    count = np.zeros((n_runs,), np.int32)
    seg = np.zeros((ckpt_every * n_runs * int(lib.emu_record_bytes()) // 8 + 2,), np.float64)
    tape_entry = int(lib.emu_tape_bytes())
    tape_entry = tape_entry if tape_entry > 1 else 0
    cap = max_ckpts * ckpt_every
    v = 16 // tape_entry if tape_entry else 1
    tape = np.zeros((max(n_runs * (-(-cap // v) * v) * tape_entry // 8, 2),), np.float64)
    tape_flags = np.zeros((n_runs * (-(-cap // 32)),), np.uint32)
    step_count = np.zeros((n_runs,), np.int32)
    gi = np.zeros((n, n_runs), p)
    gp = np.zeros((max(npar, 1), n_runs), p)

    a = _native.SolveArgs()
    a.inits = inits.ctypes.data
    a.params = params.ctypes.data
    a.driver_coeffs = coeffs.ctypes.data if coeffs is not None else None
    a.state_out = state.ctypes.data
    a.status_out = status.ctypes.data
    a.work_counter = work.ctypes.data
    a.n_runs = a.run_stride = n_runs
    a.max_steps = int(solver.max_steps)
    a.duration = float(duration)
    a.save_stop = float(prep["save_stop"])
    a.summary_stop = float(prep["summary_stop"])
    a.n_save_rows = int(n_save)
    a.n_summary_rows = int(prep["n_summ"])
    g = _native.AdjointArgs()
    g.ckpt = ckpt.ctypes.data
    g.ckpt_count = count.ctypes.data
    g.lane_words = words
    g.ckpt_every = ckpt_every
    g.max_ckpts = max_ckpts
    if tape_entry > 0:
        g.tape, g.tape_flags, g.step_count = tape.ctypes.data, tape_flags.ctypes.data, step_count.ctypes.data
    lib.emu_adjoint(ctypes.byref(a), ctypes.byref(g), 0, 1, 32)
    grad_state = np.ascontiguousarray(grad_state_fn(state), dtype=p)
    g.seg = seg.ctypes.data
    g.grad_state = grad_state.ctypes.data
    g.grad_inits = gi.ctypes.data
    g.grad_params = gp.ctypes.data
    work[:] = 0
    lib.emu_adjoint(ctypes.byref(a), ctypes.byref(g), 1, 1, 32)
    return state, status, gi, gp[:npar]


def run_emulated_hetero(hetero, batches):
    """The heterogeneous kernel of a HeteroSolver on the CPU; returns one
    output dict per family (``state``, ``status``, ``totals``)."""
    from cubie_b200 import _native
    from cubie_b200.kernelgen import generate_hetero_kernel
    preps, outs, keep = [], [], []
    h = _native.HeteroArgs()
    first = [0]
    for k, (s, b) in enumerate(zip(hetero.solvers, batches)):
        prep = s.prepare(float(b["duration"]), durations=b.get("durations"), load=False)
        p = s.precision
        inits = np.ascontiguousarray(b["initial_values"], dtype=p)
        params = np.ascontiguousarray(b["parameters"], dtype=p)
        n = inits.shape[1]
        spec = prep["spec"]
        width = (len(spec.saved_state_indices) if spec.save_state else 0) + (1 if spec.save_time else 0)
        state = np.zeros((prep["n_save"], width, n), p)
        status = np.zeros((n,), np.int32)
        totals = np.zeros((4,), np.uint64)
        durs = None if b.get("durations") is None else np.ascontiguousarray(b["durations"], np.float64)
        a = _native.SolveArgs()
        a.inits, a.params = inits.ctypes.data, params.ctypes.data
        a.state_out, a.status_out, a.totals = state.ctypes.data, status.ctypes.data, totals.ctypes.data
        a.durations = durs.ctypes.data if durs is not None else None
        a.n_runs = a.run_stride = n
        a.max_steps = int(s.max_steps)
        a.duration = float(b["duration"])
        a.save_stop, a.summary_stop = float(prep["save_stop"]), float(prep["summary_stop"])
        a.n_save_rows, a.n_summary_rows = int(prep["n_save"]), int(prep["n_summ"])
        h.family[k] = a
        first.append(first[-1] + n)
        preps.append(prep)
        outs.append(dict(state=state, status=status, totals=totals))
        keep += [inits, params, durs]
    for k in range(9):
        h.first_run[k] = first[min(k, len(first) - 1)]
    work = np.zeros((8,), np.uint64)
    h.work_counter = work.ctypes.data
    h.n_families = len(hetero.solvers)
    src = generate_hetero_kernel([(s.system, pr["spec"], pr["gen"].system) for s, pr in zip(hetero.solvers, preps)])
    lib = compile_emulated(src)
    lib.emu_hetero(ctypes.byref(h), 1, 32)
    return outs
