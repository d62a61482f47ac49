"""ctypes binding of the C ABI in ``include/cubie_b200.h``.

The shared library ``libcubie_b200.so`` is built in-tree (see
``__graft_entry__.build`` / :func:`build_library`).  Nothing here falls
back to a CPU path: if the library or a GPU is missing, the calls raise.
"""

from __future__ import annotations

import ctypes
import hashlib
import os
import subprocess
import threading
from pathlib import Path
from typing import List, Optional, Sequence

PKG_DIR = Path(__file__).resolve().parent
LIB_PATH = PKG_DIR / "libcubie_b200.so"
DEVICE_INCLUDE = PKG_DIR / "csrc" / "device"
REPO_INCLUDE = PKG_DIR.parent / "include"

NVCC_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-shared",
              "-Xcompiler", "-fPIC", "-std=c++17"]


class NativeError(RuntimeError):
    """A C-ABI call returned an error code."""


class SolveArgs(ctypes.Structure):
    """Mirror of ``cbx_solve_args`` (cubie_b200/csrc/device/cbx_args.h)."""

    _fields_ = [
        ("inits", ctypes.c_void_p),
        ("params", ctypes.c_void_p),
        ("driver_coeffs", ctypes.c_void_p),
        ("state_out", ctypes.c_void_p),
        ("obs_out", ctypes.c_void_p),
        ("state_sum_out", ctypes.c_void_p),
        ("obs_sum_out", ctypes.c_void_p),
        ("counters_out", ctypes.c_void_p),
        ("status_out", ctypes.c_void_p),
        ("durations", ctypes.c_void_p),
        ("tol_scale", ctypes.c_void_p),
        ("work_counter", ctypes.c_void_p),
        ("totals", ctypes.c_void_p),
        ("abort_flag", ctypes.c_void_p),
        ("run_order", ctypes.c_void_p),
        ("n_runs", ctypes.c_longlong),
        ("run_stride", ctypes.c_longlong),
        ("max_steps", ctypes.c_longlong),
        ("duration", ctypes.c_double),
        ("warmup", ctypes.c_double),
        ("t0", ctypes.c_double),
        ("save_stop", ctypes.c_double),
        ("summary_stop", ctypes.c_double),
        ("n_save_rows", ctypes.c_int),
        ("n_summary_rows", ctypes.c_int),
    ]


class AdjointArgs(ctypes.Structure):
    """Mirror of ``cbx_adjoint_args`` (cubie_b200/csrc/device/cbx_args.h)."""

    _fields_ = [
        ("ckpt", ctypes.c_void_p),
        ("ckpt_count", ctypes.c_void_p),
        ("seg", ctypes.c_void_p),
        ("grad_state", ctypes.c_void_p),
        ("grad_inits", ctypes.c_void_p),
        ("grad_params", ctypes.c_void_p),
        ("lane_words", ctypes.c_longlong),
        ("ckpt_every", ctypes.c_int),
        ("max_ckpts", ctypes.c_int),
        ("tape", ctypes.c_void_p),
        ("tape_flags", ctypes.c_void_p),
        ("step_count", ctypes.c_void_p),
    ]


class HeteroArgs(ctypes.Structure):
    """Mirror of ``cbx_hetero_args`` (cubie_b200/csrc/device/cbx_args.h)."""

    MAX_FAMILIES = 8
    _fields_ = [
        ("family", SolveArgs * 8),
        ("first_run", ctypes.c_longlong * 9),
        ("work_counter", ctypes.c_void_p),
        ("n_families", ctypes.c_int),
        ("reserved", ctypes.c_int),
    ]


EXPORTED = (
    "cbx_version", "cbx_last_error", "cbx_nvrtc_version", "cbx_compile", "cbx_free",
    "cbx_module_load", "cbx_module_create", "cbx_module_destroy", "cbx_kernel_info",
    "cbx_occupancy", "cbx_solve", "cbx_device_info", "cbx_fp32_peak_probe", "cbx_flush_l2",
    "cbx_solve_noalloc", "cbx_adjoint_info", "cbx_adjoint_tape_bytes", "cbx_adjoint_launch", "cbx_solve_hetero",
)

_lib = None
_lock = threading.Lock()


def build_library(force: bool = False) -> Path:
    """Compile ``libcubie_b200.so`` with nvcc for sm_100a (no GPU needed)."""
    src = PKG_DIR / "csrc" / "runtime.cu"
    deps = [src, DEVICE_INCLUDE / "cbx_args.h", REPO_INCLUDE / "cubie_b200.h"]
    if LIB_PATH.exists() and not force:
        if all(LIB_PATH.stat().st_mtime >= d.stat().st_mtime for d in deps):
            return LIB_PATH
    cmd = ["nvcc", *NVCC_FLAGS, str(src), "-o", str(LIB_PATH),
           "-L/usr/local/cuda/lib64", "-L/usr/local/cuda/lib64/stubs",
           "-lnvrtc", "-ldl", "-Xlinker", "-rpath,/usr/local/cuda/lib64"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return LIB_PATH


def lib():
    """Load the shared library once (raises if it has not been built)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not LIB_PATH.exists():
            raise NativeError(f"{LIB_PATH.name} is not built; run cubie_b200._native.build_library() "
                              "or __graft_entry__.build()")
        L = ctypes.CDLL(str(LIB_PATH))
        L.cbx_version.restype = ctypes.c_int
        L.cbx_last_error.restype = ctypes.c_char_p
        L.cbx_nvrtc_version.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int)]
        L.cbx_compile.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p),
                                  ctypes.c_int, ctypes.POINTER(ctypes.c_void_p),
                                  ctypes.POINTER(ctypes.c_size_t), ctypes.c_char_p, ctypes.c_size_t]
        L.cbx_free.argtypes = [ctypes.c_void_p]
        L.cbx_free.restype = None
        L.cbx_module_load.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int,
                                      ctypes.POINTER(ctypes.c_void_p)]
        L.cbx_module_create.argtypes = [ctypes.c_char_p, ctypes.POINTER(ctypes.c_char_p), ctypes.c_int,
                                        ctypes.c_int, ctypes.POINTER(ctypes.c_void_p), ctypes.c_char_p,
                                        ctypes.c_size_t]
        L.cbx_module_destroy.argtypes = [ctypes.c_void_p]
        L.cbx_kernel_info.argtypes = [ctypes.c_void_p, ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 4
        L.cbx_occupancy.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]
        L.cbx_solve.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveArgs), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_void_p]
        L.cbx_device_info.argtypes = [ctypes.c_int] + [ctypes.POINTER(ctypes.c_int)] * 3
        L.cbx_fp32_peak_probe.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_float)]
        L.cbx_flush_l2.argtypes = [ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
        L.cbx_solve_noalloc.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveArgs), ctypes.c_int, ctypes.c_int,
                                        ctypes.c_void_p]
        L.cbx_solve_hetero.argtypes = [ctypes.c_void_p, ctypes.POINTER(HeteroArgs), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_void_p]
        L.cbx_adjoint_info.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong),
                                       ctypes.POINTER(ctypes.c_longlong)]
        L.cbx_adjoint_tape_bytes.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_longlong)]
        L.cbx_adjoint_launch.argtypes = [ctypes.c_void_p, ctypes.POINTER(SolveArgs), ctypes.POINTER(AdjointArgs),
                                         ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        _lib = L
        return L


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().cbx_last_error().decode(errors="replace")
        raise NativeError(f"{what} failed ({rc}): {msg}")


def nvrtc_version():
    a, b = ctypes.c_int(), ctypes.c_int()
    _check(lib().cbx_nvrtc_version(ctypes.byref(a), ctypes.byref(b)), "cbx_nvrtc_version")
    return a.value, b.value


def default_options(fast_math: bool = True, lineinfo: bool = True) -> List[str]:
    opts = ["--gpu-architecture=sm_100a", "--std=c++17", "-default-device",
            f"--include-path={DEVICE_INCLUDE}", "--ptxas-options=-v", "-DNDEBUG"]
    if lineinfo:
        opts.append("-lineinfo")
    if fast_math:
        opts.append("--use_fast_math")
    return opts


def _cache_dir() -> Path:
    d = os.environ.get("CUBIE_B200_CACHE_DIR")
    p = Path(d) if d else Path.home() / ".cache" / "cubie_b200"
    p.mkdir(parents=True, exist_ok=True)
    return p


def _headers_digest() -> str:
    h = hashlib.sha256()
    for f in sorted(DEVICE_INCLUDE.glob("*")):
        h.update(f.name.encode())
        h.update(f.read_bytes())
    return h.hexdigest()


def compile_cubin(source: str, options: Sequence[str], use_cache: bool = True) -> (bytes, str):
    """NVRTC-compile ``source``; returns (cubin bytes, compiler log).

    Cubins are cached on disk keyed by source, options, headers and NVRTC
    version (``CUBIE_B200_CACHE_DIR``, default ``~/.cache/cubie_b200``).
    """
    key = hashlib.sha256((source + "\0".join(options) + _headers_digest() + repr(nvrtc_version())).encode()).hexdigest()[:32]
    path = _cache_dir() / f"{key}.cubin"
    logp = _cache_dir() / f"{key}.log"
    if use_cache and path.exists():
        return path.read_bytes(), (logp.read_text() if logp.exists() else "")
    L = lib()
    opts = (ctypes.c_char_p * len(options))(*[o.encode() for o in options])
    out = ctypes.c_void_p()
    size = ctypes.c_size_t()
    log = ctypes.create_string_buffer(1 << 16)
    rc = L.cbx_compile(source.encode(), b"cbx_kernel.cu", opts, len(options), ctypes.byref(out),
                       ctypes.byref(size), log, len(log))
    _check(rc, "cbx_compile")
    data = ctypes.string_at(out, size.value)
    L.cbx_free(out)
    text = log.value.decode(errors="replace")
    if use_cache:
        tmp = path.with_suffix(f".tmp{os.getpid()}")
        tmp.write_bytes(data)
        os.replace(tmp, path)
        logp.write_text(text)
    return data, text


class Module:
    """A loaded integrator module (both kernels) on one device."""

    def __init__(self, cubin: bytes, device: int = 0, log: str = ""):
        self._handle = ctypes.c_void_p()
        self._cubin = cubin
        self.log = log
        self.device = device
        _check(lib().cbx_module_load(cubin, len(cubin), device, ctypes.byref(self._handle)), "cbx_module_load")

    def kernel_info(self, kernel: int = 0) -> dict:
        vals = [ctypes.c_int(-1) for _ in range(4)]
        _check(lib().cbx_kernel_info(self._handle, kernel, *[ctypes.byref(v) for v in vals]), "cbx_kernel_info")
        return dict(registers=vals[0].value, local_bytes=vals[1].value,
                    max_threads=vals[2].value, shared_bytes=vals[3].value)

    def occupancy(self, kernel: int, block: int) -> int:
        v = ctypes.c_int()
        _check(lib().cbx_occupancy(self._handle, kernel, block, ctypes.byref(v)), "cbx_occupancy")
        return v.value

    def launch(self, args: SolveArgs, kernel: int, block: int, grid: int = 0, stream: int = 0) -> None:
        _check(lib().cbx_solve(self._handle, ctypes.byref(args), kernel, block, grid, ctypes.c_void_p(stream)),
               "cbx_solve")

    def launch_hetero(self, args: "HeteroArgs", block: int, grid: int = 0, stream: int = 0) -> None:
        _check(lib().cbx_solve_hetero(self._handle, ctypes.byref(args), block, grid, ctypes.c_void_p(stream)),
               "cbx_solve_hetero")

    def adjoint_sizes(self) -> tuple:
        """(bytes of one checkpoint image, bytes of one replay record)."""
        v, r = ctypes.c_longlong(), ctypes.c_longlong()
        _check(lib().cbx_adjoint_info(self._handle, ctypes.byref(v), ctypes.byref(r)), "cbx_adjoint_info")
        return v.value, r.value

    def adjoint_tape_bytes(self) -> int:
        """Bytes of one step-size tape entry (0: the module keeps no tape)."""
        v = ctypes.c_longlong()
        _check(lib().cbx_adjoint_tape_bytes(self._handle, ctypes.byref(v)), "cbx_adjoint_tape_bytes")
        return v.value

    def adjoint_launch(self, args: SolveArgs, adj: AdjointArgs, phase: int, block: int, grid: int = 0,
                       stream: int = 0) -> None:
        _check(lib().cbx_adjoint_launch(self._handle, ctypes.byref(args), ctypes.byref(adj), phase, block, grid,
                                        ctypes.c_void_p(stream)), "cbx_adjoint_launch")

    def __del__(self):
        try:
            if self._handle and _lib is not None:
                _lib.cbx_module_destroy(self._handle)
        except Exception:
            pass


def device_info(device: int = 0) -> dict:
    sm, a, b = ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    _check(lib().cbx_device_info(device, ctypes.byref(sm), ctypes.byref(a), ctypes.byref(b)), "cbx_device_info")
    return dict(sm_count=sm.value, cc=(a.value, b.value))


def fp32_peak(device: int = 0) -> float:
    """Measured FP32 FMA throughput in FLOP/s."""
    fl, ms = ctypes.c_double(), ctypes.c_float()
    _check(lib().cbx_fp32_peak_probe(device, ctypes.byref(fl), ctypes.byref(ms)), "cbx_fp32_peak_probe")
    return fl.value / (ms.value * 1e-3)


def flush_l2(buffer_ptr: int, nbytes: int, stream: int = 0) -> None:
    _check(lib().cbx_flush_l2(ctypes.c_void_p(buffer_ptr), nbytes, ctypes.c_void_p(stream)), "cbx_flush_l2")
