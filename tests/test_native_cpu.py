"""The C-ABI library and NVRTC compilation, without a GPU."""

import re
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def test_library_exports_every_declared_symbol():
    from cubie_b200 import _native
    lib = _native.lib()
    header = (ROOT / "include" / "cubie_b200.h").read_text()
    declared = set(re.findall(r"\b(cbx_[a-z0-9_]+)\s*\(", header))
    assert declared, "no declarations found"
    for name in sorted(declared):
        assert hasattr(lib, name), f"{name} declared in the header but not exported"
    assert set(_native.EXPORTED) == declared


def test_version_and_nvrtc():
    from cubie_b200 import _native
    assert _native.lib().cbx_version() >= 10000
    major, minor = _native.nvrtc_version()
    assert (major, minor) >= (12, 8)


def test_args_struct_layout_matches_header():
    import ctypes
    from cubie_b200 import _native
    # 14 pointers, 3 int64, 5 float64, 2 int32
    assert ctypes.sizeof(_native.SolveArgs) == 15 * 8 + 3 * 8 + 5 * 8 + 2 * 4
    # 6 pointers, 1 int64, 2 int32, then the three tape pointers
    assert ctypes.sizeof(_native.AdjointArgs) == 9 * 8 + 8 + 2 * 4
    assert _native.AdjointArgs.tape.offset == 6 * 8 + 8 + 2 * 4


def test_compile_error_is_reported():
    from cubie_b200 import _native
    with pytest.raises(_native.NativeError, match="NVRTC"):
        _native.compile_cubin("this is not cuda", _native.default_options(), use_cache=False)


def test_launch_without_driver_fails_loudly():
    from cubie_b200 import _native
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a GPU is present")
    except Exception:
        pass
    with pytest.raises(_native.NativeError):
        _native.device_info(0)


@pytest.mark.parametrize("algorithm,linear", [
    ("dormand-prince-54", "minimal_residual"),
    ("ros3p", "minimal_residual"),
    ("ros3p", "bicgstab"),
    ("ros3p", "gmres"),
    ("radau", "minimal_residual"),
    ("radau", "gmres"),
    ("l_stable_dirk_3", "bicgstab"),
    ("l_stable_sdirk_4", "steepest_descent"),
])
@pytest.mark.parametrize("mixed", [False, True])
def test_generated_kernels_compile_for_sm100a(algorithm, linear, mixed):
    from cubie_b200 import _native, create_ODE_system
    from cubie_b200.solver import Solver
    sysm = create_ODE_system(["dx = y", "dy = mu * (1 - x**2) * y - x"], states={"x": 2.0, "y": 0.0},
                             parameters={"mu": 10.0})
    solver = Solver(sysm, algorithm=algorithm, linear_correction_type=linear, mixed_precision=mixed,
                    save_every=0.1, output_types=["state", "time", "iteration_counters", "mean", "max"],
                    summarise_every=0.5)
    prep_timing = solver._timing(1.0)
    spec = solver.kernel_spec(prep_timing)
    from cubie_b200.kernelgen import generate_kernel
    gk = generate_kernel(sysm, spec)
    cubin, log = _native.compile_cubin(gk.source, _native.default_options())
    assert len(cubin) > 1000
    assert "cbx_integrate_persistent" in log and "cbx_integrate_plain" in log
    assert "spill stores" in log
