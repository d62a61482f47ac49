"""The generated device code, compiled for the host, against the reference's
own outputs (no GPU).

Every case in ``tests/golden/cases.py`` runs through the engine's generated
CUDA translation unit built with g++ (``tests/host_emu``: the same kernel
source, one host thread per run) and is compared with the fixture the
reference's unmodified kernels produced under Numba's CUDA simulator.  The
host build performs no fused multiply-adds and the simulator none either,
so wherever the generated system code evaluates each expression in the
same order as the reference's printer the two agree bit for bit: status
codes, iteration counters and every saved state.  That holds for every
algorithm family (explicit, diagonally and fully implicit, Rosenbrock),
every step controller, both precisions and the chaotic Lorenz cases.  The
remaining cases differ only in the rounding of the system's own
expressions (the reference's expression engine orders some sums and
quotients differently, e.g. ``V**3/3`` and the driver spline's Horner
form), and are held to the tolerance envelope instead.
"""

from pathlib import Path

import numpy as np
import pytest

from cases import CASES, case_drivers, case_inputs
from host_emu.emu import run_emulated
from parity_utils import build_case_system, tol_units

from cubie_b200 import Solver

GOLDEN = Path(__file__).resolve().parent / "golden"

# expression order differs from the reference's printer in these systems
ROUNDING_ONLY = {"fhn_dp54_peaks_f32": 10.0, "fhn_dp54_derivs_f32": 10.0, "fhn_dp54_derivs_f64": 1e-3,
                 "driven_dp54_clamped_f64": 1e-3, "driven_ros3p_clamped_f64": 1e-3,
                 "hh64_dirk3_bicgstab_f32": 10.0, "rober_dae_dirk3_f64": 1e-3, "rober_dae_radau_f64": 1e-3}
# BiCGSTAB on the DAE's coupled stage system (singular mass matrix): its
# iteration counts follow last-bit differences of the expressions; the step
# and rejection counts and the states do not
KRYLOV_SENSITIVE = {"rober_dae_radau_f64"}


@pytest.mark.parametrize("name", list(CASES))
def test_emulated_kernel_reproduces_reference(name):
    case = CASES[name]
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    kw = dict(case["kwargs"])
    solver = Solver(build_case_system(case), algorithm=case["algorithm"], **kw)
    inits, params = case_inputs(case)
    out = run_emulated(solver, inits, params, case["duration"], kernel="plain", drivers=case_drivers(case))
    assert out["status"].tolist() == ref["status"].tolist()
    if "iteration_counters" in ref.files:
        if name in ROUNDING_ONLY:
            # rounding-level differences may move a Newton or Krylov count
            # by one; the step and rejection counts stay the same
            np.testing.assert_array_equal(out["counters"][:, 2:, :], ref["iteration_counters"][:, 2:, :])
            if name not in KRYLOV_SENSITIVE:
                assert np.max(np.abs(out["counters"][:, :2, :] - ref["iteration_counters"][:, :2, :])) <= 1
        else:
            np.testing.assert_array_equal(out["counters"], ref["iteration_counters"])
    assert out["state"].shape == ref["state"].shape
    if name in ROUNDING_ONLY:
        assert tol_units(out["state"], ref["state"], kw["atol"], kw["rtol"]) < ROUNDING_ONLY[name]
        if "state_summaries" in ref.files and out.get("state_sum") is not None:
            assert tol_units(out["state_sum"], ref["state_summaries"], kw["atol"], kw["rtol"]) < ROUNDING_ONLY[name]
    else:
        np.testing.assert_array_equal(out["state"], ref["state"])
        if "state_summaries" in ref.files and out.get("state_sum") is not None:
            np.testing.assert_array_equal(out["state_sum"], ref["state_summaries"])


DIRECT_CASES = ["vdp_ros3p_f32", "vdp_ros3p_bicgstab_f64", "vdp_rodas3p_f64", "vdp_radau_f64", "vdp_radau_f32",
                "vdp_sdirk4_f64", "vdp_kvaerno3_f64", "vdp_gl4_f64", "vdp_cn_f64"]


@pytest.mark.parametrize("name", DIRECT_CASES)
def test_emulated_direct_solver_matches_oracle(name):
    """The register LU (``linear_correction_type='direct'``) against the
    oracle's exact dense solve: same statuses and step/rejection counts,
    states within a small fraction of the tolerance envelope in float64."""
    from parity_utils import run_oracle
    case = CASES[name]
    kw = dict(case["kwargs"], linear_correction_type="direct", output_types=["state", "time", "iteration_counters"])
    solver = Solver(build_case_system(case), algorithm=case["algorithm"], **kw)
    inits, params = case_inputs(case)
    out = run_emulated(solver, inits, params, case["duration"], kernel="plain")
    orc = run_oracle(case, linear_correction_type="direct", output_types=["state", "time", "iteration_counters"])
    assert out["status"].tolist() == orc["status"].tolist()
    np.testing.assert_array_equal(out["counters"][:, 2:, :], orc["iteration_counters"][:, 2:, :])
    bar = 1e-3 if case["precision"] == "float64" else 10.0
    assert tol_units(out["state"], orc["state"], kw["atol"], kw["rtol"]) < bar
