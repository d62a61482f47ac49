"""The headline and cable configurations against the reference's own kernels.

The stiff Van der Pol fixtures (mu = 100, 300, 1000, one relaxation
transition per run inside the window) were made by the reference's kernels
with their defaults: FP32 stepping with minimal-residual Krylov and the
Neumann preconditioner for the stage systems (FP64 cases with BiCGSTAB).
The 64-compartment Hodgkin-Huxley cable fixture (256 states,
l_stable_dirk_3 + Newton + BiCGSTAB, step current through the array
interpolator, first spike inside the window) was made the same way.  Here
the engine runs the bench's configurations on the same inputs:

* the persistent launch in mixed precision (FP32 stepping, FP64 time,
  control and norms), with the register LU the headline uses and with
  matrix-free GMRES, the workload's literal solver;
* the warp-per-run layout for the cable, in FP32 and in mixed precision.

Bars: the same status words as the reference; saved states (and
summaries) within rtol/atol x 10 of the reference for the reference's own
algorithm; for the headline's exact stage solves, within rtol/atol x 10 of
the same method in FP64 and no further from an FP64 truth (SciPy Radau at
1e-12) than that FP64 solve.
"""

from pathlib import Path

import numpy as np
import pytest

from cases import CASES, case_drivers, case_inputs
from parity_utils import build_case_system, run_oracle, tol_units

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu

STIFF32 = ["vdp_stiff_ros3p_f32", "vdp_stiff_radau_f32"]
STIFF64 = ["vdp_stiff_ros3p_f64", "vdp_stiff_radau_f64"]


def _solve(case, **extra):
    from cubie_b200 import Solver
    kw = dict(case["kwargs"])
    kw.update(case.get("engine", {}))
    kw.update(extra)
    solver = Solver(build_case_system(case), algorithm=case["algorithm"], **kw)
    prec = np.dtype(case["precision"]).type
    inits, params = case_inputs(case)
    return solver.solve(inits.astype(prec), params.astype(prec), drivers=case_drivers(case),
                        duration=case["duration"], nan_error_trajectories=False)


def _vdp_truth(case):
    """FP64 truth at the saved times: SciPy Radau at rtol = atol = 1e-12."""
    from scipy.integrate import solve_ivp
    inits, params = case_inputs(case)
    every = case["kwargs"]["save_every"]
    times = np.arange(0.0, case["duration"] + 0.5 * every, every)
    out = np.zeros((len(times), 2, inits.shape[1]))
    for r in range(inits.shape[1]):
        mu = float(params[0, r])
        sol = solve_ivp(lambda t, y: [y[1], mu * (1 - y[0] ** 2) * y[1] - y[0]], (0.0, case["duration"]),
                        inits[:, r], method="Radau", rtol=1e-12, atol=1e-12, t_eval=times,
                        jac=lambda t, y: [[0.0, 1.0], [-2.0 * mu * y[0] * y[1] - 1.0, mu * (1.0 - y[0] ** 2)]])
        out[:, :, r] = sol.y.T
    return out


def _errors(state, truth, atol, rtol):
    return np.max(np.abs(np.asarray(state[:, :2], np.float64) - truth) / (atol + rtol * np.abs(truth)),
                  axis=(0, 1))


@pytest.mark.parametrize("name", STIFF32)
def test_reference_settings_persistent_matches_reference(cuda_device, name):
    """The reference's own settings (FP32, its default Krylov solver) on the
    persistent launch: statuses and saved states within rtol/atol x 10."""
    case = CASES[name]
    atol, rtol = case["kwargs"]["atol"], case["kwargs"]["rtol"]
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    res = _solve(case, kernel="persistent")
    assert res.status_codes.tolist() == ref["status"].tolist()
    assert tol_units(res.state, ref["state"], atol, rtol) < 10


@pytest.mark.parametrize("lin", ["direct", "gmres"])
@pytest.mark.parametrize("name", STIFF32)
def test_headline_configuration_matches_fp64_same_method(cuda_device, name, lin):
    """The headline settings (persistent launch, mixed precision, register
    LU or matrix-free GMRES, no preconditioner) on the stiff runs.

    With exact stage solves ROS3P's global error right after a relaxation
    transition at mu = 1000 is a few hundred tolerance units even in FP64:
    the local error control does not bound the error carried through the
    fast jump.  The reference's FP32 minimal-residual default happens to
    land closer (its inexact stage solves force ~13x more, smaller steps),
    so the headline is held to its own method computed in FP64 (the oracle
    with exact stage solves): the same statuses as the reference; within 1
    tolerance unit of the FP64 solve on every row before the jump (FP32
    stepping with FP64 control keeps FP64 accuracy there) and within 10 on
    the final row; and an error against the truth of the same order as the
    FP64 solve's own (a rounding-level shift of the jump moves the rows
    right after it by up to a few times the method's error)."""
    case = CASES[name]
    atol, rtol = case["kwargs"]["atol"], case["kwargs"]["rtol"]
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    res = _solve(case, kernel="persistent", mixed_precision=True, linear_correction_type=lin,
                 preconditioner_type=None)
    assert res.status_codes.tolist() == ref["status"].tolist()
    same = run_oracle(case, linear_correction_type="direct", preconditioner_type=None, precision=np.float64)
    ys = np.asarray(same["state"][:, :2], np.float64)
    d = np.max(np.abs(np.asarray(res.state[:, :2], np.float64) - ys) / (atol + rtol * np.abs(ys)), axis=1)
    before_jump = ys[:, 0, :] > 0.0          # every run starts at x0 > 1 and jumps to x ~ -2
    assert d[before_jump].max() < 1.0, d
    assert d[-1].max() < 10.0, d
    truth = _vdp_truth(case)
    e_same = _errors(same["state"], truth, atol, rtol)
    e_new = _errors(res.state, truth, atol, rtol)
    assert np.all(e_new <= 4.0 * e_same + 1.0), (e_new, e_same)


@pytest.mark.parametrize("name", STIFF64)
def test_gmres_and_direct_match_oracle_direct(cuda_device, name):
    """Matrix-free GMRES and the register LU against the oracle's exact
    dense stage solves in FP64: same statuses, states within 0.1 tolerance
    units (GMRES stops at the reference's Krylov tolerance), and for the
    LU the same step and rejection counts; both no further from the FP64
    truth than max(2 x the reference's error, 1 unit)."""
    case = CASES[name]
    atol, rtol = case["kwargs"]["atol"], case["kwargs"]["rtol"]
    out = run_oracle(case, linear_correction_type="direct")
    truth = _vdp_truth(case)
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    e_ref = _errors(ref["state"], truth, atol, rtol)
    for lin in ("gmres", "direct"):
        res = _solve(case, kernel="persistent", linear_correction_type=lin, preconditioner_type=None)
        assert res.status_codes.tolist() == out["status"].tolist()
        assert tol_units(res.state, out["state"], atol, rtol) < 0.1, lin
        if lin == "direct":
            np.testing.assert_array_equal(res.iteration_counters[:, 2:, :], out["iteration_counters"][:, 2:, :])
        e_new = _errors(res.state, truth, atol, rtol)
        assert np.all(e_new <= np.maximum(2.0 * e_ref, 1.0)), (lin, e_new, e_ref)


@pytest.mark.parametrize("mixed", [False, True])
def test_warp_cable_matches_reference(cuda_device, mixed):
    """The 256-state cable in the warp-per-run layout (the bench's cable
    kernel) against the reference's thread-per-run kernel: statuses, the
    64 saved voltages and their mean/max summaries within rtol/atol x 10."""
    name = "hh64_dirk3_bicgstab_f32"
    case = CASES[name]
    atol, rtol = case["kwargs"]["atol"], case["kwargs"]["rtol"]
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    res = _solve(case, mixed_precision=mixed)
    assert res.status_codes.tolist() == ref["status"].tolist()
    assert res.state.shape == ref["state"].shape
    assert tol_units(res.state, ref["state"], atol, rtol) < 10
    assert tol_units(res.state_summaries, ref["state_summaries"], atol, rtol) < 10
