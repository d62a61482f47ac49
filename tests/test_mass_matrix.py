"""Constant mass matrices (``create_ODE_system(..., mass=M)``: M y' = f).

The reference's implicit steps apply M in their linear operators
(beta M v - gamma a h J v) and residuals (beta M u - gamma h f), and reject
explicit algorithms for a system with a mass matrix
(SingleIntegratorRunCore.py:765-780).  The fixtures of the reference's own
kernels (a Van der Pol system with a full M under Radau IIA5, the Robertson
index-1 DAE with M = diag(1, 1, 0) under l_stable_dirk_3 and Radau) are in
tests/golden and go through the parity tests; these tests cover the rules
and ROS3P with a full M, which has no reference fixture: the reference
forms the Rosenbrock stage term C_ij K_j / h without M
(generic_rosenbrock_w.py:682-698) and fails on it (STEP_TOO_SMALL, or no
progress: its kernels did not finish the case under the simulator).  The
engine and the oracle apply M to that term (Hairer & Wanner, Solving ODEs
II, VI.4); with a nonsingular M the result is checked against SciPy on the
explicit form y' = M^-1 f.
"""

import numpy as np
import pytest

from cases import CASES, VDP_MASS, ROBER_DAE, case_inputs
from parity_utils import build_case_system, run_oracle, tol_units


def _ros3p_mass_case(lin):
    return dict(system=VDP_MASS, algorithm="ros3p", precision="float64", inputs=("vdp", 3, 73, [1.0, 3.0, 10.0]),
                duration=2.0, kwargs=dict(rtol=1e-7, atol=1e-7, save_every=0.5, linear_correction_type=lin,
                                          output_types=["state", "time", "iteration_counters"]))


def test_mass_matrix_rules():
    from cubie_b200 import Solver, create_ODE_system
    eqs = VDP_MASS["equations"]
    sysm = create_ODE_system(eqs, states={"x": 1.0, "y": 0.0}, parameters={"mu": 1.0}, mass=VDP_MASS["mass"])
    assert sysm.mass is not None and sysm.mass.shape == (2, 2)
    with pytest.raises(ValueError, match="implicit algorithm"):
        Solver(sysm, algorithm="dormand-prince-54")
    with pytest.raises(NotImplementedError):
        Solver(sysm, algorithm="l_stable_dirk_3", layout="warp")
    with pytest.raises(ValueError):
        create_ODE_system(eqs, states={"x": 1.0, "y": 0.0}, parameters={"mu": 1.0}, mass=np.eye(3))
    plain = create_ODE_system(eqs, states={"x": 1.0, "y": 0.0}, parameters={"mu": 1.0}, mass=np.eye(2))
    assert plain.mass is None                              # the identity is no mass matrix
    assert sysm.fn_hash != plain.fn_hash                  # M is part of the system's identity
    src = Solver(sysm, algorithm="radau").prepare(1.0, load=False)["gen"].source
    assert "HAS_MASS = true" in src and "R(0.5)*v[1]" in src


@pytest.mark.parametrize("lin", ["direct", "bicgstab"])
def test_rosenbrock_mass_matrix_emulated_against_oracle(lin):
    """ROS3P with a full M through the generated kernel (g++ host build)
    against the oracle: same statuses and step counts, states within 1e-3
    tolerance units in FP64."""
    from host_emu.emu import run_emulated
    from cubie_b200 import Solver
    case = _ros3p_mass_case(lin)
    kw = dict(case["kwargs"])
    solver = Solver(build_case_system(case), algorithm="ros3p", **kw)
    inits, params = case_inputs(case)
    out = run_emulated(solver, inits, params, case["duration"], kernel="plain")
    orc = run_oracle(case)
    assert out["status"].tolist() == orc["status"].tolist() == [0, 0, 0]
    np.testing.assert_array_equal(out["counters"][:, 2:, :], orc["iteration_counters"][:, 2:, :])
    assert tol_units(out["state"], orc["state"], kw["atol"], kw["rtol"]) < 1e-3


def test_rosenbrock_mass_matrix_oracle_against_explicit_form():
    """ROS3P on M y' = f against SciPy's Radau on y' = M^-1 f at 1e-12: the
    method's own global error (tens of tolerance units at most), where
    leaving M out would miss by the size of the state."""
    from scipy.integrate import solve_ivp
    case = _ros3p_mass_case("direct")
    out = run_oracle(case)
    x0, p = case_inputs(case)
    minv = np.linalg.inv(np.array(VDP_MASS["mass"]))
    assert out["status"].tolist() == [0, 0, 0]
    for r in range(x0.shape[1]):
        mu = p[0, r]
        sol = solve_ivp(lambda t, y: minv @ np.array([y[1], mu * (1 - y[0] ** 2) * y[1] - y[0]]), (0.0, 2.0),
                        x0[:, r], method="Radau", rtol=1e-12, atol=1e-12, t_eval=np.arange(0.0, 2.01, 0.5))
        assert tol_units(out["state"][:, :2, r], sol.y.T, 1e-7, 1e-7) < 100.0


@pytest.mark.gpu
@pytest.mark.parametrize("lin", ["direct", "bicgstab", "gmres"])
def test_rosenbrock_mass_matrix_gpu_against_oracle(cuda_device, lin):
    from cubie_b200 import Solver
    case = _ros3p_mass_case(lin)
    kw = dict(case["kwargs"])
    solver = Solver(build_case_system(case), algorithm="ros3p", kernel="persistent", **kw)
    inits, params = case_inputs(case)
    res = solver.solve(inits, params, duration=case["duration"], nan_error_trajectories=False)
    orc = run_oracle(case, linear_correction_type="direct" if lin == "gmres" else lin)
    assert res.status_codes.tolist() == orc["status"].tolist() == [0, 0, 0]
    assert tol_units(res.state, orc["state"], kw["atol"], kw["rtol"]) < (1.0 if lin == "gmres" else 1e-2)


@pytest.mark.gpu
def test_dae_mixed_precision_matches_fp64_fixture(cuda_device):
    """The Robertson index-1 DAE (M = diag(1, 1, 0)) with l_stable_dirk_3 in
    mixed precision against the reference's FP64 result: statuses and the
    states within 10 tolerance units; the algebraic component keeps the
    conservation law y1 + y2 + y3 = 1.  FP32 stepping resolves about 6e-8
    of an O(1) state, so the mixed solve runs at rtol 1e-5, atol 1e-6 (the
    fixture's atol 1e-8 puts the Newton tolerance, atol / 10, below what
    FP32 can resolve: the Newton iteration then stalls)."""
    from pathlib import Path
    from cubie_b200 import Solver
    case = CASES["rober_dae_dirk3_f64"]
    ref = np.load(Path(__file__).resolve().parent / "golden" / "ref_rober_dae_dirk3_f64.npz")
    kw = dict(case["kwargs"], rtol=1e-5, atol=1e-6)
    sysm = build_case_system(dict(case, precision="float32"))
    res = Solver(sysm, algorithm=case["algorithm"], mixed_precision=True, kernel="persistent", **kw).solve(
        *[a.astype(np.float32) for a in case_inputs(case)], duration=case["duration"], nan_error_trajectories=False)
    assert res.status_codes.tolist() == ref["status"].tolist()
    assert tol_units(res.state[:, :3], ref["state"][:, :3], kw["atol"], kw["rtol"]) < 10
    assert np.max(np.abs(res.state[:, :3].astype(np.float64).sum(axis=1) - 1.0)) < 1e-5
