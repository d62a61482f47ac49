"""GPU parity: the CUDA engine against the reference fixtures and the oracle.

Every case in ``tests/golden/cases.py`` runs through ``Solver`` on the GPU
(reference-precision mode, both launch kinds) and is compared with
(a) the reference's own outputs (``ref_<case>.npz``) and (b) the oracle.
Bars: float64 within 1e-2 of the tolerance envelope (atol + rtol |y|) with
identical status words; float32 within 10x the envelope (the agreement the
engine promises against the reference), chaotic Lorenz on its early window.
"""

from pathlib import Path

import numpy as np
import pytest

from cases import CASES, case_drivers, case_inputs
from parity_utils import build_case_system, run_oracle, tol_units

GOLDEN = Path(__file__).resolve().parent / "golden"
pytestmark = pytest.mark.gpu


def _solve(case, kernel="plain", **extra):
    from cubie_b200 import Solver
    system = build_case_system(case)
    inits, params = case_inputs(case)
    kw = dict(case["kwargs"])
    kw.update(case.get("engine", {}))
    kw.update(extra)
    solver = Solver(system, algorithm=case["algorithm"], kernel=kernel, **kw)
    prec = np.dtype(case["precision"]).type
    return solver.solve(inits.astype(prec), params.astype(prec), drivers=case_drivers(case),
                        duration=case["duration"], nan_error_trajectories=False)


def _bars(name):
    case = CASES[name]
    kw = case["kwargs"]
    return case, kw["atol"], kw["rtol"], (1e-2 if case["precision"] == "float64" else 10.0)


@pytest.mark.parametrize("name", list(CASES))
def test_gpu_matches_reference_fixture(cuda_device, name):
    case, atol, rtol, bar = _bars(name)
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    res = _solve(case)
    assert res.status_codes.tolist() == ref["status"].tolist()
    assert res.state.shape == ref["state"].shape
    if name.startswith("lorenz_dp54") and case["precision"] == "float32":
        k = max(2, ref["state"].shape[0] // 5)
        assert tol_units(res.state[:k], ref["state"][:k], 1e-6, 1e-5) < 10
    else:
        assert tol_units(res.state, ref["state"], atol, rtol) < bar
        if "state_summaries" in ref.files:
            assert tol_units(res.state_summaries, ref["state_summaries"], atol, rtol) < bar
    if "iteration_counters" in ref.files and case["precision"] == "float64" and \
            not case.get("counters_rounding_sensitive"):
        np.testing.assert_array_equal(res.iteration_counters[:, 2:, :], ref["iteration_counters"][:, 2:, :])


@pytest.mark.parametrize("name", [n for n, c in CASES.items() if not c.get("slow_oracle")])
def test_gpu_matches_oracle(cuda_device, name):
    case, atol, rtol, bar = _bars(name)
    out = run_oracle(case)
    res = _solve(case)
    assert res.status_codes.tolist() == out["status"].tolist()
    if name.startswith("lorenz_dp54") and case["precision"] == "float32":
        k = max(2, out["state"].shape[0] // 5)
        assert tol_units(res.state[:k], out["state"][:k], 1e-6, 1e-5) < 10
    else:
        assert tol_units(res.state, out["state"], atol, rtol) < bar


@pytest.mark.parametrize("name", ["lorenz_dp54_f64", "vdp_ros3p_f32", "vdp_radau_f64", "vdp_dirk3_bicgstab_f32"])
def test_persistent_kernel_equals_plain(cuda_device, name):
    case = CASES[name]
    a = _solve(case, kernel="plain")
    b = _solve(case, kernel="persistent")
    np.testing.assert_array_equal(a.status_codes, b.status_codes)
    np.testing.assert_array_equal(a.state, b.state)


@pytest.mark.parametrize("name", ["lorenz_dp54_f64", "vdp_ros3p_bicgstab_f64", "vdp_radau_f64"])
def test_mixed_precision_error_matches_float64(cuda_device, name):
    """FP32 stepping with FP64 time/control/norms and a compensated state
    update reaches the error of an all-FP64 solve at the same tolerance:
    both are measured against a tight FP64 oracle solution (rtol 1e-12)."""
    case = dict(CASES[name])
    kw = dict(case["kwargs"])
    kw["rtol"] = 1e-6
    kw["atol"] = 1e-6
    case["kwargs"] = kw
    truth_case = dict(case, kwargs=dict(kw, rtol=1e-12, atol=1e-12))
    truth_algo = "dormand-prince-54" if case["algorithm"] == "dormand-prince-54" else "radau"
    truth_case["algorithm"] = truth_algo
    truth = run_oracle(truth_case, linear_correction_type="minimal_residual")["state"][:, :-1]
    f64 = _solve(dict(case, precision="float64"))
    mixed = _solve(dict(case, precision="float32"), mixed_precision=True)
    assert np.all(mixed.status_codes == 0) and np.all(f64.status_codes == 0)
    k = max(2, truth.shape[0] // 5) if name.startswith("lorenz") else truth.shape[0]
    err64 = tol_units(f64.state[:k, :-1], truth[:k], 1e-6, 1e-6)
    errmx = tol_units(mixed.state[:k, :-1], truth[:k], 1e-6, 1e-6)
    assert errmx <= max(2.0 * err64, 1.0), (errmx, err64)


DIRECT_CASES = ["vdp_ros3p_f32", "vdp_ros3p_bicgstab_f64", "vdp_rodas3p_f64", "vdp_radau_f64", "vdp_sdirk4_f64",
                "vdp_kvaerno3_f64", "vdp_gl4_f64", "driven_ros3p_clamped_f64"]


@pytest.mark.parametrize("name", DIRECT_CASES)
def test_direct_solver_matches_oracle(cuda_device, name):
    """``linear_correction_type='direct'`` (register LU) against the oracle's
    exact dense solve: same status words and step/rejection counts in
    float64, trajectories within the usual bars."""
    case, atol, rtol, bar = _bars(name)
    out = run_oracle(case, linear_correction_type="direct")
    res = _solve(case, kernel="persistent", linear_correction_type="direct",
                 output_types=["state", "time", "iteration_counters"])
    assert res.status_codes.tolist() == out["status"].tolist()
    assert tol_units(res.state, out["state"], atol, rtol) < bar
    if case["precision"] == "float64":
        np.testing.assert_array_equal(res.iteration_counters[:, 2:, :], out["iteration_counters"][:, 2:, :])
