"""Julia golden gate: the oracle (CPU) and the engine (GPU) against
DifferentialEquations.jl on the reference's Float32 Lorenz ensemble.

Protocol of the reference gate
(tests/integrated_numerical_tests/julia_reference/test_julia_reference.py:70-175,
ne_gate.py:265-285): 1024 runs of Lorenz (sigma 10, beta 8/3, rho from the
vendored float32 grid, initial state (1, 0, 0)) integrated in Float32 over
t in [0, 1], final state only; one solve per algorithm at the pinned fixed
dt (atol 1e-6, rtol 1e-3 for the stage solves) and one at the pinned
adaptive tolerance under Julia-matched controller settings (dt0 0.01, dt_min
1e-6, dt_max 0.5).  Pass: RMS distance to Julia's finals <= 2 x Julia's RMS
error against the FP64 Vern9 golden states.  Pins, Julia finals and the
matched controllers come from ``golden/julia_lorenz_gate.npz``
(``golden/make_julia_fixture.py``).
"""

import json
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden" / "julia_lorenz_gate.npz"
LORENZ = ["dx = sigma * (y - x)", "dy = x * (rho - z) - y", "dz = x * y - beta * z"]
CONSTANTS = {"sigma": 10.0, "beta": 8.0 / 3.0}
MATCH_FRACTION = 2.0

_FIX = np.load(GOLDEN)
META = json.loads(bytes(_FIX["meta_json"]).decode())
GOLDEN_STATES = _FIX["golden_states"].astype(np.float64)
RHO = _FIX["golden_rho"]


def _supported_engine():
    from cubie_b200.tableaus import TABLEAU_REGISTRY
    return TABLEAU_REGISTRY


def _cases(registry, tier):
    out = []
    for alias in sorted(META):
        if alias not in registry:
            continue
        m = META[alias]
        if tier == "fixed" and "fixed_dt" in m:
            out.append(alias)
        if tier == "adaptive" and "adaptive_tol" in m:
            tab = registry[alias]
            adaptive = tab.has_error_estimate if hasattr(tab, "has_error_estimate") else tab.has_err
            if adaptive:
                out.append(alias)
    return out


def settings(alias, tier):
    m = META[alias]
    if tier == "fixed":
        return dict(step_controller="fixed", dt=m["fixed_dt"], atol=1e-6, rtol=1e-3)
    tol = m["adaptive_tol"]
    kw = dict(dt=0.01, dt_min=1e-6, dt_max=0.5, atol=tol, rtol=tol)
    kw.update(m["controller"])
    return kw


def julia_finals(alias, tier):
    return _FIX[f"{tier}__{alias}"].astype(np.float64)


def gate_ratio(finals, alias, tier):
    """(rms distance to Julia) / (Julia's rms error vs golden) (ne_gate.py:265-285)."""
    finals = np.asarray(finals, np.float64)
    jl = julia_finals(alias, tier)
    err_j = float(np.sqrt(np.mean((jl - GOLDEN_STATES) ** 2)))
    rms = float(np.sqrt(np.mean((finals - jl) ** 2)))
    return rms / err_j if np.isfinite(rms) and err_j > 0 else np.inf


def inputs():
    inits = np.tile(np.array([[1.0], [0.0], [0.0]], np.float32), (1, RHO.size))
    params = RHO.astype(np.float32)[None, :]
    return inits, params


def test_fixture_pins_match_reference_protocol():
    """Every pinned Julia point sits inside the gate's convergence window
    (4 x floor <= error < cap, relative to the golden RMS; ne_gate.py:64-82)."""
    scale = float(np.sqrt(np.mean(GOLDEN_STATES ** 2)))
    n = 0
    for alias, m in META.items():
        for tier in ("fixed", "adaptive"):
            key = f"{tier}__{alias}"
            if key not in _FIX.files:
                continue
            err = float(np.sqrt(np.mean((julia_finals(alias, tier) - GOLDEN_STATES) ** 2)))
            assert 4.0 * 4e-6 * scale <= err < 3e-2 * scale, (alias, tier, err)
            n += 1
    assert n >= 30
    assert RHO.dtype == np.float64 and np.all(RHO == RHO.astype(np.float32))


ORACLE_ALIASES = {"dormand-prince-54", "classical-rk4", "l_stable_sdirk_4", "radau_iia_5", "ros3p"}


def _oracle_cases(tier):
    from oracle.ode_oracle import TABLEAUS
    return [a for a in _cases(TABLEAUS, tier) if a in ORACLE_ALIASES]


@pytest.mark.parametrize("tier", ["fixed", "adaptive"])
def test_oracle_passes_julia_gate(tier):
    from oracle import OracleSystem, integrate
    osys = OracleSystem(LORENZ, ["x", "y", "z"], ["rho"], CONSTANTS)
    inits, params = inputs()
    aliases = _oracle_cases(tier)
    assert aliases
    for alias in aliases:
        out = integrate(osys, alias, inits, params, 1.0, precision=np.float32, save_every=1.0,
                        **settings(alias, tier))
        assert np.all(out["status"] == 0), alias
        ratio = gate_ratio(out["state"][-1].T, alias, tier)
        assert ratio <= MATCH_FRACTION, (alias, tier, ratio)


@pytest.mark.gpu
@pytest.mark.parametrize("tier", ["fixed", "adaptive"])
def test_engine_passes_julia_gate(cuda_device, tier):
    from cubie_b200 import Solver, create_ODE_system
    sysm = create_ODE_system(LORENZ, states={"x": 1.0, "y": 0.0, "z": 0.0}, parameters={"rho": 21.0},
                             constants=CONSTANTS, precision=np.float32, strict=True)
    inits, params = inputs()
    aliases = _cases(_supported_engine(), tier)
    assert aliases
    failures = []
    for alias in aliases:
        solver = Solver(sysm, algorithm=alias, output_types=["state"], save_every=1.0, **settings(alias, tier))
        res = solver.solve(inits, params, duration=1.0, blocksize=64)
        ratio = gate_ratio(res.state[-1].T, alias, tier)
        if not (np.all(res.status_codes == 0) and ratio <= MATCH_FRACTION):
            failures.append((alias, ratio, int(np.sum(res.status_codes != 0))))
    assert not failures, failures
