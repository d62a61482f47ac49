"""Helpers shared by the parity tests."""

import numpy as np

from pathlib import Path

from cases import CASES, case_drivers, case_inputs

GOLDEN = Path(__file__).resolve().parent / "golden"


def build_case_system(case):
    from cubie_b200 import create_ODE_system
    sd = case["system"]
    prec = np.dtype(case["precision"]).type
    return create_ODE_system(sd["equations"], states={s: 0.0 for s in sd["states"]},
                             parameters={p: 0.0 for p in sd["parameters"]}, constants=sd["constants"],
                             drivers=sd.get("drivers"), precision=prec, strict=True, mass=sd.get("mass"))


def oracle_driver_table(case, name):
    """The reference's own coefficient table for a driven case (stored in
    its fixture), as an oracle driver evaluator."""
    from oracle import DriverTable
    ref = np.load(GOLDEN / f"ref_{name}.npz")
    period, t0, _, wrap, padded, _ = ref["driver_meta"]
    return DriverTable(ref["driver_coefficients"], period, t0, bool(wrap), bool(padded),
                       np.dtype(case["precision"]).type)


def run_oracle(case, **overrides):
    from oracle import OracleSystem, integrate
    sd = case["system"]
    osys = OracleSystem(sd["equations"], sd["states"], sd["parameters"], sd["constants"],
                        drivers=sd.get("drivers", ()), mass=sd.get("mass"))
    if sd.get("drivers"):
        name = next(n for n, c in CASES.items() if c is case)
        osys.driver_table = oracle_driver_table(case, name)
    inits, params = case_inputs(case)
    kw = dict(case["kwargs"])
    kw["precision"] = np.dtype(case["precision"]).type
    kw.update(overrides)
    return integrate(osys, case["algorithm"], inits, params, case["duration"], **kw)


def tol_units(a, b, atol, rtol):
    """|a - b| in units of atol + rtol |b| (NaN-safe max)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    return float(np.nanmax(np.abs(a - b) / (atol + rtol * np.abs(b)))) if a.size else 0.0
