"""Extract the reference's Julia golden-gate data into a small fixture.

The reference vendors DifferentialEquations.jl results for a Float32 Lorenz
ensemble (1024 runs, rho on a float32-rounded grid in [0, 21], initial
state (1, 0, 0), sigma = 10, beta = 8/3, t in [0, 1]) together with an
FP64 Vern9 (tol 1e-13) golden final state per run
(tests/integrated_numerical_tests/julia_reference/data/README.md).  Its
gate (tests/integrated_numerical_tests/julia_reference/ne_gate.py:205-262)
picks, per algorithm, one "pinned" dt (fixed-step tier) and one pinned
tolerance (adaptive tier) at the difficult end of the Julia convergence
region, then requires the ensemble RMS distance between the solver's
final states and Julia's to be at most 2x Julia's own RMS error against
the golden states (ne_gate.py:265-285).

This script evaluates that pin selection once and stores, for every
algorithm alias the data covers, the pinned dt / tolerance with Julia's
final states there, the Julia-matched controller settings
(ne_gate.py:126-178) and the golden ensemble.  Output:
``julia_lorenz_gate.npz`` beside this file.  Run from the repo root:

    python tests/golden/make_julia_fixture.py
"""

import csv
import json
from pathlib import Path

import numpy as np

DATA = Path("/root/reference/tests/integrated_numerical_tests/julia_reference/data")
OUT = Path(__file__).resolve().parent / "julia_lorenz_gate.npz"

# Protocol constants of the gate (ne_gate.py:37-82).
DTS = [2.0 ** -k for k in range(1, 14)]
TOLS = [10.0 ** -k for k in range(2, 7)]
FLOOR_REL = 4e-6
PIN_CAP_REL = 3e-2
PIN_MARGIN_MULT = 4.0


def ensemble_error(finals, golden):
    d = np.asarray(finals, np.float64) - golden
    return float(np.sqrt(np.mean(d * d)))


def pin_fixed(dts, finals, golden, scale):
    """Finest dt of the first contiguous in-region run (ne_gate.py:205-234)."""
    lo, hi = PIN_MARGIN_MULT * FLOOR_REL * scale, PIN_CAP_REL * scale
    errs = {float(dt): ensemble_error(finals[i], golden) for i, dt in enumerate(dts)}
    pin = None
    for dt in DTS:
        e = errs.get(dt)
        if e is not None and np.isfinite(e) and lo <= e < hi:
            pin = dt
        elif pin is not None:
            break
    return pin


def pin_adaptive(tols, finals, golden, scale):
    """Tightest in-region tolerance (ne_gate.py:237-262)."""
    lo, hi = PIN_MARGIN_MULT * FLOOR_REL * scale, PIN_CAP_REL * scale
    errs = {float(t): ensemble_error(finals[i], golden) for i, t in enumerate(tols)}
    ok = [t for t in TOLS if t in errs and np.isfinite(errs[t]) and lo <= errs[t] < hi]
    return min(ok) if ok else None


def matched_controller(row, order):
    """Solver kwargs mirroring Julia's resolved controller (ne_gate.py:126-178)."""
    f = {k: (float(row[k]) if row.get(k) not in ("", None) else None)
         for k in ("beta1", "beta2", "qmin", "qmax", "gamma", "qsteady_min", "qsteady_max")}
    if row["controller"] == "PIController":
        return {"step_controller": "pi", "kp": f["beta1"] * (order + 1), "ki": -f["beta2"] * (order + 1),
                "safety": f["gamma"], "min_gain": f["qmin"], "max_gain": f["qmax"],
                "deadband_min": 1.0 / f["qsteady_max"], "deadband_max": 1.0 / f["qsteady_min"]}
    if row["controller"] == "PredictiveController":
        return {"step_controller": "gustafsson", "safety": f["gamma"]}
    return None


def main():
    ref = np.load(DATA / "julia_reference_ne.npz")
    with open(DATA / "algorithms.csv", newline="") as fh:
        algos = {r["cubie_alias"]: r for r in csv.DictReader(fh)}
    with open(DATA / "controller_constants.csv", newline="") as fh:
        ctrl = {r["cubie_alias"]: r for r in csv.DictReader(fh)}
    golden = ref["golden_states"].astype(np.float64)
    scale = float(np.sqrt(np.mean(golden ** 2)))
    out = {"golden_rho": ref["golden_rho"], "golden_states": golden}
    meta = {}
    for alias, row in algos.items():
        order = int(row["order"])
        entry = {"order": order, "family": row["family"]}
        fk = f"fixed_{alias}_dts"
        if fk in ref.files:
            pin = pin_fixed(ref[fk], ref[f"fixed_{alias}_finals"], golden, scale)
            if pin is not None:
                i = [float(d) for d in ref[fk]].index(pin)
                entry["fixed_dt"] = pin
                out[f"fixed__{alias}"] = ref[f"fixed_{alias}_finals"][i].astype(np.float32)
        ak = f"adaptive_{alias}_tols"
        if ak in ref.files and alias in ctrl:
            pin = pin_adaptive(ref[ak], ref[f"adaptive_{alias}_finals"], golden, scale)
            settings = matched_controller(ctrl[alias], order)
            if pin is not None and settings is not None:
                i = [float(t) for t in ref[ak]].index(pin)
                entry["adaptive_tol"] = pin
                entry["controller"] = settings
                out[f"adaptive__{alias}"] = ref[f"adaptive_{alias}_finals"][i].astype(np.float32)
        meta[alias] = entry
    out["meta_json"] = np.frombuffer(json.dumps(meta, sort_keys=True).encode(), dtype=np.uint8)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({OUT.stat().st_size} bytes, {len(meta)} aliases)")


if __name__ == "__main__":
    main()
