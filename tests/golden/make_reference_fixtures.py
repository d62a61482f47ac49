"""Generate parity fixtures from the reference's own integrator (CPU).

Runs every case in ``cases.py`` through the unmodified reference package
(``ccam80/cubie``) under Numba's CUDA simulator, which executes the
reference's Numba device functions on the host, and stores the outputs as
``tests/golden/ref_<case>.npz``.  Needs the reference checkout (default
``/root/reference``) and only runs where it exists; the committed fixtures
are what the tests read.

Usage::

    python tests/golden/make_reference_fixtures.py [--reference PATH] [case ...]

Each case runs in a fresh subprocess with ``NUMBA_ENABLE_CUDASIM=1`` and the
import shim in ``refsim/`` on ``PYTHONPATH``.  ``auto_memory=False`` keeps
every reference buffer in per-thread local memory (its default placement),
so buffer aliasing that only occurs in shared memory plays no part.
"""

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent

WORKER = r"""
import json, sys, time
import numpy as np
sys.path.insert(0, {here!r})
from cases import CASES, case_inputs, case_drivers
from cubie import create_ODE_system, Solver
name = {name!r}
case = CASES[name]
sysd = case["system"]
prec = np.dtype(case["precision"]).type
drivers = case_drivers(case)
system = create_ODE_system(dxdt=sysd["equations"], states={{s: 0.0 for s in sysd["states"]}},
                           parameters={{p: 0.0 for p in sysd["parameters"]}}, constants=sysd["constants"],
                           drivers=sysd.get("drivers"), precision=prec, name="fixture_" + name, strict=True,
                           **({{"mass": np.asarray(sysd["mass"], dtype=prec)}} if sysd.get("mass") is not None else {{}}))
inits, params = case_inputs(case)
solver = Solver(system, algorithm=case["algorithm"], cache=False, auto_memory=False, **case["kwargs"])
t = time.time()
res = solver.solve(inits.astype(prec), params.astype(prec), drivers=drivers, duration=case["duration"],
                   grid_type="verbatim", nan_error_trajectories=False)
elapsed = time.time() - t
out = dict(inits=inits, params=params, status=np.asarray(res.status_codes), elapsed=elapsed)
if res.state is not None:
    out["state"] = np.asarray(res.state)
if res.iteration_counters is not None:
    out["iteration_counters"] = np.asarray(res.iteration_counters)
if res.state_summaries is not None:
    out["state_summaries"] = np.asarray(res.state_summaries)
out["summaries_legend"] = np.array(json.dumps({{str(k): v for k, v in res.summaries_legend.items()}}))
if drivers is not None:
    from cubie.array_interpolator import ArrayInterpolator
    interp = ArrayInterpolator(prec, dict(drivers))
    out["driver_coefficients"] = np.asarray(interp.coefficients)
    out["driver_meta"] = np.array([interp.driver_sample_period, interp.t0, interp.num_segments,
                                   float(interp.wrap), float(interp.boundary_condition == "clamped"),
                                   float(interp.order)])
np.savez_compressed({outfile!r}, **out)
print(name, "ok", round(elapsed, 2), "s; status", out["status"].tolist())
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("cases", nargs="*")
    args = ap.parse_args()
    sys.path.insert(0, str(HERE))
    from cases import CASES
    names = args.cases or list(CASES)
    env = dict(os.environ)
    env["NUMBA_ENABLE_CUDASIM"] = "1"
    env["PYTHONPATH"] = os.pathsep.join([str(HERE / "refsim"), str(Path(args.reference) / "src")])
    for name in names:
        outfile = str(HERE / f"ref_{name}.npz")
        code = WORKER.format(here=str(HERE), name=name, outfile=outfile)
        t = time.time()
        proc = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                              cwd="/tmp")
        tail = (proc.stdout + proc.stderr).strip().splitlines()[-3:]
        print(f"{name}: rc={proc.returncode} wall={time.time() - t:.1f}s :: " + " | ".join(tail))


if __name__ == "__main__":
    main()
