"""Time the reference's own CPU path on a sample of the headline workload.

The reference's kernels (ccam80/cubie, unmodified) run on the host under
Numba's CUDA simulator through the import shim in ``refsim/``, one process
per run and per core, on the first ``--runs`` seeded draws of the stiff Van
der Pol workload the bench measures (seed 2: mu = 10^U[0,3],
(x0, y0) ~ U[-2,2]^2, t in [0, 2 mu], rtol = atol = 1e-6, ROS3P with the
reference's defaults in FP32; its outputs include the iteration counters,
without which the reference's FP32 ROS3P stops at once with
STEP_TOO_SMALL).  A run that does not finish within
``--timeout`` seconds counts as unsolved.  Solved: status 0 and the final
state within 10 tolerance units of SciPy's Radau at 1e-10.  Needs the
reference checkout (default ``/root/reference``), so it runs where the
reference is; it writes ``ref_simulator_timing.json`` beside itself.

Usage::

    python tests/golden/time_reference_simulator.py [--runs 8] [--timeout 900]
"""

import argparse
import json
import os
import subprocess
import sys
import time
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

WORKER = r"""
import json, sys, time
import numpy as np
from cubie import create_ODE_system, Solver
x0, y0, mu = {x0!r}, {y0!r}, {mu!r}
system = create_ODE_system(dxdt=["dx = y", "dy = mu * (1 - x**2) * y - x"], states={{"x": 0.0, "y": 0.0}},
                           parameters={{"mu": 0.0}}, precision=np.float32, name="timing", strict=True)
# the reference's FP32 ROS3P returns STEP_TOO_SMALL at once unless the
# iteration counters are among its outputs (an aliasing of its per-thread
# buffers); with them, and rows every mu, it integrates the run
solver = Solver(system, algorithm="ros3p", cache=False, auto_memory=False, rtol=1e-6, atol=1e-6,
                output_types=["state", "time", "iteration_counters"], save_every=float(mu))
t = time.time()
res = solver.solve(np.array([[x0], [y0]], np.float32), np.array([[mu]], np.float32), duration=2.0 * mu,
                   grid_type="verbatim", nan_error_trajectories=False)
print(json.dumps(dict(elapsed=time.time() - t, status=int(np.asarray(res.status_codes)[0]),
                      y=[float(v) for v in np.asarray(res.state)[-1, :2, 0]])))
"""


def truth(x0, y0, mu):
    from scipy.integrate import solve_ivp
    s = solve_ivp(lambda t, y: [y[1], mu * (1 - y[0] ** 2) * y[1] - y[0]], (0.0, 2.0 * mu), [x0, y0],
                  method="Radau", rtol=1e-10, atol=1e-10,
                  jac=lambda t, y: [[0.0, 1.0], [-2.0 * mu * y[0] * y[1] - 1.0, mu * (1.0 - y[0] ** 2)]])
    return s.y[:, -1]


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    ap.add_argument("--runs", type=int, default=8)
    ap.add_argument("--timeout", type=float, default=900.0)
    args = ap.parse_args()
    rng = np.random.default_rng(2)
    n = args.runs
    mu = 10.0 ** rng.uniform(0.0, 3.0, n)
    x0 = rng.uniform(-2.0, 2.0, (2, n))
    env = dict(os.environ, NUMBA_ENABLE_CUDASIM="1",
               PYTHONPATH=os.pathsep.join([str(HERE / "refsim"), str(Path(args.reference) / "src")]))

    def one(i):
        code = WORKER.format(x0=float(np.float32(x0[0, i])), y0=float(np.float32(x0[1, i])),
                             mu=float(np.float32(mu[i])))
        t = time.time()
        try:
            p = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True,
                               timeout=args.timeout, cwd="/tmp")
            out = json.loads(p.stdout.strip().splitlines()[-1])
        except (subprocess.TimeoutExpired, ValueError, IndexError):
            out = dict(elapsed=None, status=None, y=None)
        out["wall"] = time.time() - t
        return out

    cores = os.cpu_count() or 1
    t0 = time.time()
    with ThreadPoolExecutor(cores) as ex:
        res = list(ex.map(one, range(n)))
    wall = time.time() - t0
    solved = 0
    for i, r in enumerate(res):
        r["mu"] = float(mu[i])
        if r["status"] == 0 and r["y"] is not None:
            tr = truth(float(x0[0, i]), float(x0[1, i]), float(mu[i]))
            err = np.max(np.abs(np.array(r["y"]) - tr) / (1e-6 + 1e-6 * np.abs(tr)))
            r["error_tol_units"] = float(err)
            solved += int(err <= 10.0)
    cpu_s = sum(r["wall"] for r in res)
    rec = dict(runs=n, cores=cores, wall_s=wall, cpu_s=cpu_s, solved=solved, timeout_s=args.timeout,
               value=solved / wall, unit="systems/s",
               sample=(f"first {n} seeded runs of the stiff Van der Pol workload (seed 2), the reference's own "
                       f"ROS3P kernels with their defaults (FP32, minimal residual + Neumann order 2) under Numba's "
                       f"CUDA simulator, one process per run on {cores} host cores, {args.timeout:.0f} s limit per "
                       f"run (unfinished runs count as unsolved)"),
               per_run=res)
    (HERE / "ref_simulator_timing.json").write_text(json.dumps(rec, indent=1))
    print(json.dumps({k: rec[k] for k in ("runs", "cores", "wall_s", "solved", "value")}))


if __name__ == "__main__":
    main()
