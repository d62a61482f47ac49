"""Coefficient fixtures from the reference's ``ArrayInterpolator``.

Runs the unmodified reference (``src/cubie/array_interpolator.py``) in a
subprocess with the import shim in ``refsim/`` and Numba's CUDA simulator,
builds interpolators for seeded sample arrays over every boundary condition
and a range of orders, and stores their coefficient tables and the values
the reference's ``get_interpolated`` returns at seeded query times in
``ref_interpolator.npz``.  Needs the reference checkout (default
``/root/reference``); the committed fixture is what the tests read.

Usage::

    python tests/golden/make_interpolator_fixture.py [--reference PATH]
"""

import argparse
import os
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

CONFIGS = [
    # name, order, wrap, boundary_condition, n_samples, n_inputs, precision
    ("cubic_clamped_f32", 3, False, "clamped", 12, 2, "float32"),
    ("cubic_clamped_f64", 3, False, "clamped", 12, 2, "float64"),
    ("cubic_periodic_f64", 3, True, "periodic", 10, 1, "float64"),
    ("cubic_natural_f64", 3, False, "natural", 9, 2, "float64"),
    ("cubic_notaknot_f64", 3, False, "not-a-knot", 11, 1, "float64"),
    ("quadratic_clamped_f64", 2, False, "clamped", 8, 1, "float64"),
    ("quintic_natural_f64", 5, False, "natural", 14, 1, "float64"),
    ("linear_clamped_f32", 1, False, "clamped", 6, 1, "float32"),
]

WORKER = r"""
import sys
import numpy as np
from cubie.array_interpolator import ArrayInterpolator
configs = {configs!r}
out = {{}}
for name, order, wrap, bc, ns, ni, prec in configs:
    rng = np.random.default_rng(len(name) * 7919 + ns)
    p = np.dtype(prec).type
    samples = rng.uniform(-1.0, 1.0, (ns, ni))
    if bc == "periodic":
        samples[-1] = samples[0]
    d = {{"driver_sample_period": 0.25, "t0": 0.5, "order": order, "wrap": wrap, "boundary_condition": bc}}
    for k in range(ni):
        d["d%d" % k] = samples[:, k]
    interp = ArrayInterpolator(p, d)
    q = np.sort(rng.uniform(0.0, 0.5 + 0.25 * (ns + 2), 40))
    vals = np.asarray(interp.get_interpolated(q.astype(p)))
    out[name + "__samples"] = samples
    out[name + "__coefficients"] = np.asarray(interp.coefficients)
    out[name + "__query"] = q
    out[name + "__values"] = vals
np.savez_compressed({outfile!r}, **out)
print("ok", len(configs))
"""


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    env = dict(os.environ)
    env["NUMBA_ENABLE_CUDASIM"] = "1"
    env["PYTHONPATH"] = os.pathsep.join([str(HERE / "refsim"), str(Path(args.reference) / "src")])
    outfile = str(HERE / "ref_interpolator.npz")
    code = WORKER.format(configs=CONFIGS, outfile=outfile)
    proc = subprocess.run([sys.executable, "-c", code], env=env, capture_output=True, text=True, cwd="/tmp")
    print(proc.stdout.strip()[-500:], proc.stderr.strip()[-2000:])
    sys.exit(proc.returncode)


if __name__ == "__main__":
    main()
