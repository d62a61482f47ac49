"""Write the reference's coefficient tableaus to ``ref_tableaus.npz``.

Reads the reference's tableau modules (``generic_erk_tableaus.py``,
``generic_dirk_tableaus.py``, ``generic_firk_tableaus.py``,
``generic_rosenbrockw_tableaus.py`` under
``src/cubie/integrators/algorithms``) and stores, for every alias in their
registries, ``<alias>/<field>`` arrays: ``a`` (square), ``b``, ``c``,
``b_hat`` (when present), ``order``, the dense-prediction ratios and, for
Rosenbrock tableaus, ``C``, ``gamma`` and ``gamma_stages``.  The modules
are evaluated with a minimal stand-in for their base class, so no CUDA
backend is needed.  Needs the reference checkout (default
``/root/reference``); the committed ``.npz`` is what the tests read.

Usage::

    python tests/golden/make_tableau_fixture.py [--reference PATH]
"""

import argparse
import re
from pathlib import Path
from typing import Optional

import attrs
import numpy as np

HERE = Path(__file__).resolve().parent
MODULES = {
    "erk": ("generic_erk_tableaus", "ERK_TABLEAU_REGISTRY"),
    "dirk": ("generic_dirk_tableaus", "DIRK_TABLEAU_REGISTRY"),
    "firk": ("generic_firk_tableaus", "FIRK_TABLEAU_REGISTRY"),
    "rosenbrock": ("generic_rosenbrockw_tableaus", "ROSENBROCK_TABLEAUS"),
}


@attrs.frozen
class _Base:
    """Fields of the reference's ``ButcherTableau`` (base_algorithm_step.py:
    248-257); validation hooks are no-ops."""

    a: tuple = attrs.field()
    b: tuple = attrs.field()
    c: tuple = attrs.field()
    order: int = attrs.field()
    b_hat: Optional[tuple] = attrs.field(default=None)
    dense_prediction_ratio_float16: float = attrs.field(default=0.0)
    dense_prediction_ratio_float32: float = attrs.field(default=0.0)
    dense_prediction_ratio_float64: float = attrs.field(default=0.0)

    def __attrs_post_init__(self):
        pass

    def _validate_weight_sums(self):
        pass

    def _validate_stage_node_consistency(self):
        pass


def _square(rows, s):
    m = np.zeros((s, s))
    for i, row in enumerate(rows):
        m[i, :len(row)] = row
    return m


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    alg = Path(args.reference) / "src/cubie/integrators/algorithms"
    out = {}
    for kind, (mod, reg) in MODULES.items():
        src = (alg / f"{mod}.py").read_text()
        src = re.sub(r"^from cubie[^\n]*\n", "", src, flags=re.M)
        g = {"ButcherTableau": _Base, "int32": np.int32, "__name__": "ref_" + mod}
        exec(compile(src, mod, "exec"), g)
        for alias, tab in g[reg].items():
            s = len(tab.b)
            out[f"{alias}/kind"] = np.array(kind)
            out[f"{alias}/a"] = _square(tab.a, s)
            out[f"{alias}/b"] = np.asarray(tab.b, float)
            out[f"{alias}/c"] = np.asarray(tab.c, float)
            out[f"{alias}/order"] = np.array(int(tab.order))
            out[f"{alias}/dense32"] = np.array(float(tab.dense_prediction_ratio_float32))
            out[f"{alias}/dense64"] = np.array(float(tab.dense_prediction_ratio_float64))
            if tab.b_hat is not None:
                out[f"{alias}/b_hat"] = np.asarray(tab.b_hat, float)
            if kind == "rosenbrock":
                out[f"{alias}/C"] = _square(tab.C, s)
                out[f"{alias}/gamma"] = np.array(float(tab.gamma))
                out[f"{alias}/gamma_stages"] = np.asarray(tab.gamma_stages, float)
    np.savez_compressed(HERE / "ref_tableaus.npz", **out)
    print(len({k.split("/")[0] for k in out}), "aliases written")


if __name__ == "__main__":
    main()
