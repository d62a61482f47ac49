"""Butcher and Rosenbrock tableaus and the algorithm-name registry.

The coefficient tables are the published ones; the same tables (and the
same alias names) appear in the reference's
``generic_erk_tableaus.py:99`` (Dormand--Prince 5(4)),
``generic_rosenbrockw_tableaus.py:86-132`` (ROS3P),
``generic_firk_tableaus.py:131-150`` (Radau IIA 5),
``generic_dirk_tableaus.py:329-362`` (L-stable DIRK3) and their registries.
Derived facts (first-same-as-last, rows of ``a`` equal to ``b``/``b_hat``,
embedded error weights, dense stage prediction polynomials) follow the
reference's definitions in ``base_algorithm_step.py:300-580`` and
``stage_predictors.py:76-300``.
"""

from __future__ import annotations

from dataclasses import dataclass, field
from math import atan, cos, sin, sqrt
from typing import Dict, Optional, Tuple

import numpy as np

ERK, DIRK, FIRK, ROSENBROCK = "erk", "dirk", "firk", "rosenbrock"


@dataclass(frozen=True)
class Tableau:
    kind: str
    a: Tuple[Tuple[float, ...], ...]
    b: Tuple[float, ...]
    c: Tuple[float, ...]
    order: int
    b_hat: Optional[Tuple[float, ...]] = None
    C: Optional[Tuple[Tuple[float, ...], ...]] = None       # Rosenbrock
    gamma: float = 0.0                                       # Rosenbrock
    gamma_stages: Optional[Tuple[float, ...]] = None         # Rosenbrock
    dense_ratio_float32: float = 0.0
    dense_ratio_float64: float = 0.0
    name: str = ""

    # -- basic structure ----------------------------------------------
    @property
    def stage_count(self) -> int:
        return len(self.b)

    def a_matrix(self) -> np.ndarray:
        s = self.stage_count
        m = np.zeros((s, s))
        for i, row in enumerate(self.a):
            m[i, : len(row)] = row
        return m

    @property
    def d(self) -> Optional[Tuple[float, ...]]:
        """Embedded error weights b - b_hat."""
        if self.b_hat is None:
            return None
        return tuple(x - y for x, y in zip(self.b, self.b_hat))

    @property
    def has_error_estimate(self) -> bool:
        d = self.d
        return d is not None and any(w != 0.0 for w in d)

    def _matching_row(self, target) -> Optional[int]:
        if target is None:
            return None
        a = self.a_matrix()
        match = None
        for r in range(self.stage_count):
            if all(abs(a[r, k] - target[k]) <= 1e-15 for k in range(self.stage_count)):
                match = r
        return match

    @property
    def b_row(self) -> Optional[int]:
        return self._matching_row(self.b)

    @property
    def b_hat_row(self) -> Optional[int]:
        return self._matching_row(self.b_hat)

    @property
    def accumulates_output(self) -> bool:
        return self.b_row is None

    @property
    def accumulates_error(self) -> bool:
        return self.b_hat_row is None

    @property
    def first_stage_explicit(self) -> bool:
        return self.a_matrix()[0, 0] == 0.0

    @property
    def first_same_as_last(self) -> bool:
        a = self.a_matrix()
        return bool(self.c and self.c[0] == 0.0 and self.c[-1] == 1.0
                    and np.allclose(a[-1], self.b, atol=0.0, rtol=0.0)
                    and not np.any(a[0]))

    # -- dense stage prediction (stage_predictors.py:76-300) -------------
    @property
    def prediction_sample_stages(self) -> Tuple[int, ...]:
        last = {}
        for stage, node in enumerate(self.c):
            last[node] = stage
        return tuple(last.values())

    @property
    def prediction_source_stages(self) -> Tuple[int, ...]:
        latest = {}
        out = []
        for stage, node in enumerate(self.c):
            out.append(latest.get(node, stage))
            latest[node] = stage
        return tuple(out)

    def _predictor_matrix(self, nodes, ratio, samples) -> np.ndarray:
        s = len(nodes)
        distinct = np.asarray([nodes[i] for i in samples])
        mat = np.zeros((s, s))
        for ti, tn in enumerate(1.0 + ratio * np.asarray(nodes)):
            for bi, bn in enumerate(distinct):
                w = ratio
                for oi, on in enumerate(distinct):
                    if oi != bi:
                        w *= (tn - on) / (bn - on)
                mat[ti, samples[bi]] = w
        return mat

    def supports_dense_prediction(self) -> bool:
        """The read-ahead may amplify sample error at most 10x relative to
        Gauss-Legendre nodes of the same count (stage_predictors.py:76-90)."""
        nodes = np.asarray(self.c, dtype=float)
        samples = self.prediction_sample_stages
        amp = float(np.abs(self._predictor_matrix(nodes, 1.0, samples)).sum(axis=1).max())
        k = len(samples)
        g = 0.5 * (np.polynomial.legendre.leggauss(k)[0] + 1.0)
        ref = float(np.abs(self._predictor_matrix(g, 1.0, tuple(range(k)))).sum(axis=1).max())
        return amp <= 10.0 * ref

    def dense_ratio_limit(self, precision) -> float:
        return self.dense_ratio_float32 if np.dtype(precision) == np.float32 else self.dense_ratio_float64

    def dense_prediction(self, precision) -> bool:
        return self.dense_ratio_limit(precision) > 0.0 and self.supports_dense_prediction()

    def prediction_coefficients(self) -> np.ndarray:
        """Array [power, target, source]: coefficient of ratio**(power+1)."""
        nodes = np.asarray(self.c, dtype=float)
        s = self.stage_count
        samples = self.prediction_sample_stages
        distinct = [nodes[i] for i in samples]
        k = len(distinct)
        P = np.polynomial.polynomial
        shifted = []
        for bi in range(k):
            others = [distinct[j] for j in range(k) if j != bi]
            coef = P.polyfromroots(others) if others else np.array([1.0])
            coef = coef / P.polyval(distinct[bi], coef)
            poly = np.polynomial.Polynomial(coef)(np.polynomial.Polynomial([1.0, 1.0]))
            cf = np.zeros(k)
            cf[: len(poly.coef)] = poly.coef
            shifted.append(cf)
        out = np.zeros((k, s, s))
        for p in range(k):
            for t in range(s):
                for bi in range(k):
                    out[p, t, samples[bi]] = shifted[bi][p] * nodes[t] ** p
        return out


# ---------------------------------------------------------------------------
# Explicit Runge--Kutta
# ---------------------------------------------------------------------------
DORMAND_PRINCE_54 = Tableau(
    kind=ERK, name="dormand-prince-54", order=5,
    a=((0, 0, 0, 0, 0, 0, 0),
       (1 / 5, 0, 0, 0, 0, 0, 0),
       (3 / 40, 9 / 40, 0, 0, 0, 0, 0),
       (44 / 45, -56 / 15, 32 / 9, 0, 0, 0, 0),
       (19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729, 0, 0, 0),
       (9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656, 0, 0),
       (35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0)),
    b=(35 / 384, 0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0),
    b_hat=(5179 / 57600, 0, 7571 / 16695, 393 / 640, -92097 / 339200, 187 / 2100, 1 / 40),
    c=(0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1, 1),
)

CLASSICAL_RK4 = Tableau(
    kind=ERK, name="classical-rk4", order=4,
    a=((0, 0, 0, 0), (0.5, 0, 0, 0), (0, 0.5, 0, 0), (0, 0, 1, 0)),
    b=(1 / 6, 1 / 3, 1 / 3, 1 / 6), c=(0, 0.5, 0.5, 1),
)

HEUN_21 = Tableau(kind=ERK, name="heun-21", order=2, a=((0, 0), (1, 0)), b=(0.5, 0.5), c=(0, 1))

BOGACKI_SHAMPINE_32 = Tableau(
    kind=ERK, name="bogacki-shampine-32", order=3,
    a=((0, 0, 0, 0), (0.5, 0, 0, 0), (0, 0.75, 0, 0), (2 / 9, 1 / 3, 4 / 9, 0)),
    b=(2 / 9, 1 / 3, 4 / 9, 0), b_hat=(7 / 24, 1 / 4, 1 / 3, 1 / 8), c=(0, 0.5, 0.75, 1),
)

# ---------------------------------------------------------------------------
# Rosenbrock-W: ROS3P (Rang & Angermann 2005)
# ---------------------------------------------------------------------------
def _ros3p() -> Tableau:
    g = 0.5 + sqrt(3.0) / 6.0
    ig = 1.0 / g
    b_aux = ig * (2.0 / 3.0 - ig / 6.0)
    return Tableau(
        kind=ROSENBROCK, name="ros3p", order=3,
        a=((0, 0, 0), (ig, 0, 0), (ig, 0, 0)),
        C=((0, 0, 0),
           (-(ig ** 2), 0, 0),
           (-ig * (1.0 + ig * (2.0 - 0.5 * ig)), -ig * (2.0 - 0.5 * ig), 0)),
        b=(ig * (1.0 + b_aux), b_aux, ig / 3.0),
        b_hat=(2.113248654051871, 1.0, 0.4226497308103742),
        c=(0, 1, 1), gamma=g,
        gamma_stages=(g, -0.2113248654051871, 0.5 - 2.0 * g),
    )


ROS3P = _ros3p()

# ---------------------------------------------------------------------------
# Fully implicit: Radau IIA (order 5) and Gauss--Legendre (order 4)
# ---------------------------------------------------------------------------
def _radau_embedded_weights(c, order):
    """Least-squares weights with sum_i w_i c_i^(k-1) = 1/k, k = 1..order."""
    c = np.asarray(c)
    M = np.vander(c, N=order, increasing=True).T
    r = np.array([1.0 / k for k in range(1, order + 1)])
    if order == len(c):
        return np.linalg.solve(M, r)
    return np.linalg.lstsq(M, r, rcond=None)[0]


_S6 = sqrt(6.0)
_RADAU_C = ((4 - _S6) / 10.0, (4 + _S6) / 10.0, 1.0)
RADAU_IIA_5 = Tableau(
    kind=FIRK, name="radau_iia_5", order=5,
    a=(((88 - 7 * _S6) / 360.0, (296 - 169 * _S6) / 1800.0, (-2 + 3 * _S6) / 225.0),
       ((296 + 169 * _S6) / 1800.0, (88 + 7 * _S6) / 360.0, (-2 - 3 * _S6) / 225.0),
       ((16 - _S6) / 36.0, (16 + _S6) / 36.0, 1.0 / 9.0)),
    b=((16 - _S6) / 36.0, (16 + _S6) / 36.0, 1.0 / 9.0),
    b_hat=tuple(_radau_embedded_weights(_RADAU_C, 2).tolist()),
    c=_RADAU_C, dense_ratio_float32=8.0, dense_ratio_float64=8.0,
)

_S3 = sqrt(3.0)
GAUSS_LEGENDRE_2 = Tableau(
    kind=FIRK, name="firk_gauss_legendre_2", order=4,
    a=((0.25, 0.25 - _S3 / 6.0), (0.25 + _S3 / 6.0, 0.25)),
    b=(0.5, 0.5), c=(0.5 - _S3 / 6.0, 0.5 + _S3 / 6.0),
    dense_ratio_float32=8.0, dense_ratio_float64=8.0,
)

# ---------------------------------------------------------------------------
# Diagonally implicit
# ---------------------------------------------------------------------------
_S2 = sqrt(2.0)
_ARC = atan(_S2 / 4.0) / 3.0
_LG = -_S2 * cos(_ARC) / 2.0 + _S6 * sin(_ARC) / 2.0 + 1.0
_LB1 = (-6.0 * _LG ** 2 + 16.0 * _LG - 1.0) / 4.0
_LB2 = (6.0 * _LG ** 2 - 20.0 * _LG + 5.0) / 4.0
L_STABLE_DIRK3 = Tableau(
    kind=DIRK, name="l_stable_dirk_3", order=3,
    a=((_LG, 0, 0), ((1.0 - _LG) / 2.0, _LG, 0), (_LB1, _LB2, _LG)),
    b=(_LB1, _LB2, _LG), c=(_LG, (1.0 + _LG) / 2.0, 1.0),
    dense_ratio_float32=0.85, dense_ratio_float64=1.07,
)

L_STABLE_SDIRK4 = Tableau(
    kind=DIRK, name="l_stable_sdirk_4", order=4,
    a=((0.25, 0, 0, 0, 0),
       (0.5, 0.25, 0, 0, 0),
       (17 / 50, -1 / 25, 0.25, 0, 0),
       (371 / 1360, -137 / 2720, 15 / 544, 0.25, 0),
       (25 / 24, -49 / 48, 125 / 16, -85 / 12, 0.25)),
    b=(25 / 24, -49 / 48, 125 / 16, -85 / 12, 0.25),
    b_hat=(59 / 48, -17 / 96, 225 / 32, -85 / 12, 0.0),
    c=(0.25, 0.75, 11 / 20, 0.5, 1.0),
    dense_ratio_float32=0.79, dense_ratio_float64=0.79,
)

IMPLICIT_MIDPOINT = Tableau(kind=DIRK, name="implicit_midpoint", order=2, a=((0.5,),), b=(1.0,), c=(0.5,),
                            dense_ratio_float32=1.0, dense_ratio_float64=1.0)

# ---------------------------------------------------------------------------
# Registry (algorithms/__init__.py:55-85 and the four tableau registries)
# ---------------------------------------------------------------------------
TABLEAU_REGISTRY: Dict[str, Tableau] = {
    "heun-21": HEUN_21,
    "bogacki-shampine-32": BOGACKI_SHAMPINE_32, "rk23": BOGACKI_SHAMPINE_32, "ode23": BOGACKI_SHAMPINE_32,
    "dormand-prince-54": DORMAND_PRINCE_54, "dopri54": DORMAND_PRINCE_54,
    "rk45": DORMAND_PRINCE_54, "ode45": DORMAND_PRINCE_54,
    "classical-rk4": CLASSICAL_RK4, "rk4": CLASSICAL_RK4,
    "ros3p": ROS3P,
    "radau_iia_5": RADAU_IIA_5, "radau": RADAU_IIA_5,
    "firk_gauss_legendre_2": GAUSS_LEGENDRE_2,
    "l_stable_dirk_3": L_STABLE_DIRK3, "l_stable_sdirk_4": L_STABLE_SDIRK4,
    "implicit_midpoint": IMPLICIT_MIDPOINT,
}

FAMILY_DEFAULTS: Dict[str, Tableau] = {
    "erk": DORMAND_PRINCE_54,
    "dirk": L_STABLE_DIRK3,
    "firk": GAUSS_LEGENDRE_2,
    "rosenbrock": ROS3P,
}


def resolve_algorithm(name) -> Tableau:
    """Return the tableau for an algorithm alias or family name."""
    if isinstance(name, Tableau):
        return name
    key = str(name).lower()
    if key in TABLEAU_REGISTRY:
        return TABLEAU_REGISTRY[key]
    if key in FAMILY_DEFAULTS:
        return FAMILY_DEFAULTS[key]
    raise ValueError(f"Unknown algorithm '{name}'.")


# Per-family controller defaults (generic_erk.py:77-88,
# generic_rosenbrock_w.py:71-79, generic_firk.py:71-80, generic_dirk.py:69-78).
ADAPTIVE_DEFAULTS = {
    ERK: dict(step_controller="pi", kp=0.7, ki=-0.4, deadband_min=1.0, deadband_max=1.0,
              min_gain=0.2, max_gain=10.0, safety=0.9),
    ROSENBROCK: dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
                     min_gain=0.2, max_gain=8.0, safety=0.9),
    FIRK: dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
               min_gain=0.2, max_gain=8.0, safety=0.9),
    DIRK: dict(step_controller="gustafsson", deadband_min=1.0, deadband_max=1.2,
               min_gain=0.2, max_gain=8.0, safety=0.9),
}
