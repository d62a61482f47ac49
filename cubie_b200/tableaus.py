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
    # DIRK: an implicit stage that follows an explicit one starts its Newton
    # iteration from h times the explicit stage's derivative (an explicit
    # Euler predictor) instead of the last solved increment
    euler_guess: bool = False

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

    def stage_derivative_needed(self, stage: int) -> bool:
        """Whether a DIRK/ERK step must evaluate f at ``stage``'s state: a
        later stage or the output/error sums read it, it is an explicit
        stage, or it is the cached first derivative of the next step."""
        a = self.a_matrix()
        s = self.stage_count
        if a[stage, stage] == 0.0:
            return True
        if stage == s - 1 and self.first_same_as_last:
            return True
        if any(a[j, stage] != 0.0 for j in range(stage + 1, s)):
            return True
        if self.accumulates_output and self.b[stage] != 0.0:
            return True
        d = self.d
        return bool(self.has_error_estimate and self.accumulates_error and d[stage] != 0.0)

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

# Explicit Euler (ExplicitEulerStep, explicit_euler.py): one stage, order 1,
# no error estimate.
EULER = Tableau(kind=ERK, name="euler", order=1, a=((0,),), b=(1.0,), c=(0,))

# Ralston's third-order three-stage method (Math. Comp. 16, 1962); no
# embedded estimate.
RALSTON_33 = Tableau(kind=ERK, name="ralston-33", order=3,
                     a=((0, 0, 0), (0.5, 0, 0), (0, 0.75, 0)), b=(2 / 9, 1 / 3, 4 / 9), c=(0, 0.5, 0.75))

# Cash-Karp 5(4) (ACM TOMS 16, 1990): fifth-order weights propagated.
CASH_KARP_54 = Tableau(
    kind=ERK, name="cash-karp-54", order=5,
    a=((0, 0, 0, 0, 0, 0),
       (1 / 5, 0, 0, 0, 0, 0),
       (3 / 40, 9 / 40, 0, 0, 0, 0),
       (3 / 10, -9 / 10, 6 / 5, 0, 0, 0),
       (-11 / 54, 5 / 2, -70 / 27, 35 / 27, 0, 0),
       (1631 / 55296, 175 / 512, 575 / 13824, 44275 / 110592, 253 / 4096, 0)),
    b=(37 / 378, 0, 250 / 621, 125 / 594, 0, 512 / 1771),
    b_hat=(2825 / 27648, 0, 18575 / 48384, 13525 / 55296, 277 / 14336, 1 / 4),
    c=(0, 1 / 5, 3 / 10, 3 / 5, 1, 7 / 8),
)

# Runge-Kutta-Fehlberg 4(5) (NASA TR R-315, 1969): fifth-order weights
# propagated.
FEHLBERG_45 = Tableau(
    kind=ERK, name="fehlberg-45", order=5,
    a=((0, 0, 0, 0, 0, 0),
       (1 / 4, 0, 0, 0, 0, 0),
       (3 / 32, 9 / 32, 0, 0, 0, 0),
       (1932 / 2197, -7200 / 2197, 7296 / 2197, 0, 0, 0),
       (439 / 216, -8, 3680 / 513, -845 / 4104, 0, 0),
       (-8 / 27, 2, -3544 / 2565, 1859 / 4104, -11 / 40, 0)),
    b=(16 / 135, 0, 6656 / 12825, 28561 / 56430, -9 / 50, 2 / 55),
    b_hat=(25 / 216, 0, 1408 / 2565, 2197 / 4104, -1 / 5, 0),
    c=(0, 1 / 4, 3 / 8, 12 / 13, 1, 1 / 2),
)

# Backward Euler (BackwardsEulerStep, backwards_euler.py): one implicit
# stage z = h f(t + h, y + z), order 1, fixed steps.  Newton starts from the
# previous step's increment as it stands (no read-ahead scaling).
BACKWARDS_EULER = Tableau(kind=DIRK, name="backwards_euler", order=1, a=((1.0,),), b=(1.0,), c=(1.0,))

# Trapezoidal rule as an explicit-first-stage DIRK (stiffly accurate, order
# 2, fixed steps).
TRAPEZOIDAL_DIRK = Tableau(kind=DIRK, name="trapezoidal_dirk", order=2, a=((0, 0), (0.5, 0.5)), b=(0.5, 0.5),
                           c=(0, 1), dense_ratio_float32=0.39, dense_ratio_float64=1.21)

# Alexander's two-stage L-stable SDIRK (SIAM J. Numer. Anal. 14, 1977),
# gamma = 1 - 1/sqrt(2); order 2, fixed steps.
_SG = (2.0 - sqrt(2.0)) / 2.0
SDIRK_2_2 = Tableau(kind=DIRK, name="sdirk_2_2", order=2, a=((_SG, 0), (1.0 - _SG, _SG)), b=(1.0 - _SG, _SG),
                    c=(_SG, 1.0), dense_ratio_float32=1.07, dense_ratio_float64=1.21)


def _rodas3p() -> Tableau:
    """RODAS3P (Steinebach; five stages, order 3 with an order-2 embedded
    solution): the last two stage bases coincide and the solution adds
    the fifth increment, the embedded one the fourth."""
    base = (2.90625, 3.375, 0.40625)
    return Tableau(
        kind=ROSENBROCK, name="rodas3p", order=3,
        a=((0, 0, 0, 0, 0), (4 / 3, 0, 0, 0, 0), (0, 0, 0, 0, 0), (*base, 0, 0), (*base, 0, 0)),
        C=((0, 0, 0, 0, 0), (-4.0, 0, 0, 0, 0), (8.25, 6.75, 0, 0, 0), (1.21875, -5.0625, -1.96875, 0, 0),
           (4.03125, -15.1875, -4.03125, 6.0, 0)),
        b=(*base, 0.0, 1.0), b_hat=(*base, 1.0, 0.0),
        c=(0, 4 / 9, 0, 1, 1), gamma=1 / 3, gamma_stages=(1 / 3, -1 / 9, 1.0, 0.0, 0.0),
    )


def _rosenbrock23() -> Tableau:
    """Shampine-Reichelt Rosenbrock 2(3) (ode23s) in the three-stage
    increment form used by OrdinaryDiffEq's Rosenbrock23: d = 1/(2+sqrt 2),
    solution y + (K1 + K2)/d, error weights matching (h/6)(k1 - 2 k2 + k3)."""
    r2 = sqrt(2.0)
    d = 1.0 / (2.0 + r2)
    inv_d = 2.0 + r2
    return Tableau(
        kind=ROSENBROCK, name="rosenbrock23", order=2,
        a=((0, 0, 0), (0.5 * inv_d, 0, 0), (inv_d, inv_d, 0)),
        C=((0, 0, 0), (-inv_d, 0, 0), (-2.0 * inv_d, -(14.0 + 8.0 * r2), 0)),
        b=(inv_d, inv_d, 0.0), b_hat=(5.0 * r2 / 6.0 + 5.0 / 3.0, 1.0 / 3.0, -1.0 / 3.0 - r2 / 6.0),
        c=(0, 0.5, 1.0), gamma=d, gamma_stages=(d, 0.0, -d),
    )


RODAS3P = _rodas3p()
ROSENBROCK23 = _rosenbrock23()


# Kvaerno ESDIRK 3(2) and 5(4) (BIT Numer. Math. 44, 2004): explicit first
# stage, stiffly accurate; the embedded solution is the stage before last.
_KG3 = 0.4358665215
KVAERNO3 = Tableau(
    kind=DIRK, name="kvaerno3", order=3,
    a=((0, 0, 0, 0), (_KG3, _KG3, 0, 0), (0.490563388419108, 0.073570090080892, _KG3, 0),
       (0.308809969973036, 1.490563388254106, -1.235239879727145, _KG3)),
    b=(0.308809969973036, 1.490563388254106, -1.235239879727145, _KG3),
    b_hat=(0.490563388419108, 0.073570090080892, _KG3, 0.0),
    c=(0, 2 * _KG3, 1.0, 1.0), dense_ratio_float32=0.85, dense_ratio_float64=1.28,
)
_KG5 = 0.26
_KV5_ROWS = (
    (0.0,),
    (_KG5, _KG5),
    (0.13, 0.84033320996790809, _KG5),
    (0.22371961478320505, 0.47675532319799699, -0.06470895363112615, _KG5),
    (0.16648564323248321, 0.1045001884159172, 0.03631482272098715, -0.13090704451073998, _KG5),
    (0.13855640231268224, 0.0, -0.04245337201752043, 0.02446657898003141, 0.61943039072480676, _KG5),
    (0.13659751177640291, 0.0, -0.05496908796538376, -0.04118626728321046, 0.62993304899016403,
     0.06962479448202728, _KG5),
)
KVAERNO5 = Tableau(
    kind=DIRK, name="kvaerno5", order=5, a=_KV5_ROWS, b=_KV5_ROWS[6], b_hat=(*_KV5_ROWS[5], 0.0),
    c=(0.0, 2 * _KG5, 1.230333209967908, 0.895765984350076, 0.436393609858648, 1.0, 1.0),
)


def _gauss_legendre(stages: int) -> Tableau:
    """Gauss-Legendre collocation with ``stages`` nodes (order 2s; Hairer &
    Wanner II, Thm IV.5.2): nodes are the shifted Legendre roots,
    ``a[i][j]`` integrates the j-th Lagrange basis polynomial over
    ``[0, c_i]`` and ``b[j]`` over ``[0, 1]``, computed here in float64."""
    x, _ = np.polynomial.legendre.leggauss(stages)
    c = 0.5 * (x + 1.0)
    a = np.zeros((stages, stages))
    b = np.zeros(stages)
    for j in range(stages):
        basis = np.polynomial.Polynomial([1.0])
        for m in range(stages):
            if m != j:
                basis *= np.polynomial.Polynomial([-c[m], 1.0]) / (c[j] - c[m])
        prim = basis.integ()
        b[j] = prim(1.0) - prim(0.0)
        for i in range(stages):
            a[i, j] = prim(c[i]) - prim(0.0)
    return Tableau(kind=FIRK, name=f"firk_gauss_legendre_{stages}", order=2 * stages,
                   a=tuple(tuple(float(v) for v in row) for row in a), b=tuple(float(v) for v in b),
                   c=tuple(float(v) for v in c), dense_ratio_float32=8.0, dense_ratio_float64=8.0)


# Four-stage Gauss-Legendre (order 8) as the published float64 literals of
# that construction; they agree with ``_gauss_legendre(4)`` to a few ulps and
# are kept as published so results match other implementations bit for bit.
_GL4_A = (
    (0.08696371128436345, -0.026604180084998798, 0.012627462689404742, -0.003555149685795684),
    (0.188118117499868, 0.16303628871563644, -0.027880428602470995, 0.006735500594538164),
    (0.1671919219741886, 0.3539530060337439, 0.16303628871563638, -0.014190694931141147),
    (0.17748257225452202, 0.3134451147418685, 0.3526767575162713, 0.08696371128436325),
)
GAUSS_LEGENDRE_4 = Tableau(
    kind=FIRK, name="firk_gauss_legendre_4", order=8, a=_GL4_A,
    b=(0.17392742256872662, 0.32607257743127305, 0.3260725774312722, 0.1739274225687269),
    c=(0.06943184420297371, 0.33000947820757187, 0.6699905217924281, 0.9305681557970262),
    dense_ratio_float32=8.0, dense_ratio_float64=8.0,
)


# Higher-order explicit pairs.  The coefficients are the published float64
# values: Tsitouras 5(4) (Comput. Math. Appl. 62, 2011), Verner's
# "efficient" 7(6) pair (RKV76.IIa) and Dormand-Prince 8(5,3) (Hairer,
# Norsett & Wanner I, DOP853) with its fifth-order embedded weights.
_TS5_A = (
    (0.0,),
    (0.161,),
    (-0.008480655492356989, 0.335480655492357),
    (2.8971530571054935, -6.359448489975075, 4.3622954328695815),
    (5.325864828439257, -11.748883564062828, 7.4955393428898365, -0.09249506636175525),
    (5.86145544294642, -12.92096931784711, 8.159367898576159, -0.071584973281401, -0.028269050394068383),
    (0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081, 2.324710524099774),
)
_TS5_B = (0.09646076681806523, 0.01, 0.4798896504144996, 1.379008574103742, -3.290069515436081, 2.324710524099774,
          0.0)
_TS5_BHAT = (0.09824077787029101, 0.010816434459656746, 0.4720087724042376, 1.5237195812770048, -3.872426680888636,
             2.7827926300289607, -0.015151515151515152)
_TS5_C = (0.0, 0.161, 0.327, 0.9, 0.9800255409045097, 1.0, 1.0)
_VN7_A = (
    (0.0,),
    (0.005,),
    (-1.07679012345679, 1.185679012345679),
    (0.04083333333333333, 0.0, 0.1225),
    (0.6389139236255726, 0.0, -2.455672638223657, 2.272258714598084),
    (-2.6615773750187572, 0.0, 10.804513886456137, -8.3539146573962, 0.820487594956657),
    (6.067741434696771, 0.0, -24.711273635911084, 20.427517930788895, -1.9061579788166472, 1.006172249242068),
    (12.054670076253203, 0.0, -49.75478495046899, 41.142888638604674, -4.461760149974004, 2.042334822239175,
     -0.09834843665406108),
    (10.138146522881808, 0.0, -42.6411360317175, 35.76384003992257, -4.3480228403929075, 2.0098622683770357,
     0.3487490460338272, -0.27143900510483127),
    (-45.030072034298676, 0.0, 187.3272437654589, -154.02882369350186, 18.56465306347536, -7.141809679295079,
     1.3088085781613785, 0.0, 0.0),
)
_VN7_B = (0.04715561848627222, 0.0, 0.0, 0.25750564298434153, 0.2621665397741262, 0.15216092656738558,
          0.49399691700324844, -0.29430311714032503, 0.0813174723249511, 0.0)
_VN7_BHAT = (0.044608606606341174, 0.0, 0.0, 0.26716403785713727, 0.2201018300177293, 0.2188431703143157,
             0.22898717054112028, 0.0, 0.0, 0.020295184663356284)
_VN7_C = (0.0, 0.005, 0.10888888888888888, 0.16333333333333333, 0.4555, 0.6095094489978381, 0.884, 0.925, 1.0, 1.0)
_DP8_A = (
    (0.0,),
    (0.05260015195876773,),
    (0.0197250569845379, 0.0591751709536137),
    (0.02958758547680685, 0.0, 0.08876275643042054),
    (0.2413651341592667, 0.0, -0.8845494793282861, 0.924834003261792),
    (0.037037037037037035, 0.0, 0.0, 0.17082860872947386, 0.12546768756682242),
    (0.037109375, 0.0, 0.0, 0.17025221101954405, 0.06021653898045596, -0.017578125),
    (0.03709200011850479, 0.0, 0.0, 0.17038392571223998, 0.10726203044637328, -0.015319437748624402,
     0.008273789163814023),
    (0.6241109587160757, 0.0, 0.0, -3.360892629446941, -0.868219346841726, 27.592099699446706, 20.154067550477894,
     -43.48988418106996),
    (0.47766253643826434, 0.0, 0.0, -2.4881146199716677, -0.590290826836843, 21.230051448181193,
     15.279233632882423, -33.28821096898486, -0.020331201708508627),
    (-0.9371424300859873, 0.0, 0.0, 5.186372428844064, 1.0914373489967295, -8.149787010746927, -18.52006565999696,
     22.739487099350505, 2.493605552679653, -3.0467644718982196),
    (2.2733101475165385, 0.0, 0.0, -10.53449546673725, -2.0008720582248625, -17.9589318631188, 27.94888452941996,
     -2.8589982771350235, -8.87285693353063, 12.360567175794303, 0.6433927460157635),
)
_DP8_B = (0.05429373411656876, 0.0, 0.0, 0.0, 0.0, 4.450312892752409, 1.8915178993145003, -5.801203960010585,
          0.3111643669578199, -0.1521609496625161, 0.20136540080403034, 0.04471061572777259)
_DP8_BHAT = (0.04117368912237387, 0.0, 0.0, 0.0, 0.0, 5.675469339128613, 2.3872768489717506, -7.465581142465572,
             0.6614932157077936, -0.4863400683755336, 0.11944219431891465, 0.06706592359165887)
_DP8_C = (0.0, 0.05260015195876773, 0.0789002279381516, 0.1183503419072274, 0.2816496580927726, 0.3333333333333333,
          0.25, 0.3076923076923077, 0.6512820512820513, 0.6, 0.8571428571428571, 1.0)

TSIT5 = Tableau(kind=ERK, name="tsit5", order=5, a=_TS5_A, b=_TS5_B, b_hat=_TS5_BHAT, c=_TS5_C)
VERN7 = Tableau(kind=ERK, name="vern7", order=7, a=_VN7_A, b=_VN7_B, b_hat=_VN7_BHAT, c=_VN7_C)
DOP853 = Tableau(kind=ERK, name="dormand-prince-853", order=8, a=_DP8_A, b=_DP8_B, b_hat=_DP8_BHAT, c=_DP8_C)


# Crank-Nicolson (CrankNicolsonStep, crank_nicolson.py) as a three-stage
# DIRK: the explicit derivative at the step start, the trapezoidal stage
# z = h f(t + h, y + h f(y)/2 + z/2) (the solution) and a backward Euler
# stage z = h f(t + h, y + z) (the embedded first-order solution).  The
# trapezoidal solve starts from h f(y), the backward Euler one from the
# trapezoidal increment, as in the reference step.
CRANK_NICOLSON = Tableau(kind=DIRK, name="crank_nicolson", order=2,
                         a=((0, 0, 0), (0.5, 0.5, 0), (0, 0, 1.0)), b=(0.5, 0.5, 0.0), b_hat=(0.0, 0.0, 1.0),
                         c=(0, 1.0, 1.0), euler_guess=True)

# Backward Euler with an explicit Euler predictor (BackwardsEulerPCStep,
# backwards_euler_predict_correct.py): the derivative at the step start
# (the previous step's last one) seeds the Newton solve of the implicit
# stage; fixed steps.
BACKWARDS_EULER_PC = Tableau(kind=DIRK, name="backwards_euler_pc", order=1, a=((0, 0), (0, 1.0)), b=(0.0, 1.0),
                             c=(0, 1.0), euler_guess=True)

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
    "euler": EULER, "ralston-33": RALSTON_33, "cash-karp-54": CASH_KARP_54, "fehlberg-45": FEHLBERG_45,
    "backwards_euler": BACKWARDS_EULER, "trapezoidal_dirk": TRAPEZOIDAL_DIRK, "ode23t": TRAPEZOIDAL_DIRK,
    "sdirk_2_2": SDIRK_2_2, "rodas3p": RODAS3P, "rosenbrock23": ROSENBROCK23, "ode23s": ROSENBROCK23,
    "rosenbrock23_sciml": ROSENBROCK23, "kvaerno3": KVAERNO3, "kvaerno5": KVAERNO5,
    "firk_gauss_legendre_4": GAUSS_LEGENDRE_4, "tsit5": TSIT5, "Tsit5": TSIT5, "vern7": VERN7, "Vern7": VERN7,
    "dormand-prince-853": DOP853, "dop853": DOP853, "crank_nicolson": CRANK_NICOLSON,
    "backwards_euler_pc": BACKWARDS_EULER_PC,
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
